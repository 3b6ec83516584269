// NEMO Arakawa C-grid meshes (mesh.nemo_grid: cgrid): the exact C-grid
// interpolation of Delandmeter & van Sebille (2019) as numerics/nemo_cgrid.py
// states it (a T-cell is a quad of F-point corners; the face velocities give
// normal fluxes; inside the cell the logical velocity is linear along its own
// axis), the 2-D step form that reads it, and the 3-D step in the fractional
// level coordinate s = k + zeta.  Plain form: the cited Numba functions'
// float64 operation order.
#pragma once
#include "kc_step.cuh"
#include "kc_mixed.cuh"

namespace kc {

// the stage's value of a face raster at flat index idx (the payload blended
// like every field, io.py:68-117)
template <typename T>
__device__ __forceinline__ double cg_val(const T* a, const T* b, const T* t, double alpha0, double alpha,
                                         long long idx) {
    if (alpha < 1e-12) {
        const double x = (double)__ldg(&a[idx]);
        if (alpha0 == 0.0) return x;
        return (1.0 - alpha0) * x + alpha0 * (double)__ldg(&b[idx]);
    }
    if (alpha > 1.0 - 1e-12) return (double)__ldg(&t[idx]);
    return tblend((double)__ldg(&a[idx]), (double)__ldg(&b[idx]), (double)__ldg(&t[idx]), alpha0, alpha);
}

// nemo_cgrid.py:75-81 _nemo_cgrid_e3face
__device__ __forceinline__ double cg_e3face(const DCgrid& g, const int* kb, const double* e3, long long fi, int k) {
    if (k == __ldg(&kb[fi])) return __ldg(&e3[fi]);
    return __ldg(&g.zw[k + 1]) - __ldg(&g.zw[k]);
}

// Python's max(a, b) / min(a, b): the first argument unless the second is
// strictly larger / smaller
__device__ __forceinline__ double pymax(double a, double b) { return b > a ? b : a; }

// nemo_cgrid.py:84-222 _interp_nemo_cgrid_core at (xp, yp) with anchor nn:
// the containing cell (hint >= 0, else the local search), the closed-form
// bilinear inverse, the face fluxes (model widths, or each edge's plane
// length from the host table), the logical velocity; in 3-D zp is the
// fractional level s and W = ds/dt.  False outside the mesh or for a
// degenerate cell; a dry-ring cell or a level at or below the floor reads
// zero velocity.
//
// MIXED (the mixed form, 3-D): the six face / interface values are read
// (float32, or float16 with per-level scales) and time-blended in float32,
// and the fluxes formed in float32; the cell search, the bilinear inverse, the
// metric terms and positions stay float64.
template <typename T, bool MIXED = false>
static __device__ __noinline__ bool cgrid_core(const DMesh& m, const DBlend<T>& f, double alpha, double xp, double yp,
                                               double zp, int nn, int hint, double td, bool three_d, double& U,
                                               double& V, double& W) {
    U = 0.0;
    V = 0.0;
    W = 0.0;
    const DCgrid& g = m.cg;
    int e = hint;
    if (e < 0) {
        e = contain_local(m, xp, yp, nn);
        if (e < 0) return false;
    }
    const int nl = __ldg(&g.nlev[e]);
    if (nl <= 0) return true;
    const long long nx = g.nx;
    const long long c = __ldg(&g.cell[e]);
    int kz = 0;
    long long nynx = 0;
    double fW = 1.0, fE = 1.0, fS = 1.0, fN = 1.0, e3c = 1.0;
    if (three_d) {
        nynx = g.nynx;
        if (zp >= (double)nl) return true;
        kz = (int)floor(zp);
        if (kz < 0) kz = 0;
        if (kz > g.K - 1) kz = g.K - 1;
        e3c = __ldg(&g.zw[kz + 1]) - __ldg(&g.zw[kz]);
        if (kz == nl - 1) e3c = __ldg(&g.e3b[c]);
        fW = cg_e3face(g, g.kbu, g.e3u, c - 1, kz) / e3c;
        fE = cg_e3face(g, g.kbu, g.e3u, c, kz) / e3c;
        fS = cg_e3face(g, g.kbv, g.e3v, c - nx, kz) / e3c;
        fN = cg_e3face(g, g.kbv, g.e3v, c, kz) / e3c;
    }
    const long long ko = (long long)kz * nynx;
    double uW, uE, vS, vN;
    TBlendF tb;
    if constexpr (MIXED) {
        tb = tblend_mode(f.alpha0, alpha);
        const long long rn = nynx > 0 ? nynx : 0;
        uW = (double)blend_val<T>(tb, f.a.u, f.a.su, f.b.u, f.b.su, f.t.u, f.t.su, kz, rn, (int)(c - 1));
        uE = (double)blend_val<T>(tb, f.a.u, f.a.su, f.b.u, f.b.su, f.t.u, f.t.su, kz, rn, (int)c);
        vS = (double)blend_val<T>(tb, f.a.v, f.a.sv, f.b.v, f.b.sv, f.t.v, f.t.sv, kz, rn, (int)(c - nx));
        vN = (double)blend_val<T>(tb, f.a.v, f.a.sv, f.b.v, f.b.sv, f.t.v, f.t.sv, kz, rn, (int)c);
    } else {
        uW = cg_val(f.a.u, f.b.u, f.t.u, f.alpha0, alpha, ko + c - 1);
        uE = cg_val(f.a.u, f.b.u, f.t.u, f.alpha0, alpha, ko + c);
        vS = cg_val(f.a.v, f.b.v, f.t.v, f.alpha0, alpha, ko + c - nx);
        vN = cg_val(f.a.v, f.b.v, f.t.v, f.alpha0, alpha, ko + c);
    }
    const double M = SLM;
    const double cosl = cr::cos_cr(yp * DEG2RAD);
    const int4 cr = __ldg(&g.corners[e]);
    double px[4], py[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int nd = k == 0 ? cr.x : (k == 1 ? cr.y : (k == 2 ? cr.z : cr.w));
        const double2 ll = __ldg(&m.ll[nd]);
        px[k] = wrap180(ll.x - xp) * cosl * M;
        py[k] = (ll.y - yp) * M;
    }
    const double a0 = px[0], a1 = px[1] - px[0], a2 = px[3] - px[0], a3 = px[0] - px[1] + px[2] - px[3];
    const double b0 = py[0], b1 = py[1] - py[0], b2 = py[3] - py[0], b3 = py[0] - py[1] + py[2] - py[3];
    const double scale = pymax(pymax(pymax(pymax(fabs(a1), fabs(a2)), fabs(b1)), fabs(b2)), 1e-30);
    const double aa = a3 * b2 - a2 * b3;
    const double bb = a3 * b0 - a0 * b3 + a1 * b2 - a2 * b1;
    const double cc = a1 * b0 - a0 * b1;
    double eta;
    if (fabs(aa) < 1e-12 * scale * scale) {
        if (fabs(bb) < 1e-300) return false;
        eta = -cc / bb;
    } else {
        double disc = bb * bb - 4.0 * aa * cc;
        if (disc < 0.0) disc = 0.0;
        const double sq = sqrt(disc);
        const double r1 = (-bb + sq) / (2.0 * aa);
        const double r2 = (-bb - sq) / (2.0 * aa);
        const double d1 = pymax(pymax(0.0, -r1), r1 - 1.0);
        const double d2 = pymax(pymax(0.0, -r2), r2 - 1.0);
        eta = d1 <= d2 ? r1 : r2;
    }
    eta = pymin(pymax(eta, 0.0), 1.0);
    const double den = a1 + a3 * eta, den2 = b1 + b3 * eta;
    double xi = fabs(den) >= fabs(den2) ? (0.0 - a0 - a2 * eta) / den : (0.0 - b0 - b2 * eta) / den2;
    xi = pymin(pymax(xi, 0.0), 1.0);
    double U0, U1, V0, V1;
    double lW, lE, lS, lN;
    if (g.has_e) {
        lW = __ldg(&g.e2u[c - 1]);
        lE = __ldg(&g.e2u[c]);
        lS = __ldg(&g.e1v[c - nx]);
        lN = __ldg(&g.e1v[c]);
    } else {   // edges S (c0-c1), E (c1-c2), N (c2-c3), W (c3-c0)
        const double4 L = g.L[e];
        lW = L.w;
        lE = L.y;
        lS = L.x;
        lN = L.z;
    }
    if constexpr (MIXED) {
        U0 = (double)((float)fW * (float)uW * (float)lW);
        U1 = (double)((float)fE * (float)uE * (float)lE);
        V0 = (double)((float)fS * (float)vS * (float)lS);
        V1 = (double)((float)fN * (float)vN * (float)lN);
    } else {
        U0 = fW * uW * lW;
        U1 = fE * uE * lE;
        V0 = fS * vS * lS;
        V1 = fN * vN * lN;
    }
    const double dxdxi = (1.0 - eta) * a1 + eta * (px[2] - px[3]);
    const double dydxi = (1.0 - eta) * b1 + eta * (py[2] - py[3]);
    const double dxdeta = (1.0 - xi) * a2 + xi * (px[2] - px[1]);
    const double dydeta = (1.0 - xi) * b2 + xi * (py[2] - py[1]);
    const double det = dxdxi * dydeta - dxdeta * dydxi;
    const double adet = fabs(det);
    if (adet < 1e-12 * scale * scale) return false;
    const double dxi = ((1.0 - xi) * U0 + xi * U1) / adet;
    const double deta = ((1.0 - eta) * V0 + eta * V1) / adet;
    const double Uv = dxdxi * dxi + dxdeta * deta;
    const double Vv = dydxi * dxi + dydeta * deta;
    double Wv = 0.0;
    if (three_d) {
        const double zeta = pymin(pymax(zp - kz, 0.0), 1.0);
        if constexpr (MIXED) {
            const float wl = blend_val<T>(tb, f.a.w, f.a.sw, f.b.w, f.b.sw, f.t.w, f.t.sw, kz, nynx, (int)c);
            const float wu = blend_val<T>(tb, f.a.w, f.a.sw, f.b.w, f.b.sw, f.t.w, f.t.sw, kz + 1, nynx, (int)c);
            const float zf = (float)zeta;
            Wv = (double)((1.0f - zf) * wl + zf * wu) * __ldg(&g.area[c]) / (adet * e3c);
        } else {
            Wv = ((1.0 - zeta) * cg_val(f.a.w, f.b.w, f.t.w, f.alpha0, alpha, ko + c) +
                  zeta * cg_val(f.a.w, f.b.w, f.t.w, f.alpha0, alpha, ko + nynx + c)) *
                 __ldg(&g.area[c]) / (adet * e3c);
        }
    }
    U = td * Uv;
    V = td * Vv;
    W = td * Wv;
    return true;
}

// The 2-D step form of a C-grid mesh (numerics/nemo_cgrid.py:355-388
// interp_nemo_cgrid: the surface faces), for step2d_particle.
template <typename T>
struct CgridForm {
    static constexpr bool kExact = true;
    static __device__ __forceinline__ Site site(double lon, double lat) { return make_site_fast(lon, lat); }
    static __device__ __forceinline__ bool uv2(const DMesh& m, const DBlend<T>& f, const DStep& s, double lon,
                                               double lat, int nn, int hint, double alpha, double& U, double& V) {
        double W;
        return cgrid_core<T>(m, f, alpha, lon, lat, 0.0, nn, hint, s.time_dir, false, U, V, W);
    }
};

// nemo_cgrid.py:391-402 _cell_thickness: the clipped level and its
// thickness in cell e (ok: found; raster cell 0 otherwise)
__device__ __forceinline__ double cg_cell(const DCgrid& g, int e, bool ok, int& k) {
    const long long c = ok ? __ldg(&g.cell[e]) : 0;
    const int nl = __ldg(&g.nlev_r[c]);
    if (k < 0) k = 0;
    if (k > g.K - 1) k = g.K - 1;
    return (k == nl - 1 && g.shrunk) ? __ldg(&g.e3b[c]) : __ldg(&g.zw[k + 1]) - __ldg(&g.zw[k]);
}

// nemo_cgrid.py:405-413 _level_coord: z -> s (searchsorted right, minus one)
__device__ __forceinline__ double cg_z2s(const DCgrid& g, int e, bool ok, double z) {
    int k = 0;
    if (isnan(z)) k = g.K;
    else
        while (k < g.K + 1 && __ldg(&g.zw[k]) <= z) ++k;
    k -= 1;
    const double e3 = cg_cell(g, e, ok, k);
    return k + (z - __ldg(&g.zw[k])) / e3;
}

// ... and s -> z
__device__ __forceinline__ double cg_s2z(const DCgrid& g, int e, bool ok, double s) {
    int k = (int)floor(s);
    const double e3 = cg_cell(g, e, ok, k);
    return __ldg(&g.zw[k]) + (s - k) * e3;
}

// nemo_cgrid.py:416-512 nemo_cgrid3d_step for one particle: Euler / RK2
// (midpoint) / RK4 in the fractional level s of the start cell, stage n at
// x0 + a_n k_{n-1}, the weighted sum of the stage increments, s clamped at
// the surface, the end cell's domain check and s -> z (an unchanged s in an
// unchanged cell keeps z).  A particle that is not alive gets the nearest
// node of its position and nothing else.
template <typename T, int SCHEME, bool MIXED = false>
__device__ __forceinline__ void step3d_cgrid_particle(const DMesh& m, const DBlend<T>& f, const DState& st,
                                                      const DStep& s, long long i) {
    constexpr int NS = SCHEME == 0 ? 1 : (SCHEME == 1 ? 2 : 4);
    const double lon0 = st.lon[i], lat0 = st.lat[i], z0 = st.z[i];
    const Site q0 = make_site_fast(lon0, lat0);   // the anchor search only: positions use cos_cr below
    const int nn0 = start_anchor(m, st, q0, st.nn[i], i);
    if (st.status[i] != ALIVE) {
        st.U[i] = 0.0;
        st.V[i] = 0.0;
        st.W[i] = 0.0;
        st.nn[i] = nn0;
        if (st.nn_ok) st.nn_ok[i] = 1;
        return;
    }
    const DCgrid& g = m.cg;
    const double dt = s.dt;
    const int e0 = contain_local(m, lon0, lat0, nn0);
    const bool ok0 = e0 >= 0;
    const double s0 = cg_z2s(g, e0, ok0, z0);
    double k0 = 0.0, k1 = 0.0, k2 = 0.0;   // the previous stage's increments
    double d0 = 0.0, d1 = 0.0, d2 = 0.0;   // their weighted sum
    double first_u = 0.0, first_v = 0.0, first_w = 0.0;
    bool ok = true;
#pragma unroll
    for (int n = 0; n < NS; ++n) {
        double ln = lon0, lt = lat0, sn = s0;
        if (n) {
            const double a = (SCHEME == 2 && n == 3) ? 1.0 : 0.5;
            ln = wrap180(lon0 + a * k0);
            lt = clamp_lat(lat0 + a * k1);
            sn = s0 + a * k2;
        }
        double Un = 0.0, Vn = 0.0, Wn = 0.0;
        if (ok) {
            const int nnn = n ? site_anchor(m, make_site_fast(ln, lt)) : nn0;
            ok = cgrid_core<T, MIXED>(m, f, s.ak[n], ln, lt, sn, nnn, n ? -1 : (ok0 ? e0 : -1), s.time_dir, true,
                                      Un, Vn, Wn);
        }
        if (n == 0) {
            first_u = Un;
            first_v = Vn;
            first_w = Wn;
        }
        double z0n = cr::cos_cr(lt * DEG2RAD) * SLM;
        if (z0n < 1.0) z0n = 1.0;
        k0 = dt * Un / z0n;
        k1 = dt * Vn / SLM;
        k2 = dt * Wn;
        const double b = SCHEME == 0 ? 1.0 : (SCHEME == 1 ? (n == 0 ? 0.0 : 1.0) : ((n == 0 || n == 3) ? 1.0 / 6 : 1.0 / 3));
        d0 += b * k0;
        d1 += b * k1;
        d2 += b * k2;
    }
    double ln = lon0, lt = lat0, sv = s0;
    if (ok) {
        ln = wrap180(lon0 + d0);
        lt = clamp_lat(lat0 + d1);
        sv = s0 + d2;
        if (sv < 0.0) sv = 0.0;
    }
    int nne = site_anchor(m, make_site_fast(ln, lt));
    const int e1 = contain_local(m, ln, lt, nne);
    const bool in_dom = e1 >= 0;
    double zn = z0;
    int status = ALIVE;
    signed char fr = st.fr[i];
    if (!ok || !in_dom) {
        ln = lon0;
        lt = lat0;
        nne = nn0;
        status = OUTSIDE;
        fr = !ok ? FR_INTERP : FR_OOB;
    } else if (!(sv == s0 && e1 == e0)) {
        zn = cg_s2z(g, e1, in_dom, sv);
    }
    int kk = (int)floor(s0);
    const double e3 = cg_cell(g, e0, ok0, kk);
    st.U[i] = first_u;
    st.V[i] = first_v;
    st.W[i] = first_w * e3;
    st.lon[i] = ln;
    st.lat[i] = lt;
    st.z[i] = zn;
    st.status[i] = status;
    st.nn[i] = nne;
    st.fr[i] = fr;
    if (st.nn_ok) st.nn_ok[i] = 1;
}

}  // namespace kc
