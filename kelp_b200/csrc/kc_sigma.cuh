// Sigma meshes (mesh.vertical_coord "sigma", FESOM-C): the 3-D step that
// integrates the particle's sigma fraction s = z / H_p, H_p the water column
// max(depth + eta, Dmin) interpolated at the particle with the W method, so
// the free surface and the bottom slope carry the particle exactly
// (integrators.py:1322-1440).  Every stage places the particle at
// z = s * H_p(x_stage, t_stage), reads u/v in its own layer (or, depth-linear,
// at s itself), and the W of the stage's column; the end of the step sits in
// the end-of-step column and is clamped there.  Plain form only: the same
// float64 operation order as the cited Numba functions.
#pragma once
#include "kc_step.cuh"

namespace kc {

// The stage's free surface at a node: the payload's eta blended in time like
// u/v (io.py:68-117 _blend in float64; the stage lerps of _make_stage_vels).
template <typename T>
__device__ __forceinline__ double eta_at(const DBlend<T>& f, int node, double alpha) {
    if (f.pchip)
        return pchip4(__ldg(&f.a.eta[node]), __ldg(&f.b.eta[node]), __ldg(&f.t.eta[node]), __ldg(&f.d.eta[node]), f.pt,
                      alpha);
    if (alpha < 1e-12) {
        const double a = __ldg(&f.a.eta[node]);
        if (f.alpha0 == 0.0) return a;
        return (1.0 - f.alpha0) * a + f.alpha0 * __ldg(&f.b.eta[node]);
    }
    if (alpha > 1.0 - 1e-12) return __ldg(&f.t.eta[node]);
    return tblend(__ldg(&f.a.eta[node]), __ldg(&f.b.eta[node]), __ldg(&f.t.eta[node]), f.alpha0, alpha);
}

// The free surface at a node at one instant of the step (integrators.py:
// 1358-1441, the sigma branches :5031-5079, :5424-5436, :5797-5815): slot 0
// the start, 1..3 the RK stages (c = 0.5, 0.5, 1 for RK4; 0.5 for RK2), 4 the
// end of the step (also the column of the split kick).  The tracking layer's
// surfaces replace the payload's own where it supplies them (s.eta_s at the
// start, s.eta_e at the end); a steady step (no next snapshot, no PCHIP)
// blends its stages from the start towards the end surface as
// _eta_blend does ((1 - c) a + c b), a time-aware step reads each stage
// field's own surface.
template <typename T>
__device__ __forceinline__ double eta_src(const DBlend<T>& f, const DStep& s, int node, int slot) {
    if (slot != 0 && !s.sig_steady && !(slot == 4 && s.eta_e))
        return eta_at(f, node, slot == 4 ? s.alpha_end : s.ak[slot]);
    const double e0 = s.eta_s ? __ldg(&s.eta_s[node]) : eta_at(f, node, s.ak[0]);
    if (slot == 0) return e0;
    const double e1 = s.eta_e ? __ldg(&s.eta_e[node]) : e0;
    if (slot == 4 || slot == 3) return e1;
    return (1.0 - 0.5) * e0 + 0.5 * e1;
}

// vertical_sigma.py:472-478 _col_H
template <typename T>
__device__ __forceinline__ double col_H(const DMesh& m, const DBlend<T>& f, const DStep& s, int node, int slot) {
    double H = __ldg(&m.depth[node]) + eta_src(f, s, node, slot);
    if (H < s.Dmin) H = s.Dmin;
    return H;
}

// The particle's column height from the anchor's 1-ring of node columns
// (vertical.py:447-485 order), as the W methods interpolate it: the
// least-squares plane (w_code 2, vertical_sigma.py:493-531 _H_leastsq_single,
// floored at Dmin) or the inverse-distance mean (3, :534-563 _H_idw_single;
// a node within 1 m gives its own column); the anchor's column where the
// fit fails.
template <typename T>
static __device__ __noinline__ double H_ring(const DMesh& m, const DBlend<T>& f, const DStep& s, int slot, double xp,
                                             double yp, int node) {
    double z0 = cr::cos_cr(yp * DEG2RAD) * SLM;
    if (z0 < 1.0) z0 = 1.0;
    if (s.w_code == 3) {
        double sw = 0.0, swh = 0.0, hit = 0.0;
        bool is_hit = false;
        for_ring(m, node, [&](int nd) {
            const double h = col_H(m, f, s, nd, slot);
            const double2 p = __ldg(&m.ll[nd]);
            const double dx = wrap180(p.x - xp) * z0;
            const double dy = (p.y - yp) * SLM;
            const double d2 = dx * dx + dy * dy;
            if (d2 < 1.0) {
                is_hit = true;
                hit = h;
                return false;
            }
            sw += 1.0 / d2;
            swh += h / d2;
            return true;
        });
        if (is_hit) return hit;
        if (sw < 1e-30) return col_H(m, f, s, node, slot);
        return swh / sw;
    }
    double a11 = 0.0, a12 = 0.0, a13 = 0.0, a22 = 0.0, a23 = 0.0, a33 = 0.0, fw = 0.0, f1w = 0.0, f2w = 0.0;
    const int cnt = for_ring(m, node, [&](int nd) {
        const double h = col_H(m, f, s, nd, slot);
        const double2 p = __ldg(&m.ll[nd]);
        const double ex = wrap180(p.x - xp) * z0;
        const double ey = (p.y - yp) * SLM;
        a11 += 1.0;
        a12 += ex;
        a13 += ey;
        a22 += ex * ex;
        a23 += ex * ey;
        a33 += ey * ey;
        fw += h;
        f1w += h * ex;
        f2w += h * ey;
        return true;
    });
    if (cnt < 3) return col_H(m, f, s, node, slot);
    const double a21 = a12, a31 = a13, a32 = a23;
    const double det = a11 * a22 * a33 + a12 * a23 * a31 + a13 * a21 * a32 - a13 * a22 * a31 - a12 * a21 * a33 -
                       a11 * a23 * a32;
    if (fabs(det) < 1e-30 || fabs(det) < 1e-12 * fabs(a11 * a22 * a33)) return col_H(m, f, s, node, slot);
    const double inv = 1.0 / fabs(det);
    const double b11 = a22 * a33 - a23 * a32, b12 = a13 * a32 - a12 * a33, b13 = a12 * a23 - a13 * a22;
    double H = (b11 * fw + b12 * f1w + b13 * f2w) * inv;
    if (H < s.Dmin) H = s.Dmin;
    return H;
}

// One evaluation site of the sigma step: the W method's element and vertex
// weights (vertical_sigma.py:565-632 _bary_locate, nv = 0 for the nearest
// method or when no element of the anchor contains the point), the vertex
// columns, and the particle's column H (vertical_sigma.py:1034-1060).
struct SigSite {
    int nv;
    int v[4];
    double w[4];
    double Hv[4];
    double H;
};

// The element search is the barycentric W's own (w_search_elem: first
// element of the anchor's 1-ring with a fan triangle whose weights are all
// >= -1e-6, frame of mesh.py:1973-2003); its weights are the accepting
// triangle's for a triangle and Wachspress for a quad.
template <typename T>
static __device__ __noinline__ void sigma_site(const DMesh& m, const DBlend<T>& f, const DStep& s, int slot,
                                               double xp, double yp, int node, SigSite& q) {
    q.nv = 0;
    if (s.w_code >= 2) {
        q.H = H_ring<T>(m, f, s, slot, xp, yp, node);
        return;
    }
    if (s.w_code == 1) {
        const int el = w_search_elem(m, xp, yp, node);
        if (el >= 0) {
            Ring r;
            load_ring(m, __ldg(&m.en[el]), r);
            const int nvv = r.n;
            double lmin = fmin(fmin(r.ln[0], r.ln[1]), r.ln[2]), lmax = fmax(fmax(r.ln[0], r.ln[1]), r.ln[2]);
            if (nvv == 4) { lmin = fmin(lmin, r.ln[3]); lmax = fmax(lmax, r.ln[3]); }
            double lon0;
            if (lmax - lmin > 180.0) {
                double d = 0.0;
                for (int v = 0; v < nvv; ++v) d += wrap180(r.ln[v] - r.ln[0]);
                lon0 = r.ln[0] + d / (double)nvv;
            } else {
                double sm = 0.0;
                for (int v = 0; v < nvv; ++v) sm += r.ln[v];
                lon0 = sm / (double)nvv;
            }
            double lat0 = 0.0;
            for (int v = 0; v < nvv; ++v) lat0 += r.la[v];
            lat0 /= (double)nvv;
            const double cos_lat0 = __ldg(&m.ecos[el]).y;
            const double R = 6371000.0;
            double vx[4], vy[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                vx[v] = wrap180(r.ln[v] - lon0) * DEG2RAD * R * cos_lat0;
                vy[v] = (r.la[v] - lat0) * DEG2RAD * R;
            }
            const double px = wrap180(xp - lon0) * DEG2RAD * R * cos_lat0;
            const double py = (yp - lat0) * DEG2RAD * R;
            if (nvv == 4) {
                wachspress_quad(px, py, vx, vy, q.w);
            } else {
                const double ax = vx[0], ay = vy[0], bx = vx[1], by = vy[1], cx = vx[2], cy = vy[2];
                const double denom = (by - cy) * (ax - cx) + (cx - bx) * (ay - cy);
                q.w[0] = ((by - cy) * (px - cx) + (cx - bx) * (py - cy)) / denom;
                q.w[1] = ((cy - ay) * (px - cx) + (ax - cx) * (py - cy)) / denom;
                q.w[2] = 1.0 - q.w[0] - q.w[1];
                q.w[3] = 0.0;
            }
            double H = 0.0;
            for (int v = 0; v < nvv; ++v) {
                q.v[v] = r.v[v];
                q.Hv[v] = col_H(m, f, s, r.v[v], slot);
                H += q.w[v] * q.Hv[v];
            }
            q.nv = nvv;
            q.H = H;
            return;
        }
    }
    q.H = col_H(m, f, s, node, slot);
}

// vertical_sigma.py:297-334: the interface bracket of depth z in a column of
// height H (level k alone when a < 0)
__device__ __forceinline__ WLoc sig_locate(const DMesh& m, double z, double H) {
    const int K = m.K;
    const double* sg = m.sigma;
    if (K < 2) return {0, -1.0};
    if (z <= (1.0 - __ldg(&sg[0])) * H) return {0, -1.0};
    if (z >= (1.0 - __ldg(&sg[K - 1])) * H) return {K - 1, -1.0};
    int k = K - 2;
    for (int j = 0; j < K - 1; ++j)
        if (z < (1.0 - __ldg(&sg[j + 1])) * H) { k = j; break; }
    const double zk = (1.0 - __ldg(&sg[k])) * H, zk1 = (1.0 - __ldg(&sg[k + 1])) * H;
    const double dz = zk1 - zk;
    if (dz < 1e-12) return {k, -1.0};
    return {k, (z - zk) / dz};
}

// vertical_sigma.py:481-489 _sigma_frac
__device__ __forceinline__ double sigma_frac(double z, double H) {
    double fr = z / H;
    if (fr < 0.0) fr = 0.0;
    else if (fr > 1.0) fr = 1.0;
    return fr;
}

// W of a sigma stage (vertical_sigma.py:971-1031): nearest = the anchor's
// column at z (:337-360); barycentric = every vertex column at the
// particle's sigma (:766-816), the own column at min(z, H) outside every
// element.
// W by the 1-ring (vertical_sigma.py:656-765 _interp_w_sigma_leastsq_single,
// :820-905 _interp_w_sigma_idw_single): every node's column sampled at the
// particle's sigma z / Hp (Hp the site's column by the same method), the
// plane fit or the inverse-distance mean; the anchor's own column at
// min(z, H) where the fit fails.
template <typename T>
static __device__ __noinline__ double w_sig_ring(const DMesh& m, const DBlend<T>& f, const DStep& s, int slot,
                                                 double alpha, double xp, double yp, double z, int node, double Hp) {
    const double td = s.time_dir;
    auto own = [&]() {
        const double H = col_H(m, f, s, node, slot);
        return w_at(f, alpha, sig_locate(m, z < H ? z : H, H), node, td);
    };
    double z0 = cr::cos_cr(yp * DEG2RAD) * SLM;
    if (z0 < 1.0) z0 = 1.0;
    const double fr = sigma_frac(z, Hp);
    if (s.w_code == 3) {
        double sw = 0.0, swv = 0.0, hit = 0.0;
        bool is_hit = false;
        for_ring(m, node, [&](int nd) {
            const double H = col_H(m, f, s, nd, slot);
            const double wv = w_at(f, alpha, sig_locate(m, fr * H, H), nd, td);
            const double2 p = __ldg(&m.ll[nd]);
            const double dx = wrap180(p.x - xp) * z0;
            const double dy = (p.y - yp) * SLM;
            const double d2 = dx * dx + dy * dy;
            if (d2 < 1.0) {
                is_hit = true;
                hit = wv;
                return false;
            }
            const double wt = 1.0 / d2;
            sw += wt;
            swv += wt * wv;
            return true;
        });
        if (is_hit) return hit;
        if (sw < 1e-30) return own();
        return swv / sw;
    }
    double a11 = 0.0, a12 = 0.0, a13 = 0.0, a22 = 0.0, a23 = 0.0, a33 = 0.0, fw = 0.0, f1w = 0.0, f2w = 0.0;
    const int cnt = for_ring(m, node, [&](int nd) {
        const double H = col_H(m, f, s, nd, slot);
        const double wv = w_at(f, alpha, sig_locate(m, fr * H, H), nd, td);
        const double2 p = __ldg(&m.ll[nd]);
        const double ex = wrap180(p.x - xp) * z0;
        const double ey = (p.y - yp) * SLM;
        a11 += 1.0;
        a12 += ex;
        a13 += ey;
        a22 += ex * ex;
        a23 += ex * ey;
        a33 += ey * ey;
        fw += wv;
        f1w += wv * ex;
        f2w += wv * ey;
        return true;
    });
    if (cnt < 3) return own();
    const double a21 = a12, a31 = a13, a32 = a23;
    const double det = a11 * a22 * a33 + a12 * a23 * a31 + a13 * a21 * a32 - a13 * a22 * a31 - a12 * a21 * a33 -
                       a11 * a23 * a32;
    if (fabs(det) < 1e-30 || fabs(det) < 1e-12 * fabs(a11 * a22 * a33)) return own();
    const double inv = 1.0 / fabs(det);
    const double b11 = a22 * a33 - a23 * a32, b12 = a13 * a32 - a12 * a33, b13 = a12 * a23 - a13 * a22;
    return (b11 * fw + b12 * f1w + b13 * f2w) * inv;
}

template <typename T>
__device__ __forceinline__ double w_sig(const DMesh& m, const DBlend<T>& f, const DStep& s, int slot, double xp,
                                        double yp, double z, int node, const SigSite& q) {
    const double alpha = slot == 4 ? s.alpha_end : s.ak[slot];
    if (s.w_code >= 2) return w_sig_ring<T>(m, f, s, slot, alpha, xp, yp, z, node, q.H);
    if (q.nv == 0) {
        const double zc = (s.w_code == 0 || z < q.H) ? z : q.H;
        return w_at(f, alpha, sig_locate(m, zc, q.H), node, s.time_dir);
    }
    const double fr = sigma_frac(z, q.H);
    double acc = 0.0;
    for (int v = 0; v < q.nv; ++v)
        acc += q.w[v] * w_at(f, alpha, sig_locate(m, fr * q.Hv[v], q.Hv[v]), q.v[v], s.time_dir);
    return acc;
}

// vertical_sigma.py:73-109 find_layer_sigma in the particle's column (its
// height floored at Dmin first, :135-144)
__device__ __forceinline__ int find_layer_sig(const DMesh& m, double z, double H, double Dmin) {
    if (H < Dmin) H = Dmin;
    const int K = m.K;
    const double* sg = m.sigma;
    if (K < 2) return 0;
    if (z <= (1.0 - __ldg(&sg[0])) * H) return 0;
    if (z >= (1.0 - __ldg(&sg[K - 1])) * H) return K - 2;
    for (int k = 0; k < K - 1; ++k)
        if (z < (1.0 - __ldg(&sg[k + 1])) * H) return k;
    return K - 2;
}

// vertical_sigma.py:236-255: surface at 0, bottom z0b_min above the column's bed
__device__ __forceinline__ double clamp_sig(double z, double H, const DStep& s) {
    if (H < s.Dmin) H = s.Dmin;
    if (z < 0.0) z = 0.0;
    double bottom = H - s.z0b_min;
    if (bottom < 0.0) bottom = 0.0;
    if (z > bottom) z = bottom;
    return z;
}

// integrators.py:1351-1376 _sigma_frac_for_uv (a NaN stays NaN)
__device__ __forceinline__ double sfrac_uv(double z, double H) {
    double fr = z / H;
    if (fr < 0.0) fr = 0.0;
    if (fr > 1.0) fr = 1.0;
    return fr;
}

// u/v and W of one sigma stage at depth z with the site's column: the layer
// in the particle's column, or depth-linear u/v read at s
// (vertical_uv.py:196-211); hint >= 0 is the edge walk's element.
template <typename T>
__device__ __forceinline__ bool sig_stage(const DMesh& m, const DBlend<T>& f, const DStep& s, double lon, double lat,
                                          int nn, int hint, double z, int slot, const SigSite& q, double& U,
                                          double& V, double& W) {
    const double alpha = s.ak[slot];
    bool ok;
    if (s.uv_dl) ok = interp_uv_bary_dl<T>(m, f, lon, lat, nn, hint, sfrac_uv(z, q.H), s.time_dir, alpha, U, V);
    else ok = interp_uv_bary<T>(m, f, lon, lat, nn, hint, s.time_dir, find_layer_sig(m, z, q.H, s.Dmin), alpha, U, V);
    W = w_sig<T>(m, f, s, slot, lon, lat, z, nn, q);
    return ok;
}

// One particle of the sigma step: integrators.py:4997-5147 (Euler),
// :5380-5608 (RK2, unfused), :5760-6011 (RK4, unfused), their sigma
// branches; the split kick keeps s = z / H_p into the kicked column
// (:783-803).  A failure reverts to the start with the start anchor.
template <typename T, int SCHEME, bool WALK>
__device__ __forceinline__ void step3d_sigma_particle(const DMesh& m, const DBlend<T>& f, const DState& st,
                                                      const DStep& s, long long i) {
    int status = st.status[i];
    if (status != ALIVE) {
        st.U[i] = 0.0;
        st.V[i] = 0.0;
        st.W[i] = 0.0;
        return;
    }
    const double lon0 = st.lon[i], lat0 = st.lat[i], z0p = st.z[i];
    const int pre_nn = st.nn[i];
    const double dt = s.dt;
    signed char fr = st.fr[i];
    double lon_new = lon0, lat_new = lat0, z_new = z0p;
    const Site q0 = make_site(lon0, lat0);
    const int node_i = start_anchor(m, st, q0, pre_nn, i);
    int nn_out = node_i;
    const int e1 = stage_elem<WALK>(m, lon0, lat0, WALK ? st.elem[i] : -1, node_i);
    int e_last = e1, e_out = e1;

    SigSite c1;
    sigma_site<T>(m, f, s, 0, lon0, lat0, node_i, c1);
    double U1, V1, W1;
    bool ok = sig_stage<T>(m, f, s, lon0, lat0, node_i, e1, z0p, 0, c1, U1, V1, W1);
    st.U[i] = U1;
    st.V[i] = V1;
    st.W[i] = W1;
    double a = lon0, b = lat0, s_new = 0.0;
    if (ok) {
        if (SCHEME == 0) {
            a = wrap180(lon0 + dt * U1 / metric_z0(q0));
            b = clamp_lat(lat0 + dt * V1 / SLM);
            s_new = (z0p + W1 * dt) / c1.H;
        } else if (SCHEME == 1) {
            const double lm = wrap180(lon0 + 0.5 * dt * U1 / metric_z0(q0));
            const double tm = clamp_lat(lat0 + 0.5 * dt * V1 / SLM);
            const double s_mid = (z0p + W1 * 0.5 * dt) / c1.H;
            const Site qm = make_site(lm, tm);
            const int nm = site_anchor(m, qm);
            e_last = stage_elem<WALK>(m, lm, tm, e1, nm);
            SigSite c2;
            sigma_site<T>(m, f, s, 1, lm, tm, nm, c2);
            const double zm = s_mid * c2.H;
            double U2, V2, W2;
            if (!sig_stage<T>(m, f, s, lm, tm, nm, e_last, zm, 1, c2, U2, V2, W2)) {
                ok = false;
            } else {
                a = wrap180(lon0 + dt * U2 / metric_z0(qm));
                b = clamp_lat(lat0 + dt * V2 / SLM);
                s_new = z0p / c1.H + dt * W2 / c2.H;
            }
        } else {
            const double dl1 = dt * U1 / metric_z0(q0), dd1 = dt * V1 / SLM;
            const double s0 = z0p / c1.H, f1 = W1 / c1.H;
            const double l2 = wrap180(lon0 + 0.5 * dl1), t2 = clamp_lat(lat0 + 0.5 * dd1);
            const Site q2 = make_site(l2, t2);
            const int n2 = site_anchor(m, q2);
            const int e2 = stage_elem<WALK>(m, l2, t2, e1, n2);
            SigSite c;
            sigma_site<T>(m, f, s, 1, l2, t2, n2, c);
            double U2, V2, W2;
            if (!sig_stage<T>(m, f, s, l2, t2, n2, e2, (s0 + 0.5 * dt * f1) * c.H, 1, c, U2, V2, W2)) {
                ok = false;
            } else {
                const double dl2 = dt * U2 / metric_z0(q2), dd2 = dt * V2 / SLM, f2 = W2 / c.H;
                const double l3 = wrap180(lon0 + 0.5 * dl2), t3 = clamp_lat(lat0 + 0.5 * dd2);
                const Site q3 = make_site(l3, t3);
                const int n3 = site_anchor(m, q3);
                const int e3 = stage_elem<WALK>(m, l3, t3, e2, n3);
                sigma_site<T>(m, f, s, 2, l3, t3, n3, c);
                double U3, V3, W3;
                if (!sig_stage<T>(m, f, s, l3, t3, n3, e3, (s0 + 0.5 * dt * f2) * c.H, 2, c, U3, V3, W3)) {
                    ok = false;
                } else {
                    const double dl3 = dt * U3 / metric_z0(q3), dd3 = dt * V3 / SLM, f3 = W3 / c.H;
                    const double l4 = wrap180(lon0 + dl3), t4 = clamp_lat(lat0 + dd3);
                    const Site q4 = make_site(l4, t4);
                    const int n4 = site_anchor(m, q4);
                    e_last = stage_elem<WALK>(m, l4, t4, e3, n4);
                    sigma_site<T>(m, f, s, 3, l4, t4, n4, c);
                    double U4, V4, W4;
                    if (!sig_stage<T>(m, f, s, l4, t4, n4, e_last, (s0 + dt * f3) * c.H, 3, c, U4, V4, W4)) {
                        ok = false;
                    } else {
                        const double dl4 = dt * U4 / metric_z0(q4), dd4 = dt * V4 / SLM, f4 = W4 / c.H;
                        const double dl = (dl1 + 2.0 * dl2 + 2.0 * dl3 + dl4) / 6.0;
                        const double dd = (dd1 + 2.0 * dd2 + 2.0 * dd3 + dd4) / 6.0;
                        a = wrap180(lon0 + dl);
                        b = clamp_lat(lat0 + dd);
                        s_new = s0 + dt * (f1 + 2.0 * f2 + 2.0 * f3 + f4) / 6.0;
                    }
                }
            }
        }
    }
    if (!ok) {
        status = OUTSIDE;
        fr = FR_INTERP;
    } else {
        const Site qn = make_site(a, b);
        const int nn_new = site_anchor(m, qn);
        const int ein = end_elem<WALK>(m, a, b, e_last, nn_new);
        if (ein < 0) {
            status = OUTSIDE;
            fr = FR_OOB;
        } else {
            SigSite ce;
            sigma_site<T>(m, f, s, 4, a, b, nn_new, ce);
            lon_new = a;
            lat_new = b;
            nn_out = nn_new;
            e_out = ein;
            status = ALIVE;
            z_new = clamp_sig(s_new * ce.H, ce.H, s);
            if (s.kick) {
                const long long pid = st.pid ? st.pid[i] : i;
                int kel, kwel;
                apply_kick<true>(m, s, pid, realization_of(st, s, i), qn, lon0, lat0, z0p, pre_nn, false, lon_new, lat_new,
                           z_new, status, nn_out, fr, false, kel, kwel);
                if (status == ALIVE) {
                    const double H_post = ce.H;
                    sigma_site<T>(m, f, s, 4, lon_new, lat_new, nn_out, ce);
                    z_new = clamp_sig(z_new / H_post * ce.H, ce.H, s);
                }
            }
            if (s.az_on && status == ALIVE) {
                // integrators.py:917-930, diffusion.py:458-482 _loop_az_kick_sigma:
                // the constant Az (no drift), folded into [0, max(H, Dmin) -
                // z0b_min] of the end-of-step column at the particle
                double H = ce.H;
                if (H < s.Dmin) H = s.Dmin;
                double bot = H - s.z0b_min;
                if (bot < 0.0) bot = 0.0;
                double xi, unused;
                normal_pair<true>(m.rx, s.seed, realization_of(st, s, i),
                                  (unsigned long long)(st.pid ? st.pid[i] : i) + s.pid_offset, s.step_i, 1ull, xi,
                                  unused);
                const double sdt = s.time_dir * s.dt;
                const double abs_dt = sdt >= 0.0 ? sdt : -sdt;
                const double dz = 0.0 * abs_dt + sqrt(2.0 * s.az_const * abs_dt) * xi;
                z_new = reflect_depth(z_new + dz, 0.0, bot);
            }
        }
    }
    st.lon[i] = lon_new;
    st.lat[i] = lat_new;
    st.z[i] = z_new;
    st.status[i] = status;
    st.nn[i] = nn_out;
    st.fr[i] = fr;
    if constexpr (WALK) st.elem[i] = e_out;
    mark_anchor(st, i, status, nn_out, node_i);
}

}  // namespace kc
