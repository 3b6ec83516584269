// Device-side interpolation, time blending, vertical helpers, the counter RNG
// and the great-circle diffusion kick of the KELP time-stepping path.  Same
// floating-point operation order as the cited Numba functions (see the note
// at the top of kc_geom.cuh on -fmad=false and the trigonometric tables).
#pragma once
#include "kc_geom.cuh"
#include "kc_crmath.cuh"

namespace kc {

// Snapshot views: u/v rows are (L, N) row-major, w rows (K, N).  Half
// precision storage carries one power-of-two scale per row (value =
// stored * scale); the scale pointers are null for float and double.
template <typename T>
struct DField {
    const T* u;
    const T* v;
    const T* w;
    const float* su;
    const float* sv;
    const float* sw;
    const T* az;     // vertical diffusivity (K, N) on the interfaces, or null
    const double* eta;   // free surface (N) (sigma meshes), or null
};

template <typename T>
struct DBlend {
    DField<T> a, b, t;   // bracket pair and stage target
    double alpha0;       // bracket fraction of the step's start time
    long long n;         // row stride (nodes)
    // PCHIP reconstruction (pchip = 1): a, b, t, d are the four-record
    // stencil at times pt, and every stage "alpha" is the stage's time
    DField<T> d;
    double pt[4];
    int pchip;
};

// temporal_reconstruct.py:167-180 _fc_slope_scalar: Fritsch-Carlson interior
// slope, the weighted harmonic mean of the secants, 0 where they change sign
__device__ __forceinline__ double fc_slope(double dp, double dn, double hp, double hn) {
    if (dp * dn > 0.0) {
        const double w1 = 2.0 * hn + hp, w2 = hn + 2.0 * hp;
        return (w1 + w2) / (w1 / dp + w2 / dn);
    }
    return 0.0;
}

// temporal_reconstruct.py:183-215 _pchip_value_scalar: the monotone cubic
// Hermite value at tq in the central interval [pt1, pt2]
__device__ __forceinline__ double pchip4(double f0, double f1, double f2, double f3, const double* t, double tq) {
    const double h0 = t[1] - t[0], h1 = t[2] - t[1], h2 = t[3] - t[2];
    const double d0 = (f1 - f0) / h0, d1 = (f2 - f1) / h1, d2 = (f3 - f2) / h2;
    const double m1 = fc_slope(d0, d1, h0, h1), m2 = fc_slope(d1, d2, h1, h2);
    const double s = (tq - t[1]) / h1, s2 = s * s, s3 = s2 * s;
    const double h00 = 2.0 * s3 - 3.0 * s2 + 1.0, h10 = s3 - 2.0 * s2 + s;
    const double h01 = -2.0 * s3 + 3.0 * s2, h11 = s3 - s2;
    return h00 * f1 + h10 * h1 * m1 + h01 * f2 + h11 * h1 * m2;
}

// The PCHIP stage value of entry idx of one field (pointers of the stencil)
template <typename T>
__device__ __forceinline__ double pchip_at(const T* p0, const T* p1, const T* p2, const T* p3, long long idx,
                                          const double* t, double tq) {
    return pchip4((double)__ldg(&p0[idx]), (double)__ldg(&p1[idx]), (double)__ldg(&p2[idx]), (double)__ldg(&p3[idx]),
                  t, tq);
}

// Nested two-level time blend with the reference's endpoint shortcuts
// (interpolate.py:1404-1436, vertical.py:1042-1061 _tblend_scalar).
__device__ __forceinline__ double tblend(double a, double b, double t, double alpha0, double alpha) {
    if (alpha < 1e-12) {
        if (alpha0 == 0.0) return a;
        return (1.0 - alpha0) * a + alpha0 * b;
    }
    if (alpha > 1.0 - 1e-12) return t;
    if (alpha0 == 0.0) return (1.0 - alpha) * a + alpha * t;
    double a0 = (1.0 - alpha0) * a + alpha0 * b;
    return (1.0 - alpha) * a0 + alpha * t;
}

// The compacted vertex ring of interpolate.py:1368-1377 (skip -1 slots and a
// repeat of vertex 0), with coordinates.
struct Ring {
    int v[4];
    double ln[4], la[4];
    int n;
};

__device__ __forceinline__ void put_ring(Ring& r, int n, int nd, double2 a) {
    if (n == 0) { r.v[0] = nd; r.ln[0] = a.x; r.la[0] = a.y; }
    else if (n == 1) { r.v[1] = nd; r.ln[1] = a.x; r.la[1] = a.y; }
    else if (n == 2) { r.v[2] = nd; r.ln[2] = a.x; r.la[2] = a.y; }
    else { r.v[3] = nd; r.ln[3] = a.x; r.la[3] = a.y; }
}

__device__ __forceinline__ void load_ring(const DMesh& m, int4 e, Ring& r) {
    int n = 0;
    int first = -1;
    if (e.x >= 0) { put_ring(r, n++, e.x, __ldg(&m.ll[e.x])); first = e.x; }
    if (e.y >= 0 && !(n > 0 && e.y == first)) { put_ring(r, n++, e.y, __ldg(&m.ll[e.y])); if (first < 0) first = e.y; }
    if (e.z >= 0 && !(n > 0 && e.z == first)) { put_ring(r, n++, e.z, __ldg(&m.ll[e.z])); if (first < 0) first = e.z; }
    if (e.w >= 0 && !(n > 0 && e.w == first)) put_ring(r, n++, e.w, __ldg(&m.ll[e.w]));
    if (n == 3) { r.v[3] = r.v[0]; r.ln[3] = r.ln[0]; r.la[3] = r.la[0]; }   // defined, never weighted
    r.n = n;
}

// The compacted ring as vertex ids only (load_ring's order and dedupe; slot
// 3 repeats slot 0 for a triangle): the coordinates are read where they are
// used, so no double-precision vertex array stays live across the loops.
struct RingId {
    int v[4];
    int n;
};

__device__ __forceinline__ void ring_ids(int4 e, RingId& r) {
    int n = 0, first = -1;
    r.v[0] = r.v[1] = r.v[2] = r.v[3] = -1;
    auto push = [&](int id) {
        if (n == 0) r.v[0] = id;
        else if (n == 1) r.v[1] = id;
        else if (n == 2) r.v[2] = id;
        else r.v[3] = id;
        ++n;
    };
    if (e.x >= 0) { push(e.x); first = e.x; }
    if (e.y >= 0 && !(n > 0 && e.y == first)) { push(e.y); if (first < 0) first = e.y; }
    if (e.z >= 0 && !(n > 0 && e.z == first)) { push(e.z); if (first < 0) first = e.z; }
    if (e.w >= 0 && !(n > 0 && e.w == first)) push(e.w);
    if (n == 3) r.v[3] = r.v[0];
    r.n = n;
}

// Vertex weights of the point in the containing element, projected around the
// wrapped-delta centroid (interpolate.py:1376-1402) with radius R; false for
// the degenerate-triangle sentinel or an element with fewer than 3 vertices.
// Two passes over the vertices (sums, then the projection), each operation
// in the reference's order.
__device__ __forceinline__ bool bary_weights_core(const DMesh& m, int elem, double xp, double yp, double R,
                                                  RingId& r, double* w) {
    ring_ids(__ldg(&m.en[elem]), r);
    const int nv = r.n;
    if (nv < 3) return false;
    const double2 a0 = __ldg(&m.ll[r.v[0]]);
    const double lon_ref = a0.x;
    double dsum = 0.0 + wrap180(a0.x - lon_ref), lat0 = 0.0 + a0.y;
#pragma unroll
    for (int k = 1; k < 4; ++k) {
        if (k < nv) {
            const double2 a = __ldg(&m.ll[r.v[k]]);
            dsum += wrap180(a.x - lon_ref);
            lat0 += a.y;
        }
    }
    const double lon0 = lon_ref + dsum / (double)nv;
    lat0 /= (double)nv;
    const double cosl = __ldg(&m.ecos[elem]).y;
    double vx[4], vy[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const double2 a = __ldg(&m.ll[r.v[k]]);
        vx[k] = wrap180(a.x - lon0) * DEG2RAD * R * cosl;
        vy[k] = (a.y - lat0) * DEG2RAD * R;
    }
    const double px = wrap180(xp - lon0) * DEG2RAD * R * cosl;
    const double py = (yp - lat0) * DEG2RAD * R;
    if (nv == 3) {
        bary_tri(px, py, vx[0], vy[0], vx[1], vy[1], vx[2], vy[2], w[0], w[1], w[2]);
        w[3] = 0.0;
        return !(w[0] == -1.0);
    }
    wachspress_quad(px, py, vx, vy, w);
    return !(w[0] == -1.0);
}

// interpolate.py:1340-1440 _interp_barycentric_core_tinterp (row = 0) and
// interpolate.py:1443-1529 its 3-D twin (row = the particle's layer).
// The core given its containing element `elem` (>= 0).
template <typename T>
__device__ KC_INL_STAGE bool interp_uv_at(const DMesh& m, const DBlend<T>& f, int elem, double xp, double yp,
                                          double time_dir, int row, double alpha, double& U, double& V) {
    U = 0.0;
    V = 0.0;
    RingId r;
    double w[4];
    if (!bary_weights_core(m, elem, xp, yp, m.r_earth, r, w)) return false;
    const long long base = (long long)row * f.n;
    const double alpha0 = f.alpha0;
    const double beta0 = 1.0 - alpha0;
    const double beta = 1.0 - alpha;
    double Us = 0.0, Vs = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (k >= r.n) break;
        long long idx = base + r.v[k];
        double un, vn;
        if (f.pchip) {
            un = pchip_at(f.a.u, f.b.u, f.t.u, f.d.u, idx, f.pt, alpha);
            vn = pchip_at(f.a.v, f.b.v, f.t.v, f.d.v, idx, f.pt, alpha);
        } else if (alpha < 1e-12) {
            if (alpha0 == 0.0) {
                un = (double)__ldg(&f.a.u[idx]);
                vn = (double)__ldg(&f.a.v[idx]);
            } else {
                un = beta0 * (double)__ldg(&f.a.u[idx]) + alpha0 * (double)__ldg(&f.b.u[idx]);
                vn = beta0 * (double)__ldg(&f.a.v[idx]) + alpha0 * (double)__ldg(&f.b.v[idx]);
            }
        } else if (alpha > 1.0 - 1e-12) {
            un = (double)__ldg(&f.t.u[idx]);
            vn = (double)__ldg(&f.t.v[idx]);
        } else if (alpha0 == 0.0) {
            un = beta * (double)__ldg(&f.a.u[idx]) + alpha * (double)__ldg(&f.t.u[idx]);
            vn = beta * (double)__ldg(&f.a.v[idx]) + alpha * (double)__ldg(&f.t.v[idx]);
        } else {
            double ua0 = beta0 * (double)__ldg(&f.a.u[idx]) + alpha0 * (double)__ldg(&f.b.u[idx]);
            double va0 = beta0 * (double)__ldg(&f.a.v[idx]) + alpha0 * (double)__ldg(&f.b.v[idx]);
            un = beta * ua0 + alpha * (double)__ldg(&f.t.u[idx]);
            vn = beta * va0 + alpha * (double)__ldg(&f.t.v[idx]);
        }
        Us += w[k] * un;
        Vs += w[k] * vn;
    }
    U = time_dir * Us;
    V = time_dir * Vs;
    return true;
}

template <typename T>
__device__ __forceinline__ bool interp_uv_bary(const DMesh& m, const DBlend<T>& f, double xp, double yp, int nn,
                                               int hint, double time_dir, int row, double alpha, double& U,
                                               double& V) {
    const int elem = hint >= 0 ? hint : contain_local(m, xp, yp, nn);
    if (elem < 0) {
        U = 0.0;
        V = 0.0;
        return false;
    }
    return interp_uv_at<T>(m, f, elem, xp, yp, time_dir, row, alpha, U, V);
}

// vertical_uv.py:457-523 uv_bracket: (k, alpha) of depth z among the data
// points p[0..last_i]; alpha < 0 reads point k alone.
__device__ __forceinline__ void uv_bracket(const double* __restrict__ p, int li, double z, int& k, double& alpha) {
    if (li <= 0) { k = 0; alpha = -1.0; return; }
    double zc = z;
    const double p0 = __ldg(&p[0]), pl = __ldg(&p[li]);
    if (zc > pl) zc = pl;
    if (zc < p0) zc = p0;
    if (zc <= p0) { k = 0; alpha = -1.0; return; }
    if (zc >= pl) { k = li; alpha = -1.0; return; }
    // first j in [0, li-1] with zc < p[j+1] (exists: zc < p[li])
    int lo = 0, hi = li - 1;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (zc < __ldg(&p[mid + 1])) hi = mid;
        else lo = mid + 1;
    }
    k = lo;
    const double pk = __ldg(&p[k]);
    const double dz = __ldg(&p[k + 1]) - pk;
    if (dz < 1e-12) { alpha = -1.0; return; }
    const double a = (zc - pk) / dz;
    if (a <= 0.0) { alpha = -1.0; return; }
    if (a >= 1.0) { k = k + 1; alpha = -1.0; return; }
    alpha = a;
}

// The time blend of one stored (point, node) value (interpolate.py:1847-1876
// _tinterp_point_uv).
template <typename T>
__device__ __forceinline__ void tinterp_point_uv(const DBlend<T>& f, int k, int nd, double alpha, double& u,
                                                 double& v) {
    const long long idx = (long long)k * f.n + nd;
    const double alpha0 = f.alpha0;
    if (f.pchip) {
        u = pchip_at(f.a.u, f.b.u, f.t.u, f.d.u, idx, f.pt, alpha);
        v = pchip_at(f.a.v, f.b.v, f.t.v, f.d.v, idx, f.pt, alpha);
        return;
    }
    if (alpha < 1e-12) {
        if (alpha0 == 0.0) {
            u = (double)__ldg(&f.a.u[idx]);
            v = (double)__ldg(&f.a.v[idx]);
            return;
        }
        const double beta0 = 1.0 - alpha0;
        u = beta0 * (double)__ldg(&f.a.u[idx]) + alpha0 * (double)__ldg(&f.b.u[idx]);
        v = beta0 * (double)__ldg(&f.a.v[idx]) + alpha0 * (double)__ldg(&f.b.v[idx]);
        return;
    }
    if (alpha > 1.0 - 1e-12) {
        u = (double)__ldg(&f.t.u[idx]);
        v = (double)__ldg(&f.t.v[idx]);
        return;
    }
    const double beta = 1.0 - alpha;
    if (alpha0 == 0.0) {
        u = beta * (double)__ldg(&f.a.u[idx]) + alpha * (double)__ldg(&f.t.u[idx]);
        v = beta * (double)__ldg(&f.a.v[idx]) + alpha * (double)__ldg(&f.t.v[idx]);
        return;
    }
    const double beta0 = 1.0 - alpha0;
    const double ua0 = beta0 * (double)__ldg(&f.a.u[idx]) + alpha0 * (double)__ldg(&f.b.u[idx]);
    const double va0 = beta0 * (double)__ldg(&f.a.v[idx]) + alpha0 * (double)__ldg(&f.b.v[idx]);
    u = beta * ua0 + alpha * (double)__ldg(&f.t.u[idx]);
    v = beta * va0 + alpha * (double)__ldg(&f.t.v[idx]);
}

// interpolate.py:1879-1971 _interp_barycentric_core_tinterp_dl with the wall
// rule of :1664-1711 _dl_node_wall: the layer twin's geometry, each vertex
// read linearly in depth between its bracketing data points (time first),
// vertices dry at the depth left out.
template <typename T>
__device__ __noinline__ bool interp_uv_dl_at(const DMesh& m, const DBlend<T>& f, int elem, double xp, double yp,
                                             double z, double time_dir, double alpha, double& U, double& V) {
    U = 0.0;
    V = 0.0;
    RingId r;
    double w[4];
    if (!bary_weights_core(m, elem, xp, yp, m.r_earth, r, w)) return false;
    const int nv = r.n;
    double zq = z;
    if (isnan(zq)) zq = INFINITY;   // dry wherever the bed is finite
    bool wet[4];
    int n_wet = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        wet[k] = k < nv && zq <= __ldg(&m.dl_bed[r.v[k]]);
        n_wet += wet[k] ? 1 : 0;
    }
    if (n_wet == 0) {
        int kd = 0;
        for (int k = 1; k < nv; ++k)
            if (__ldg(&m.dl_bed[r.v[k]]) > __ldg(&m.dl_bed[r.v[kd]])) kd = k;
        const int nd = r.v[kd];
        double un, vn;
        tinterp_point_uv<T>(f, __ldg(&m.dl_last[nd]), nd, alpha, un, vn);
        U = time_dir * un;
        V = time_dir * vn;
        return true;
    }
    double den = 1.0;
    if (n_wet < nv) {
        double wsum = 0.0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (wet[k]) {
                if (w[k] < 0.0) w[k] = 0.0;
                wsum += w[k];
            }
        }
        if (wsum < 1e-12) {
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (wet[k]) w[k] = 1.0;
            den = (double)n_wet;
        } else {
            den = wsum;
        }
    }
    double Us = 0.0, Vs = 0.0;
    for (int k = 0; k < nv; ++k) {
        const int nd = r.v[k];
        if (n_wet < nv && !wet[k]) continue;
        int kb;
        double ab;
        uv_bracket(m.dl_p, __ldg(&m.dl_last[nd]), zq, kb, ab);
        double un, vn;
        tinterp_point_uv<T>(f, kb, nd, alpha, un, vn);
        if (!(ab < 0.0)) {
            double un1, vn1;
            tinterp_point_uv<T>(f, kb + 1, nd, alpha, un1, vn1);
            un = (1.0 - ab) * un + ab * un1;
            vn = (1.0 - ab) * vn + ab * vn1;
        }
        Us += w[k] * un;
        Vs += w[k] * vn;
    }
    if (n_wet < nv) {
        Us = Us / den;
        Vs = Vs / den;
    }
    U = time_dir * Us;
    V = time_dir * Vs;
    return true;
}

template <typename T>
__device__ __forceinline__ bool interp_uv_bary_dl(const DMesh& m, const DBlend<T>& f, double xp, double yp, int nn,
                                                  int hint, double z, double time_dir, double alpha, double& U,
                                                  double& V) {
    const int elem = hint >= 0 ? hint : contain_local(m, xp, yp, nn);
    if (elem < 0) {
        U = 0.0;
        V = 0.0;
        return false;
    }
    return interp_uv_dl_at<T>(m, f, elem, xp, yp, z, time_dir, alpha, U, V);
}

// First k in [lo, hi] with z < zl[k + 1] (the caller guarantees one exists):
// the linear scans of the reference as a binary search over the monotone
// interface table (same index).
__device__ __forceinline__ int first_above(const double* __restrict__ zl, int lo, int hi, double z) {
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (z < __ldg(&zl[mid + 1])) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

// vertical.py:39-91 find_layer; the deepest valid layer of the node (the
// reference's first scan) comes from a host table.
__device__ __forceinline__ int find_layer(const DMesh& m, double z, int node) {
    const int K = m.K;
    if (K < 2) return 0;
    if (z <= __ldg(&m.zlev[0])) return 0;
    const int max_layer = __ldg(&m.max_layer[node]);
    const double bottom = __ldg(&m.depth[node]);
    if (z >= bottom || z >= __ldg(&m.zlev[max_layer + 1])) return max_layer;
    return first_above(m.zlev, 0, max_layer, z);
}

// Where depth z falls among the interfaces, as vertical.py:1064-1098
// _interp_w_linear_single_tinterp decides it: one level read (k, a < 0) or
// the linear blend of levels k and k + 1 with fraction a.  It depends on z
// alone, so the vertices of one element share it unless their own depth
// clamps z.
struct WLoc {
    int k;
    double a;
};

__device__ __forceinline__ WLoc w_locate(const DMesh& m, double z) {
    const int K = m.K;
    const double* zl = m.zlev;
    if (K < 2 || z <= __ldg(&zl[0])) return {0, -1.0};
    if (z >= __ldg(&zl[K - 1])) return {K - 1, -1.0};
    const int k = first_above(zl, 0, K - 2, z);
    const double zk = __ldg(&zl[k]), zk1 = __ldg(&zl[k + 1]);
    const double dz = zk1 - zk;
    if (dz < 1e-12) return {k, -1.0};
    return {k, (z - zk) / dz};
}

constexpr int kRingMax = 64;   // vertical.py:443 _MAX_NEIGHBOURS

__device__ __forceinline__ int slot_of(const int4& e, int v) {
    return v == 0 ? e.x : (v == 1 ? e.y : (v == 2 ? e.z : e.w));
}

// vertical.py:447-485 _collect_neighbour_nodes, visited in place: the
// centre, then every vertex slot of the centre's elements in node->element
// order, each node at its first occurrence only, at most kRingMax nodes.
// f(node) returns false to stop; the return value counts the nodes visited.
template <class F>
__device__ __forceinline__ int for_ring(const DMesh& m, int nn, F&& f) {
    if (!f(nn)) return 1;
    int count = 1;
    const int s = m.n2e_off[nn], e = m.n2e_off[nn + 1];
    for (int k = s; k < e && count < kRingMax; ++k) {
        const int4 ek = m.en[m.n2e[k]];
        for (int v = 0; v < 4 && count < kRingMax; ++v) {
            const int nd = slot_of(ek, v);
            if (nd < 0 || nd == nn) continue;
            bool dup = false;
            for (int u = 0; u < v && !dup; ++u) dup = slot_of(ek, u) == nd;
            for (int kk = s; kk < k && !dup; ++kk) {
                const int4 ej = m.en[m.n2e[kk]];
                dup = ej.x == nd || ej.y == nd || ej.z == nd || ej.w == nd;
            }
            if (dup) continue;
            ++count;
            if (!f(nd)) return count;
        }
    }
    return count;
}

// The time-blended W of one node at a located depth (the value part of
// vertical.py:1064-1098; tblend per level, :1042-1061).
template <typename T>
__device__ __forceinline__ double w_at(const DBlend<T>& f, double alpha, const WLoc& L, int node, double time_dir) {
    const long long n = f.n;
    auto at = [&](int k) {
        const long long idx = (long long)k * n + node;
        if (f.pchip) return pchip_at(f.a.w, f.b.w, f.t.w, f.d.w, idx, f.pt, alpha);
        if (alpha < 1e-12) {
            const double a = (double)__ldg(&f.a.w[idx]);
            if (f.alpha0 == 0.0) return a;
            return (1.0 - f.alpha0) * a + f.alpha0 * (double)__ldg(&f.b.w[idx]);
        }
        if (alpha > 1.0 - 1e-12) return (double)__ldg(&f.t.w[idx]);
        return tblend((double)__ldg(&f.a.w[idx]), (double)__ldg(&f.b.w[idx]), (double)__ldg(&f.t.w[idx]),
                      f.alpha0, alpha);
    };
    if (L.a < 0.0) return time_dir * at(L.k);
    const double w_lo = at(L.k);
    const double w_hi = at(L.k + 1);
    return time_dir * ((1.0 - L.a) * w_lo + L.a * w_hi);
}

// vertical.py:1064-1098 _interp_w_linear_single_tinterp
template <typename T>
__device__ __forceinline__ double w_linear(const DMesh& m, const DBlend<T>& f, double alpha, double z, int node,
                                           double time_dir) {
    return w_at(f, alpha, w_locate(m, z), node, time_dir);
}

// Python's min(a, b): the first argument unless the second is smaller.
__device__ __forceinline__ double pymin(double a, double b) { return b < a ? b : a; }

// W of a vertex at min(z, its depth), reusing the location of z when the
// vertex's depth does not clamp it.
template <typename T>
__device__ __forceinline__ double w_vertex(const DMesh& m, const DBlend<T>& f, double alpha, double z,
                                           const WLoc& Lz, int nd, double time_dir) {
    const double zc = pymin(z, __ldg(&m.depth[nd]));
    return w_at(f, alpha, zc == z ? Lz : w_locate(m, zc), nd, time_dir);
}

// W from the anchor's 1-ring of nodes (vertical.py:447-485 order), each
// node's W at the particle's depth, or at its own bottom where the particle
// is deeper (w_vertex): the least-squares plane through them evaluated at
// the particle (vertical.py:493-601 _interp_w_leastsq_single; fewer than
// three nodes or a singular system: the anchor's own W), or their
// inverse-square-distance mean (:1148-1229 _interp_w_idw_single; a node
// within 1 m is taken as is, no weight: the anchor's own W).  The cos of
// the latitude is the correctly rounded one, the C library's value but
// where the library misrounds.
template <typename T>
static __device__ __noinline__ double w_ring(const DMesh& m, const DBlend<T>& f, int w_code, double alpha,
                                             double xp, double yp, double z, int node, double td) {
    const WLoc Lz = w_locate(m, z);
    double z0 = cr::cos_cr(yp * DEG2RAD) * SLM;
    if (z0 < 1.0) z0 = 1.0;
    if (w_code == 3) {
        double sw = 0.0, swv = 0.0, hit_val = 0.0;
        bool hit = false;
        for_ring(m, node, [&](int nd) {
            const double wv = w_vertex<T>(m, f, alpha, z, Lz, nd, td);
            const double2 p = __ldg(&m.ll[nd]);
            const double dx = wrap180(p.x - xp) * z0;
            const double dy = (p.y - yp) * SLM;
            const double d2 = dx * dx + dy * dy;
            if (d2 < 1.0) {
                hit = true;
                hit_val = wv;
                return false;
            }
            const double wt = 1.0 / d2;
            sw += wt;
            swv += wt * wv;
            return true;
        });
        if (hit) return hit_val;
        if (!(sw < 1e-30)) return swv / sw;
        return w_vertex<T>(m, f, alpha, z, Lz, node, td);
    }
    double a11 = 0.0, a12 = 0.0, a13 = 0.0, a22 = 0.0, a23 = 0.0, a33 = 0.0, fw = 0.0, f1w = 0.0, f2w = 0.0;
    const int cnt = for_ring(m, node, [&](int nd) {
        const double wv = w_vertex<T>(m, f, alpha, z, Lz, nd, td);
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
    if (cnt >= 3) {
        const double a21 = a12, a31 = a13, a32 = a23;
        const double det = a11 * a22 * a33 + a12 * a23 * a31 + a13 * a21 * a32 - a13 * a22 * a31 - a12 * a21 * a33 -
                           a11 * a23 * a32;
        if (!(fabs(det) < 1e-30 || fabs(det) < 1e-12 * fabs(a11 * a22 * a33))) {
            const double inv = 1.0 / fabs(det);
            const double b11 = a22 * a33 - a23 * a32;
            const double b12 = a13 * a32 - a12 * a33;
            const double b13 = a12 * a23 - a13 * a22;
            return (b11 * fw + b12 * f1w + b13 * f2w) * inv;
        }
    }
    return w_vertex<T>(m, f, alpha, z, Lz, node, td);
}

// True when no fan triangle of the ring can give the point three weights
// >= -1e-6 in the projected test below, decided from longitude offsets
// (wrapped around vertex 0) and latitudes alone.  In exact arithmetic a point
// whose barycentric weights are all >= -eps lies within 2 eps times the
// element's extent of its bounding box along each projected axis; the
// projection scales each axis by a positive factor, so the test holds in
// degrees.  The margin is 1e-5 of the extent (five times the bound) plus
// 1e-9 degrees for rounding, and elements spanning 90 degrees or more of
// longitude (pole cells) are never skipped.
__device__ __forceinline__ bool w_ring_rejects(const Ring& r, int nvv, double xp, double yp) {
    double dmin = 0.0, dmax = 0.0, lmin = r.la[0], lmax = r.la[0];
#pragma unroll
    for (int v = 1; v < 4; ++v) {
        if (v < nvv) {
            const double d = wrap180(r.ln[v] - r.ln[0]);
            dmin = fmin(dmin, d);
            dmax = fmax(dmax, d);
            lmin = fmin(lmin, r.la[v]);
            lmax = fmax(lmax, r.la[v]);
        }
    }
    if (!(dmax - dmin < 90.0)) return false;
    const double my = 1e-5 * (lmax - lmin) + 1e-9;
    if (yp < lmin - my || yp > lmax + my) return true;
    const double mx = 1e-5 * (dmax - dmin) + 1e-9;
    const double dp = wrap180(xp - r.ln[0]);
    return dp < dmin - mx || dp > dmax + mx;
}

// vertical.py:744-881 _interp_w_bary_single_tinterp: the anchor's own fan
// search (denominator tolerance 1e-14, R = 6371000, origin by
// mesh.py:1973-2003 _seam_safe_lon0), triangles blended inline, quads through
// Wachspress, nearest-node fallback.  Elements the point provably lies
// outside of (w_ring_rejects) skip the projected test, whose verdict for them
// is "outside" anyway.
template <typename T>
__device__ __noinline__ double w_bary(const DMesh& m, const DBlend<T>& f, double alpha, double xp, double yp,
                                      double z, int node, double time_dir) {
    const WLoc Lz = w_locate(m, z);
    int s = __ldg(&m.n2e_off[node]), e = __ldg(&m.n2e_off[node + 1]);
    for (int kk = s; kk < e; ++kk) {
        const int el = __ldg(&m.n2e[kk]);
        Ring r;
        load_ring(m, __ldg(&m.en[el]), r);
        const int nvv = r.n;
        if (nvv < 3) continue;
        if (w_ring_rejects(r, nvv, xp, yp)) continue;
        double lmin = fmin(fmin(r.ln[0], r.ln[1]), r.ln[2]), lmax = fmax(fmax(r.ln[0], r.ln[1]), r.ln[2]);
        if (nvv == 4) { lmin = fmin(lmin, r.ln[3]); lmax = fmax(lmax, r.ln[3]); }
        double lon0;
        if (lmax - lmin > 180.0) {
            double d = 0.0;
#pragma unroll
            for (int v = 0; v < 4; ++v)
                if (v < nvv) d += wrap180(r.ln[v] - r.ln[0]);
            lon0 = r.ln[0] + d / (double)nvv;
        } else {
            double sm = 0.0;
#pragma unroll
            for (int v = 0; v < 4; ++v)
                if (v < nvv) sm += r.ln[v];
            lon0 = sm / (double)nvv;
        }
        double lat0 = 0.0;
#pragma unroll
        for (int v = 0; v < 4; ++v)
            if (v < nvv) lat0 += r.la[v];
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
#pragma unroll
        for (int t = 0; t < 2; ++t) {
            if (t >= nvv - 2) break;
            const int i1 = t + 1, i2 = t + 2;
            const double ax = vx[0], ay = vy[0];
            const double bx = t == 0 ? vx[1] : vx[2], by = t == 0 ? vy[1] : vy[2];
            const double cx = t == 0 ? vx[2] : vx[3], cy = t == 0 ? vy[2] : vy[3];
            const double denom = (by - cy) * (ax - cx) + (cx - bx) * (ay - cy);
            if (fabs(denom) < 1e-14) continue;
            const double w1 = ((by - cy) * (px - cx) + (cx - bx) * (py - cy)) / denom;
            const double w2 = ((cy - ay) * (px - cx) + (ax - cx) * (py - cy)) / denom;
            const double w3 = 1.0 - w1 - w2;
            const double eps = -1e-6;
            if (w1 >= eps && w2 >= eps && w3 >= eps) {
                if (nvv == 4) {
                    double wts[4];
                    wachspress_quad(px, py, vx, vy, wts);
                    double acc = 0.0;
#pragma unroll
                    for (int vi = 0; vi < 4; ++vi)
                        acc += wts[vi] * w_vertex(m, f, alpha, z, Lz, r.v[vi], time_dir);
                    return acc;
                }
                const int n0 = r.v[0];
                const int n1 = i1 == 1 ? r.v[1] : r.v[2];
                const int n2 = i2 == 2 ? r.v[2] : r.v[3];
                const double w_v0 = w_vertex(m, f, alpha, z, Lz, n0, time_dir);
                const double w_v1 = w_vertex(m, f, alpha, z, Lz, n1, time_dir);
                const double w_v2 = w_vertex(m, f, alpha, z, Lz, n2, time_dir);
                return w1 * w_v0 + w2 * w_v1 + w3 * w_v2;
            }
        }
    }
    return w_vertex(m, f, alpha, z, Lz, node, time_dir);
}

// The barycentric W of vertical.py:744-881 when its search is known to stop
// at element `el` (contain_local_w): that element's own frame and weights,
// the first fan triangle for a triangle, Wachspress for a quad.
template <typename T>
__device__ KC_INL_STAGE double w_bary_at(const DMesh& m, const DBlend<T>& f, double alpha, double xp, double yp,
                                         double z, int el, double time_dir) {
    const WLoc Lz = w_locate(m, z);
    RingId r;
    ring_ids(__ldg(&m.en[el]), r);
    const int nvv = r.n;
    // pass 1: the running extent and sums in the reference's order
    const double2 a0 = __ldg(&m.ll[r.v[0]]);
    double lmin = a0.x, lmax = a0.x, d = 0.0 + wrap180(a0.x - a0.x), sm = 0.0 + a0.x, lat0 = 0.0 + a0.y;
#pragma unroll
    for (int v = 1; v < 4; ++v) {
        if (v < nvv) {
            const double2 a = __ldg(&m.ll[r.v[v]]);
            if (v < 3 || nvv == 4) { lmin = fmin(lmin, a.x); lmax = fmax(lmax, a.x); }
            d += wrap180(a.x - a0.x);
            sm += a.x;
            lat0 += a.y;
        }
    }
    const double lon0 = lmax - lmin > 180.0 ? a0.x + d / (double)nvv : sm / (double)nvv;
    lat0 /= (double)nvv;
    const double cos_lat0 = __ldg(&m.ecos[el]).y;
    const double R = 6371000.0;
    double vx[4], vy[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        const double2 a = __ldg(&m.ll[r.v[v]]);
        vx[v] = wrap180(a.x - lon0) * DEG2RAD * R * cos_lat0;
        vy[v] = (a.y - lat0) * DEG2RAD * R;
    }
    const double px = wrap180(xp - lon0) * DEG2RAD * R * cos_lat0;
    const double py = (yp - lat0) * DEG2RAD * R;
    if (nvv == 4) {
        double wts[4];
        wachspress_quad(px, py, vx, vy, wts);
        double acc = 0.0;
#pragma unroll
        for (int vi = 0; vi < 4; ++vi) acc += wts[vi] * w_vertex(m, f, alpha, z, Lz, r.v[vi], time_dir);
        return acc;
    }
    const double ax = vx[0], ay = vy[0], bx = vx[1], by = vy[1], cx = vx[2], cy = vy[2];
    const double denom = (by - cy) * (ax - cx) + (cx - bx) * (ay - cy);
    const double w1 = ((by - cy) * (px - cx) + (cx - bx) * (py - cy)) / denom;
    const double w2 = ((cy - ay) * (px - cx) + (ax - cx) * (py - cy)) / denom;
    const double w3 = 1.0 - w1 - w2;
    const double w_v0 = w_vertex(m, f, alpha, z, Lz, r.v[0], time_dir);
    const double w_v1 = w_vertex(m, f, alpha, z, Lz, r.v[1], time_dir);
    const double w_v2 = w_vertex(m, f, alpha, z, Lz, r.v[2], time_dir);
    return w1 * w_v0 + w2 * w_v1 + w3 * w_v2;
}

// The element the barycentric W search of vertical.py:744-881 selects for
// the point (the first 1-ring element of the anchor with a fan triangle whose
// three weights are >= -1e-6), or -1 for its nodal fallback: w_bary's loop
// without the values.
static __device__ KC_INL_CONTAIN int w_search_elem(const DMesh& m, double xp, double yp, int node) {
    int s = __ldg(&m.n2e_off[node]), e = __ldg(&m.n2e_off[node + 1]);
    for (int kk = s; kk < e; ++kk) {
        const int el = __ldg(&m.n2e[kk]);
        Ring r;
        load_ring(m, __ldg(&m.en[el]), r);
        const int nvv = r.n;
        if (nvv < 3) continue;
        if (w_ring_rejects(r, nvv, xp, yp)) continue;
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
        for (int v = 0; v < 4; ++v) {
            vx[v] = wrap180(r.ln[v] - lon0) * DEG2RAD * R * cos_lat0;
            vy[v] = (r.la[v] - lat0) * DEG2RAD * R;
        }
        const double px = wrap180(xp - lon0) * DEG2RAD * R * cos_lat0;
        const double py = (yp - lat0) * DEG2RAD * R;
        for (int t = 0; t < nvv - 2; ++t) {
            const double ax = vx[0], ay = vy[0];
            const double bx = vx[t + 1], by = vy[t + 1], cx = vx[t + 2], cy = vy[t + 2];
            const double denom = (by - cy) * (ax - cx) + (cx - bx) * (ay - cy);
            if (fabs(denom) < 1e-14) continue;
            const double w1 = ((by - cy) * (px - cx) + (cx - bx) * (py - cy)) / denom;
            const double w2 = ((cy - ay) * (px - cx) + (ax - cx) * (py - cy)) / denom;
            const double w3 = 1.0 - w1 - w2;
            if (w1 >= -1e-6 && w2 >= -1e-6 && w3 >= -1e-6) return el;
        }
    }
    return -1;
}

// mesh.py:2488-2590 _walk_containing_element: from element e, cross the edge
// of the most negative normalized signed-area coordinate (projection of
// mesh.py:2006-2051 in the element's own frame) until every coordinate is
// >= -1e-6; an accept within the 1e-2 band is verified with the exact local
// predicate; at most 256 crossings; -1 for every non-contained outcome.
static __device__ __noinline__ int edge_walk(const DMesh& m, double lon_p, double lat_p, int e) {
    if (e < 0 || (long long)e >= m.E || !m.enb) return -1;
    int prev = -1;
    for (int it = 0; it < 256; ++it) {
        Ring r;
        load_ring(m, __ldg(&m.en[e]), r);
        const int nv = r.n;
        if (nv < 3) return -1;
        double lmin = r.ln[0], lmax = r.ln[0];
#pragma unroll
        for (int k = 1; k < 4; ++k)
            if (k < nv) { lmin = fmin(lmin, r.ln[k]); lmax = fmax(lmax, r.ln[k]); }
        double lon0;
        if (lmax - lmin > 180.0) {
            double ds = 0.0;
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (k < nv) ds += wrap180(r.ln[k] - r.ln[0]);
            lon0 = r.ln[0] + ds / (double)nv;
        } else {
            double sm = 0.0;
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (k < nv) sm += r.ln[k];
            lon0 = sm / (double)nv;
        }
        double sl = 0.0;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (k < nv) sl += r.la[k];
        const double lat0 = sl / (double)nv;
        const double cl = __ldg(&m.ecos[e]).y;   // cos(mean ring latitude), the host C library's
        double x[4], y[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            x[k] = wrap180(r.ln[k] - lon0) * DEG2RAD * R_STD * cl;
            y[k] = (r.la[k] - lat0) * DEG2RAD * R_STD;
        }
        const double px = wrap180(lon_p - lon0) * DEG2RAD * R_STD * cl;
        const double py = (lat_p - lat0) * DEG2RAD * R_STD;
        double S = 0.0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (k < nv) {
                const int j = k + 1 < nv ? k + 1 : 0;
                S += x[k] * y[j] - x[j] * y[k];
            }
        }
        const double absS = fabs(S);
        if (absS < AREA_TOL) return -1;
        const double sgn = S > 0.0 ? 1.0 : -1.0;
        double worst = 1.0e100;
        int worst_k = -1;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (k < nv) {
                const int j = k + 1 < nv ? k + 1 : 0;
                const double A = (x[j] - x[k]) * (py - y[k]) - (px - x[k]) * (y[j] - y[k]);
                const double w = A * sgn / absS;
                if (w < worst) { worst = w; worst_k = k; }
            }
        }
        if (worst >= -1e-6) {
            if (worst >= 1e-2) return e;
            return element_contains(m, e, lon_p, lat_p) ? e : -1;
        }
        const int4 nb4 = __ldg(&m.enb[e]);
        const int nb = worst_k == 0 ? nb4.x : (worst_k == 1 ? nb4.y : (worst_k == 2 ? nb4.z : nb4.w));
        if (nb < 0 || nb == prev) return -1;
        prev = e;
        e = nb;
    }
    return -1;
}

// mesh.py:2593-2712 find_containing_elements_walk for one point: the walk
// from the carried element, else the local scan around the widened anchor,
// else around the exact anchor nn (the exactness heal); -1 outside.
static __device__ __noinline__ int walk_locate(const DMesh& m, double lon_p, double lat_p, int start, int nn) {
    if (start >= 0) {
        const int e = edge_walk(m, lon_p, lat_p, start);
        if (e >= 0) return e;
    }
    const int nw = nearest_widened(m, make_site(lon_p, lat_p));
    const int e = nw >= 0 ? contain_local(m, lon_p, lat_p, nw) : -1;
    if (e >= 0) return e;
    return contain_local(m, lon_p, lat_p, nn);
}

// ---------------------------------------------------------------------------
// Element-centre least squares (uv_interp "leastsq", element-layout u/v)
// ---------------------------------------------------------------------------

// interpolate.py:207-354 _interp_leastsq_core_tinterp (the steady core,
// :52-205, is its alpha0 = alpha = 0 case): a plane through the time-blended
// element-centre velocities of the anchor's element ring, in metres centred
// on the particle, solved by Cramer's rule; its value at the particle.  The
// sums run in the ring's order; a centre more than 180 degrees of raw
// longitude away is moved by one turn.  false (and 0, 0) for an empty ring or
// a normal matrix the scale-relative guard calls singular.  PCHIP stencils
// take the four-record value per element (the _pchip4 twin, :355-474).
template <typename T>
__device__ __forceinline__ bool interp_uv_lsq(const DMesh& m, const DBlend<T>& f, double xp, double yp, int nn,
                                              double time_dir, double alpha, double& U, double& V, int row = 0) {
    U = 0.0;
    V = 0.0;
    const int s0 = __ldg(&m.n2e_off[nn]), s1 = __ldg(&m.n2e_off[nn + 1]);
    if (s1 <= s0) return false;
    const double z0 = cr::cos_cr(yp * DEG2RAD) * SLM;
    const double xp_m = xp * z0;
    const double yp_m = yp * SLM;
    double a11 = 0.0, a12 = 0.0, a13 = 0.0, a22 = 0.0, a23 = 0.0, a33 = 0.0;
    double fU = 0.0, f1U = 0.0, f2U = 0.0, fV = 0.0, f1V = 0.0, f2V = 0.0;
    for (int k = s0; k < s1; ++k) {
        const int e = __ldg(&m.n2e[k]);
        const double2 c = __ldg(&m.ec[e]);
        double ex = c.x * z0 - xp_m;
        const double dlon_raw = c.x - xp;
        if (dlon_raw > 180.0) ex -= 360.0 * z0;
        else if (dlon_raw < -180.0) ex += 360.0 * z0;
        const double ey = c.y * SLM - yp_m;
        const long long idx = (long long)row * f.n + e;   // row: the layer of a 3-D field
        double uv, vv;
        if (f.pchip) {
            uv = pchip_at(f.a.u, f.b.u, f.t.u, f.d.u, idx, f.pt, alpha);
            vv = pchip_at(f.a.v, f.b.v, f.t.v, f.d.v, idx, f.pt, alpha);
        } else {
            uv = tblend((double)__ldg(&f.a.u[idx]), (double)__ldg(&f.b.u[idx]), (double)__ldg(&f.t.u[idx]), f.alpha0,
                        alpha);
            vv = tblend((double)__ldg(&f.a.v[idx]), (double)__ldg(&f.b.v[idx]), (double)__ldg(&f.t.v[idx]), f.alpha0,
                        alpha);
        }
        const double uu = time_dir * uv, vw = time_dir * vv;
        a11 = a11 + 1.0;
        a12 = a12 + ex;
        a13 = a13 + ey;
        a22 = a22 + ex * ex;
        a23 = a23 + ex * ey;
        a33 = a33 + ey * ey;
        fU = fU + uu;
        f1U = f1U + uu * ex;
        f2U = f2U + uu * ey;
        fV = fV + vw;
        f1V = f1V + vw * ex;
        f2V = f2V + vw * ey;
    }
    const double a21 = a12, a31 = a13, a32 = a23;
    const double det = a11 * a22 * a33 + a12 * a23 * a31 + a13 * a21 * a32 - a13 * a22 * a31 - a12 * a21 * a33 -
                       a11 * a23 * a32;
    if (fabs(det) < 1e-30 || fabs(det) < 1e-12 * fabs(a11 * a22 * a33)) return false;
    const double inv = 1.0 / fabs(det);
    const double b11 = a22 * a33 - a23 * a32;
    const double b12 = a13 * a32 - a12 * a33;
    const double b13 = a12 * a23 - a13 * a22;
    U = (b11 * fU + b12 * f1U + b13 * f2U) * inv;
    V = (b11 * fV + b12 * f1V + b13 * f2V) * inv;
    return true;
}

// interpolate.py:2588-2747 _interp_edge_leastsq_core (row: the layer of a
// 3-D field): the containing element (the local search around the anchor,
// mesh.py:2392-2470), the plane through its centre velocity and its edge
// neighbours' (build_elem_neighbors order); a boundary edge contributes the
// centre mirrored across the edge with the mirrored velocity (bc 0,
// freeslip: tangential kept, normal reversed) or the reversed one (bc 1,
// noslip), a zero-length boundary edge nothing; particle-centred metric
// coordinates with wrapped longitudes, Cramer's rule and the scale-relative
// singular guard of the element-centre fit.
template <typename T>
static __device__ __noinline__ bool interp_uv_edge_lsq(const DMesh& m, const DBlend<T>& f, double xp, double yp,
                                                       int nn, int bc, double time_dir, double alpha, int row,
                                                       double& U, double& V) {
    U = 0.0;
    V = 0.0;
    const int el = contain_local(m, xp, yp, nn);
    if (el < 0) return false;
    Ring r;
    load_ring(m, __ldg(&m.en[el]), r);
    const int nv = r.n;
    if (nv < 3) return false;
    const double z0 = cr::cos_cr(yp * DEG2RAD) * SLM;
    auto val = [&](int e, double& uu, double& vv) {
        const long long idx = (long long)row * f.n + e;
        if (f.pchip) {
            uu = pchip_at(f.a.u, f.b.u, f.t.u, f.d.u, idx, f.pt, alpha);
            vv = pchip_at(f.a.v, f.b.v, f.t.v, f.d.v, idx, f.pt, alpha);
        } else {
            uu = tblend((double)__ldg(&f.a.u[idx]), (double)__ldg(&f.b.u[idx]), (double)__ldg(&f.t.u[idx]), f.alpha0,
                        alpha);
            vv = tblend((double)__ldg(&f.a.v[idx]), (double)__ldg(&f.b.v[idx]), (double)__ldg(&f.t.v[idx]), f.alpha0,
                        alpha);
        }
    };
    const double2 c = __ldg(&m.ec[el]);
    const double cx = wrap180(c.x - xp) * z0;
    const double cy = (c.y - yp) * SLM;
    double uo, vo;
    val(el, uo, vo);
    const double u_own = time_dir * uo, v_own = time_dir * vo;
    double a11 = 1.0, a12 = cx, a13 = cy, a22 = cx * cx, a23 = cx * cy, a33 = cy * cy;
    double fU = u_own, f1U = u_own * cx, f2U = u_own * cy, fV = v_own, f1V = v_own * cx, f2V = v_own * cy;
    const int4 nb4 = __ldg(&m.enb[el]);
    for (int k = 0; k < nv; ++k) {
        const int nb = slot_of(nb4, k);
        double ex, ey, uu, vv;
        if (nb >= 0) {
            const double2 cn = __ldg(&m.ec[nb]);
            ex = wrap180(cn.x - xp) * z0;
            ey = (cn.y - yp) * SLM;
            double un, vn;
            val(nb, un, vn);
            uu = time_dir * un;
            vv = time_dir * vn;
        } else {
            const int k2 = k + 1 < nv ? k + 1 : 0;
            const double dax = wrap180(r.ln[k] - xp) * z0, day = (r.la[k] - yp) * SLM;
            const double dbx = wrap180(r.ln[k2] - xp) * z0, dby = (r.la[k2] - yp) * SLM;
            const double tx = dbx - dax, ty = dby - day;
            const double tt = tx * tx + ty * ty;
            if (tt <= 0.0) continue;
            const double proj = ((cx - dax) * tx + (cy - day) * ty) / tt;
            const double fx = dax + proj * tx, fy = day + proj * ty;
            ex = 2.0 * fx - cx;
            ey = 2.0 * fy - cy;
            if (bc == 1) {
                uu = -u_own;
                vv = -v_own;
            } else {
                const double ut = (u_own * tx + v_own * ty) / tt;
                uu = 2.0 * ut * tx - u_own;
                vv = 2.0 * ut * ty - v_own;
            }
        }
        a11 = a11 + 1.0;
        a12 = a12 + ex;
        a13 = a13 + ey;
        a22 = a22 + ex * ex;
        a23 = a23 + ex * ey;
        a33 = a33 + ey * ey;
        fU = fU + uu;
        f1U = f1U + uu * ex;
        f2U = f2U + uu * ey;
        fV = fV + vv;
        f1V = f1V + vv * ex;
        f2V = f2V + vv * ey;
    }
    const double a21 = a12, a31 = a13, a32 = a23;
    const double det = a11 * a22 * a33 + a12 * a23 * a31 + a13 * a21 * a32 - a13 * a22 * a31 - a12 * a21 * a33 -
                       a11 * a23 * a32;
    if (fabs(det) < 1e-30 || fabs(det) < 1e-12 * fabs(a11 * a22 * a33)) return false;
    const double inv = 1.0 / fabs(det);
    const double b11 = a22 * a33 - a23 * a32;
    const double b12 = a13 * a32 - a12 * a33;
    const double b13 = a12 * a23 - a13 * a22;
    U = (b11 * fU + b12 * f1U + b13 * f2U) * inv;
    V = (b11 * fV + b12 * f1V + b13 * f2V) * inv;
    return true;
}

// ---------------------------------------------------------------------------
// Counter RNG (diffusion.py:180-249): a keyed SplitMix64 chain over
// (seed, realization, particle, step, component), split into two open-(0,1)
// uniforms, Box-Muller to a normal pair.
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x = x + 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    x = x ^ (x >> 31);
    return x;
}

__device__ __forceinline__ uint64_t key_hash(uint64_t k0, uint64_t k1, uint64_t k2, uint64_t k3, uint64_t k4) {
    uint64_t h = k0;
    h = splitmix64(h ^ k1);
    h = splitmix64(h ^ k2);
    h = splitmix64(h ^ k3);
    h = splitmix64(h ^ k4);
    return h;
}

// The table entry code of index j (0: none): the bucket's entries (about 11
// in table b, 2 in table a) scanned in order.
__device__ __forceinline__ unsigned rngx_code(const unsigned* off, const unsigned short* ent, unsigned j) {
    const unsigned b = j >> 12, lo = j & 0xFFFu;
    const unsigned e = __ldg(&off[b + 1]);
    for (unsigned k = __ldg(&off[b]); k < e; ++k) {
        const unsigned v = __ldg(&ent[k]);
        if ((v >> 4) >= lo) return (v >> 4) == lo ? (v & 15u) : 0u;
    }
    return 0u;
}

// one-bit move of a double's bit pattern: code 1 up, 2 down
__device__ __forceinline__ double rngx_bump(double v, unsigned code) {
    const long long b = __double_as_longlong(v);
    return __longlong_as_double(code == 1u ? b + 1 : b - 1);
}

// The draw of the reference (diffusion.py:222-249).  EXACT (the plain
// form): log, cos and sin correctly rounded (kc_crmath.cuh), then moved to
// the host C library's value at the inputs listed in the exception tables x,
// so the pair equals the reference's bit for bit for every key.  Otherwise
// (the mixed form) CUDA's log and sincos.
template <bool EXACT>
__device__ __forceinline__ void normal_pair(const DRngX& x, uint64_t seed, uint64_t real_id, uint64_t pid,
                                            uint64_t step, uint64_t comp, double& g1, double& g2) {
    if constexpr (!EXACT) {
        const uint64_t h = key_hash(seed, real_id, pid, step, comp);
        const double INV = 1.0 / 4294967296.0;
        const double u1 = (double)(h >> 32) * INV + 0.5 * INV;
        const double u2 = (double)(h & 0xFFFFFFFFull) * INV + 0.5 * INV;
        const double r = sqrt(-2.0 * log(u1));
        double sn, cs;
        sincos(2.0 * 3.141592653589793 * u2, &sn, &cs);
        g1 = r * cs;
        g2 = r * sn;
        return;
    }
    uint64_t h = key_hash(seed, real_id, pid, step, comp);
    const double INV = 1.0 / 4294967296.0;
    const double HALF = 0.5 * INV;
    const unsigned j1 = (unsigned)(h >> 32), j2 = (unsigned)(h & 0xFFFFFFFFull);
    double u1 = (double)j1 * INV + HALF;
    double u2 = (double)j2 * INV + HALF;
    const double TWO_PI = 2.0 * 3.141592653589793;
    const unsigned ca = x.a_off ? rngx_code(x.a_off, x.a, j1) : 0u;
    const unsigned cb = x.b_off ? rngx_code(x.b_off, x.b, j2) : 0u;
    double r = sqrt(-2.0 * cr::log_cr(u1));
    double sn, cs;
    cr::sincos_cr(TWO_PI * u2, &sn, &cs);
    if (ca) r = rngx_bump(r, ca);
    if (cb & 3u) cs = rngx_bump(cs, cb & 3u);
    if (cb >> 2) sn = rngx_bump(sn, cb >> 2);
    g1 = r * cs;
    g2 = r * sn;
}

constexpr double R_METRIC = SLM / DEG2RAD;

// diffusion.py:538-575 sphere_displace (exponential map of the tangent kick);
// sin/cos of the start longitude and latitude come from its evaluation site.
template <bool EXACT>
__device__ __forceinline__ void sphere_displace(const Site& q, double dx, double dy, double& lon2, double& lat2) {
    double dist = sqrt(dx * dx + dy * dy);
    if (dist == 0.0) { lon2 = q.lon; lat2 = q.lat; return; }
    const double cl = q.cos_lon, sl = q.sin_lon, cp = q.cos_lat, sp = q.sin_lat;
    double delta = dist / R_METRIC;
    double sdel, c;
    if constexpr (EXACT) {
        const double2 sc = cr::sincos_cr_k(delta);
        sdel = sc.x;
        c = sc.y;
    } else {
        sincos(delta, &sdel, &c);
    }
    double s = sdel / dist;
    double tx = -sl * dx - sp * cl * dy;
    double ty = cl * dx - sp * sl * dy;
    double tz = cp * dy;
    double x2 = cp * cl * c + tx * s;
    double y2 = cp * sl * c + ty * s;
    double z2 = sp * c + tz * s;
    if (z2 > 1.0) z2 = 1.0;
    else if (z2 < -1.0) z2 = -1.0;
    lat2 = asin(z2) / DEG2RAD;
    lon2 = atan2(y2, x2) / DEG2RAD;
    lon2 = wrap180(lon2);
}

}  // namespace kc
