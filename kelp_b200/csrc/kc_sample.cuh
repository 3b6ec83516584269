// Scalar field sampling at particle positions: KELP's numerics/sampling.py
// sample_field for node fields of shape (N,) and z-level mid-layer fields
// (K-1, N), with the four horizontal rules (nearest, leastsq, barycentric,
// idw).  One thread per particle.  The neighbour stencil is not gathered
// into an array: the anchor's ring of distinct nodes is visited in the
// reference's order straight from the node->element table, and each rule
// accumulates in that order, so the sums round as the reference's do.
#pragma once
#include "kc_interp.cuh"

namespace kc {

constexpr int S_NEAREST = 0, S_LEASTSQ = 1, S_BARYCENTRIC = 2, S_IDW = 3;

struct DSample {
    const double* values;   // (N) or (rows, N), float64
    const double* zm;       // (rows) mid-layer depths, positive down (z-level meshes)
    long long n;            // N
    int rows;               // 0: a 2-D field; >= 1: a mid-layer field
    const double* sig;      // (rows + 1) sigma interfaces of a sigma mesh, else null
    const double* eta;      // (N) the free surface of a sigma mesh's columns
    double Dmin;            // the sigma columns' floor
};


// sampling.py:432-484 _interp_mid_linear_single: linear between the
// mid-layer values around z, clamped to the first / last layer.  The
// bracket is the first k with z < zm[k + 1] (a binary search finds the same
// k in the non-decreasing zm; a NaN z takes the last layer, as the scan does).
__device__ __forceinline__ double mid_linear(const DSample& S, double z, int node, double H = -1.0) {
    const int K1 = S.rows;
    const double* f = S.values;
    // the mid-layer depths: the mesh's, or a sigma column's of height H
    // (sampling.py:598-601: (1 - (s_m + s_m+1) / 2) H)
    auto zm_at = [&](int k) { return S.sig ? (1.0 - 0.5 * (S.sig[k] + S.sig[k + 1])) * H : S.zm[k]; };
    if (K1 == 1) return f[node];
    if (z <= zm_at(0)) return f[node];
    if (z >= zm_at(K1 - 1) || isnan(z)) return f[(long long)(K1 - 1) * S.n + node];
    int lo = 1, hi = K1 - 1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (z < zm_at(mid)) hi = mid;
        else lo = mid + 1;
    }
    const int k = lo - 1;
    const double zk = zm_at(k), zk1 = zm_at(k + 1);
    const double dz = zk1 - zk;
    if (dz < 1e-12) return f[(long long)k * S.n + node];
    const double a = (z - zk) / dz;
    return (1.0 - a) * f[(long long)k * S.n + node] + a * f[(long long)(k + 1) * S.n + node];
}

// The value of node nd the stencil uses: the field itself (2-D), or the
// mid-layer column at the particle depth clamped to the node's bottom
// (sampling.py:528-531).
__device__ __forceinline__ double node_value(const DMesh& m, const DSample& S, double z_p, int nd) {
    if (S.rows == 0) return S.values[nd];
    if (S.sig) {   // sampling.py:586-605: the node's column max(depth + eta, Dmin), z clamped to it
        double H = m.depth[nd] + S.eta[nd];
        if (H < S.Dmin) H = S.Dmin;
        return mid_linear(S, z_p < H ? z_p : H, nd, H);
    }
    const double bot = m.depth[nd];
    return mid_linear(S, z_p < bot ? z_p : bot, nd);
}

// Whether node nd is among the ring's first kRingMax distinct nodes (the
// reference looks a vertex's value up in that stencil).
__device__ __forceinline__ bool in_ring(const DMesh& m, int nn, int nd) {
    bool found = false;
    for_ring(m, nn, [&](int x) {
        found = x == nd;
        return !found;
    });
    return found;
}

// Whether the ring has more distinct nodes than the stencil keeps.
__device__ __forceinline__ bool ring_over_cap(const DMesh& m, int nn) {
    int count = 1;
    const int s = m.n2e_off[nn], e = m.n2e_off[nn + 1];
    for (int k = s; k < e; ++k) {
        const int4 ek = m.en[m.n2e[k]];
        for (int v = 0; v < 4; ++v) {
            const int nd = slot_of(ek, v);
            if (nd < 0 || nd == nn) continue;
            bool dup = false;
            for (int u = 0; u < v && !dup; ++u) dup = slot_of(ek, u) == nd;
            for (int kk = s; kk < k && !dup; ++kk) {
                const int4 ej = m.en[m.n2e[kk]];
                dup = ej.x == nd || ej.y == nd || ej.z == nd || ej.w == nd;
            }
            if (!dup && ++count > kRingMax) return true;
        }
    }
    return false;
}

// sampling.py:82-380 _combine_horizontal at (lon_p, lat_p, z_p) with anchor
// nn, the reference's fallback (the anchor's own value) included.  The cos
// of a latitude is the correctly rounded one, the C library's value but
// where the library misrounds.
__device__ __forceinline__ double sample_point(const DMesh& m, const DSample& S, double lon_p, double lat_p,
                                               double z_p, int nn, int method) {
    const double fallback = node_value(m, S, z_p, nn);
    if (method == S_NEAREST) return fallback;
    if (method == S_IDW) {
        double z0 = cr::cos_cr(lat_p * DEG2RAD) * SLM;
        if (z0 < 1.0) z0 = 1.0;
        double sw = 0.0, swv = 0.0, hit_val = 0.0;
        bool hit = false;
        for_ring(m, nn, [&](int nd) {
            const double val = node_value(m, S, z_p, nd);
            const double2 a = m.ll[nd];
            const double dx = wrap180(a.x - lon_p) * z0;
            const double dy = (a.y - lat_p) * SLM;
            const double d2 = dx * dx + dy * dy;
            if (d2 < 1e-12) {   // on the node: its raw value
                hit = true;
                hit_val = val;
                return false;
            }
            if (!isfinite(val)) return true;
            const double w = 1.0 / d2;
            sw += w;
            swv += w * val;
            return true;
        });
        if (hit) return hit_val;
        if (sw < 1e-30) return fallback;
        return swv / sw;
    }
    if (method == S_LEASTSQ) {
        double z0 = cr::cos_cr(lat_p * DEG2RAD) * SLM;
        if (z0 < 1.0) z0 = 1.0;
        double a11 = 0.0, a12 = 0.0, a13 = 0.0, a22 = 0.0, a23 = 0.0, a33 = 0.0, f0 = 0.0, f1 = 0.0, f2 = 0.0;
        int nfin = 0;
        const int cnt = for_ring(m, nn, [&](int nd) {
            const double val = node_value(m, S, z_p, nd);
            if (!isfinite(val)) return true;
            ++nfin;
            const double2 a = m.ll[nd];
            const double ex = wrap180(a.x - lon_p) * z0;
            const double ey = (a.y - lat_p) * SLM;
            a11 += 1.0;
            a12 += ex;
            a13 += ey;
            a22 += ex * ex;
            a23 += ex * ey;
            a33 += ey * ey;
            f0 += val;
            f1 += val * ex;
            f2 += val * ey;
            return true;
        });
        if (cnt < 3 || nfin < 3) return fallback;
        const double a21 = a12, a31 = a13, a32 = a23;
        const double det = a11 * a22 * a33 + a12 * a23 * a31 + a13 * a21 * a32 - a13 * a22 * a31 - a12 * a21 * a33 -
                           a11 * a23 * a32;
        if (fabs(det) < 1e-12 || fabs(det) < 1e-12 * fabs(a11 * a22 * a33)) return fallback;
        const double inv = 1.0 / fabs(det);
        const double b11 = a22 * a33 - a23 * a32, b12 = a13 * a32 - a12 * a33, b13 = a12 * a23 - a13 * a22;
        return (b11 * f0 + b12 * f1 + b13 * f2) * inv;
    }
    // barycentric: the first fan triangle of the anchor's elements that
    // holds the point (denominator tolerance 1e-14, eps -1e-6); Wachspress
    // over a quad's four vertices
    const int s = m.n2e_off[nn], e = m.n2e_off[nn + 1];
    for (int k = s; k < e; ++k) {
        const int4 ek = m.en[m.n2e[k]];
        int verts[4], nv = 0;
        for (int v = 0; v < 4; ++v) {
            const int nd = slot_of(ek, v);
            if (nd < 0 || (nv > 0 && nd == verts[0])) continue;
            verts[nv++] = nd;
        }
        if (nv < 3) continue;
        double ln[4], vx[4], vy[4];
        double lat0 = 0.0;
        for (int v = 0; v < nv; ++v) {
            const double2 a = m.ll[verts[v]];
            ln[v] = a.x;
            vy[v] = a.y;
            lat0 += a.y;
        }
        // mesh.py:1974-2003 _seam_safe_lon0
        double lmin = ln[0], lmax = ln[0], ssum = 0.0;
        for (int v = 0; v < nv; ++v) {
            ssum += ln[v];
            if (ln[v] < lmin) lmin = ln[v];
            if (ln[v] > lmax) lmax = ln[v];
        }
        double lon0;
        if (lmax - lmin > 180.0) {
            double d = 0.0;
            for (int v = 0; v < nv; ++v) d += wrap180(ln[v] - ln[0]);
            lon0 = ln[0] + d / nv;
        } else {
            lon0 = ssum / nv;
        }
        lat0 /= nv;
        const double cl = cr::cos_cr(lat0 * DEG2RAD);
        for (int v = 0; v < nv; ++v) {
            vx[v] = wrap180(ln[v] - lon0) * DEG2RAD * R_STD * cl;
            vy[v] = (vy[v] - lat0) * DEG2RAD * R_STD;
        }
        const double px = wrap180(lon_p - lon0) * DEG2RAD * R_STD * cl;
        const double py = (lat_p - lat0) * DEG2RAD * R_STD;
        for (int t = 0; t < nv - 2; ++t) {
            const double ax = vx[0], ay = vy[0], bx = vx[t + 1], by = vy[t + 1], cx = vx[t + 2], cy = vy[t + 2];
            const double denom = (by - cy) * (ax - cx) + (cx - bx) * (ay - cy);
            if (fabs(denom) < 1e-14) continue;
            const double w1 = ((by - cy) * (px - cx) + (cx - bx) * (py - cy)) / denom;
            const double w2 = ((cy - ay) * (px - cx) + (ax - cx) * (py - cy)) / denom;
            const double w3 = 1.0 - w1 - w2;
            if (!(w1 >= -1e-6 && w2 >= -1e-6 && w3 >= -1e-6)) continue;
            const bool capped = ring_over_cap(m, nn);
            if (nv == 4) {
                double wts[4];
                wachspress_quad(px, py, vx, vy, wts);
                double acc = 0.0;
                for (int vi = 0; vi < 4; ++vi) {
                    if (capped && !in_ring(m, nn, verts[vi])) return fallback;
                    const double vv = node_value(m, S, z_p, verts[vi]);
                    if (!isfinite(vv)) return fallback;
                    acc += wts[vi] * vv;
                }
                return acc;
            }
            const int n0 = verts[0], n1 = verts[t + 1], n2 = verts[t + 2];
            if (capped && !(in_ring(m, nn, n0) && in_ring(m, nn, n1) && in_ring(m, nn, n2))) return fallback;
            const double v0 = node_value(m, S, z_p, n0), v1 = node_value(m, S, z_p, n1),
                         v2 = node_value(m, S, z_p, n2);
            if (!(isfinite(v0) && isfinite(v1) && isfinite(v2))) return fallback;
            return w1 * v0 + w2 * v1 + w3 * v2;
        }
    }
    return fallback;
}

}  // namespace kc
