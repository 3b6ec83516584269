// Device-side interpolation, time blending, vertical helpers, the counter RNG
// and the great-circle diffusion kick of the KELP time-stepping path.  Same
// floating-point operation order as the cited Numba functions (see the note
// at the top of kc_geom.cuh on -fmad=false).
#pragma once
#include "kc_geom.cuh"

namespace kc {

// Snapshot views: u/v rows are (L, N) row-major, w rows (K, N).
template <typename T>
struct DField {
    const T* u;
    const T* v;
    const T* w;
};

template <typename T>
struct DBlend {
    DField<T> a, b, t;   // bracket pair and stage target
    double alpha0;       // bracket fraction of the step's start time
    long long n;         // row stride (nodes)
};

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

// Vertex weights of the point in the containing element, projected around the
// wrapped-delta centroid (interpolate.py:1376-1402).  Returns false for the
// degenerate-triangle sentinel or an element with fewer than 3 vertices.
__device__ __forceinline__ bool bary_weights_core(const DMesh& m, int elem, double xp, double yp, double R,
                                                  int* verts, double* w, int& nv) {
    int4 e = __ldg(&m.en[elem]);
    int raw[4] = {e.x, e.y, e.z, e.w};
    nv = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        int nd = raw[k];
        if (nd < 0) continue;
        if (nv > 0 && nd == verts[0]) continue;
        verts[nv++] = nd;
    }
    if (nv < 3) return false;
    double ln[4], la[4];
    for (int k = 0; k < nv; ++k) {
        double2 p = __ldg(&m.ll[verts[k]]);
        ln[k] = p.x;
        la[k] = p.y;
    }
    double lon_ref = ln[0];
    double dsum = 0.0, lat0 = 0.0;
    for (int k = 0; k < nv; ++k) {
        dsum += wrap180(ln[k] - lon_ref);
        lat0 += la[k];
    }
    double lon0 = lon_ref + dsum / (double)nv;
    lat0 /= (double)nv;
    double cosl = cos(lat0 * DEG2RAD);
    double vx[4], vy[4];
    for (int k = 0; k < nv; ++k) {
        vx[k] = wrap180(ln[k] - lon0) * DEG2RAD * R * cosl;
        vy[k] = (la[k] - lat0) * DEG2RAD * R;
    }
    double px = wrap180(xp - lon0) * DEG2RAD * R * cosl;
    double py = (yp - lat0) * DEG2RAD * R;
    return polygon_weights(px, py, vx, vy, nv, w);
}

// interpolate.py:1340-1440 _interp_barycentric_core_tinterp (row = 0) and
// interpolate.py:1443-1529 its 3-D twin (row = the particle's layer).
template <typename T>
__device__ __forceinline__ bool interp_uv_bary(const DMesh& m, const DBlend<T>& f, double xp, double yp, int nn,
                                               double time_dir, int row, double alpha, double& U, double& V) {
    U = 0.0;
    V = 0.0;
    int elem = contain_local(m, xp, yp, nn);
    if (elem < 0) return false;
    int verts[4];
    double w[4];
    int nv;
    if (!bary_weights_core(m, elem, xp, yp, m.r_earth, verts, w, nv)) return false;
    const long long base = (long long)row * f.n;
    const double alpha0 = f.alpha0;
    const double beta0 = 1.0 - alpha0;
    const double beta = 1.0 - alpha;
    double Us = 0.0, Vs = 0.0;
    for (int k = 0; k < nv; ++k) {
        long long idx = base + verts[k];
        double un, vn;
        if (alpha < 1e-12) {
            if (alpha0 == 0.0) {
                un = (double)f.a.u[idx];
                vn = (double)f.a.v[idx];
            } else {
                un = beta0 * (double)f.a.u[idx] + alpha0 * (double)f.b.u[idx];
                vn = beta0 * (double)f.a.v[idx] + alpha0 * (double)f.b.v[idx];
            }
        } else if (alpha > 1.0 - 1e-12) {
            un = (double)f.t.u[idx];
            vn = (double)f.t.v[idx];
        } else if (alpha0 == 0.0) {
            un = beta * (double)f.a.u[idx] + alpha * (double)f.t.u[idx];
            vn = beta * (double)f.a.v[idx] + alpha * (double)f.t.v[idx];
        } else {
            double ua0 = beta0 * (double)f.a.u[idx] + alpha0 * (double)f.b.u[idx];
            double va0 = beta0 * (double)f.a.v[idx] + alpha0 * (double)f.b.v[idx];
            un = beta * ua0 + alpha * (double)f.t.u[idx];
            vn = beta * va0 + alpha * (double)f.t.v[idx];
        }
        Us += w[k] * un;
        Vs += w[k] * vn;
    }
    U = time_dir * Us;
    V = time_dir * Vs;
    return true;
}

// vertical.py:39-91 find_layer
__device__ __forceinline__ int find_layer(const DMesh& m, double z, double bottom) {
    const int K = m.K;
    const double* zl = m.zlev;
    if (K < 2) return 0;
    if (z <= zl[0]) return 0;
    int max_layer = K - 2;
    for (int k = 0; k < K - 1; ++k) {
        if (zl[k + 1] > bottom) {
            max_layer = k - 1 > 0 ? k - 1 : 0;
            break;
        }
    }
    if (z >= bottom || z >= zl[max_layer + 1]) return max_layer;
    for (int k = 0; k <= max_layer; ++k)
        if (z < zl[k + 1]) return k;
    return max_layer;
}

// vertical.py:1064-1098 _interp_w_linear_single_tinterp
template <typename T>
__device__ __forceinline__ double w_linear(const DMesh& m, const DBlend<T>& f, double alpha, double z, int node,
                                           double time_dir) {
    const int K = m.K;
    const double* zl = m.zlev;
    const long long n = f.n;
    auto at = [&](int k) {
        long long idx = (long long)k * n + node;
        return tblend((double)f.a.w[idx], (double)f.b.w[idx], (double)f.t.w[idx], f.alpha0, alpha);
    };
    if (K < 2) return time_dir * at(0);
    if (z <= zl[0]) return time_dir * at(0);
    if (z >= zl[K - 1]) return time_dir * at(K - 1);
    int k = K - 2;
    for (int j = 0; j < K - 1; ++j) {
        if (z < zl[j + 1]) { k = j; break; }
    }
    double dz = zl[k + 1] - zl[k];
    if (dz < 1e-12) return time_dir * at(k);
    double a = (z - zl[k]) / dz;
    double w_lo = at(k);
    double w_hi = at(k + 1);
    return time_dir * ((1.0 - a) * w_lo + a * w_hi);
}

// Python's min(a, b): the first argument unless the second is smaller.
__device__ __forceinline__ double pymin(double a, double b) { return b < a ? b : a; }

// mesh.py:1973-2003 _seam_safe_lon0
__device__ __forceinline__ double seam_safe_lon0(const double* ln, int n) {
    double first = ln[0], lmin = first, lmax = first, s = 0.0;
    for (int v = 0; v < n; ++v) {
        double x = ln[v];
        s += x;
        if (x < lmin) lmin = x;
        if (x > lmax) lmax = x;
    }
    if (lmax - lmin > 180.0) {
        double d = 0.0;
        for (int v = 0; v < n; ++v) d += wrap180(ln[v] - first);
        return first + d / (double)n;
    }
    return s / (double)n;
}

// vertical.py:744-881 _interp_w_bary_single_tinterp: the anchor's own fan
// search (denominator tolerance 1e-14, R = 6371000), triangles blended
// inline, quads through Wachspress, nearest-node fallback.
template <typename T>
__device__ __noinline__ double w_bary(const DMesh& m, const DBlend<T>& f, double alpha, double xp, double yp,
                                      double z, int node, double time_dir) {
    int s = m.n2e_off[node], e = m.n2e_off[node + 1];
    if (e == s) {
        double zc = pymin(z, m.depth[node]);
        return w_linear(m, f, alpha, zc, node, time_dir);
    }
    for (int kk = s; kk < e; ++kk) {
        int el = m.n2e[kk];
        int4 en = m.en[el];
        int raw[4] = {en.x, en.y, en.z, en.w};
        int verts[4];
        int nvv = 0;
        for (int v = 0; v < 4; ++v) {
            int nd = raw[v];
            if (nd < 0) continue;
            if (nvv > 0 && nd == verts[0]) continue;
            verts[nvv++] = nd;
        }
        if (nvv < 3) continue;
        double ln[4], la[4];
        for (int v = 0; v < nvv; ++v) {
            double2 p = m.ll[verts[v]];
            ln[v] = p.x;
            la[v] = p.y;
        }
        double lon0 = seam_safe_lon0(ln, nvv);
        double lat0 = 0.0;
        for (int v = 0; v < nvv; ++v) lat0 += la[v];
        lat0 /= (double)nvv;
        double cos_lat0 = cos(lat0 * DEG2RAD);
        const double R = 6371000.0;
        double vx[4], vy[4];
        for (int v = 0; v < nvv; ++v) {
            double dlon = wrap180(ln[v] - lon0);
            double dlat = la[v] - lat0;
            vx[v] = dlon * DEG2RAD * R * cos_lat0;
            vy[v] = dlat * DEG2RAD * R;
        }
        double px = wrap180(xp - lon0) * DEG2RAD * R * cos_lat0;
        double py = (yp - lat0) * DEG2RAD * R;
        for (int t = 0; t < nvv - 2; ++t) {
            int i1 = t + 1, i2 = t + 2;
            double ax = vx[0], ay = vy[0], bx = vx[i1], by = vy[i1], cx = vx[i2], cy = vy[i2];
            double denom = (by - cy) * (ax - cx) + (cx - bx) * (ay - cy);
            if (fabs(denom) < 1e-14) continue;
            double w1 = ((by - cy) * (px - cx) + (cx - bx) * (py - cy)) / denom;
            double w2 = ((cy - ay) * (px - cx) + (ax - cx) * (py - cy)) / denom;
            double w3 = 1.0 - w1 - w2;
            const double eps = -1e-6;
            if (w1 >= eps && w2 >= eps && w3 >= eps) {
                if (nvv == 4) {
                    double wts[4];
                    polygon_weights(px, py, vx, vy, 4, wts);
                    double acc = 0.0;
                    for (int vi = 0; vi < 4; ++vi) {
                        int nvn = verts[vi];
                        double z_nv = pymin(z, m.depth[nvn]);
                        acc += wts[vi] * w_linear(m, f, alpha, z_nv, nvn, time_dir);
                    }
                    return acc;
                }
                int n0 = verts[0], n1 = verts[i1], n2 = verts[i2];
                double w_v0 = w_linear(m, f, alpha, pymin(z, m.depth[n0]), n0, time_dir);
                double w_v1 = w_linear(m, f, alpha, pymin(z, m.depth[n1]), n1, time_dir);
                double w_v2 = w_linear(m, f, alpha, pymin(z, m.depth[n2]), n2, time_dir);
                return w1 * w_v0 + w2 * w_v1 + w3 * w_v2;
            }
        }
    }
    double zc = pymin(z, m.depth[node]);
    return w_linear(m, f, alpha, zc, node, time_dir);
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

__device__ __forceinline__ void normal_pair(uint64_t seed, uint64_t real_id, uint64_t pid, uint64_t step,
                                            uint64_t comp, double& g1, double& g2) {
    uint64_t h = key_hash(seed, real_id, pid, step, comp);
    const double INV = 1.0 / 4294967296.0;
    const double HALF = 0.5 * INV;
    double u1 = (double)((h >> 32) & 0xFFFFFFFFull) * INV + HALF;
    double u2 = (double)(h & 0xFFFFFFFFull) * INV + HALF;
    const double TWO_PI = 2.0 * 3.141592653589793;
    double r = sqrt(-2.0 * log(u1));
    g1 = r * cos(TWO_PI * u2);
    g2 = r * sin(TWO_PI * u2);
}

constexpr double R_METRIC = SLM / DEG2RAD;

// diffusion.py:538-575 sphere_displace (exponential map of the tangent kick)
__device__ __forceinline__ void sphere_displace(double lon, double lat, double dx, double dy,
                                                double& lon2, double& lat2) {
    double dist = sqrt(dx * dx + dy * dy);
    if (dist == 0.0) { lon2 = lon; lat2 = lat; return; }
    double lam = lon * DEG2RAD, phi = lat * DEG2RAD;
    double cl = cos(lam), sl = sin(lam), cp = cos(phi), sp = sin(phi);
    double delta = dist / R_METRIC;
    double c = cos(delta);
    double s = sin(delta) / dist;
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
