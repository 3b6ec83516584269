// The mixed-precision form of the stage evaluation: the nearest node, the
// containing element, the layer / data-point bracket and every other
// decision that selects which values are read stay in float64 and are the
// plain form's own functions (so the element path is the reference's); the
// vertex weights, the time blends and the vertical blends run in float32 on
// float32 or scaled float16 snapshots.  Positions stay float64.
//
// Differences from the plain form, by design: the weights are computed in
// the element's frame anchored at its first vertex (barycentric and
// Wachspress coordinates are invariant under that translation and under a
// common scale of both axes, so only the cos(latitude) anisotropy is kept),
// and W barycentric takes its element from the u/v containment scan of the
// same point (contain_local_w), running its own float64 search only when that
// scan cannot decide, and reuses the u/v weights when the elements agree.
#pragma once
#include <cuda_fp16.h>
#include <type_traits>
#include "kc_step.cuh"

namespace kc {

template <typename T>
__device__ __forceinline__ float ldf(const T* p, long long i);
template <>
__device__ __forceinline__ float ldf<float>(const float* p, long long i) { return __ldg(p + i); }
template <>
__device__ __forceinline__ float ldf<__half>(const __half* p, long long i) { return __half2float(__ldg(p + i)); }

// One stored value at (row, node), scale applied for half storage.
template <typename T>
__device__ __forceinline__ float fval(const T* a, const float* sc, int row, long long n, int node) {
    const float x = ldf<T>(a, (long long)row * n + node);
    if constexpr (std::is_same<T, __half>::value) return x * __ldg(sc + row);
    return x;
}

// The nested time blend of interpolate.py:1404-1436 in float32; which
// branch applies is decided from the float64 alphas, as in the plain form.
struct TBlendF {
    int mode;        // 0: a; 1: a,b at alpha0; 2: t; 3: a,t at alpha; 4: (a,b at alpha0), t at alpha
    float alpha0, alpha;
};

__device__ __forceinline__ TBlendF tblend_mode(double alpha0, double alpha) {
    TBlendF t;
    t.alpha0 = (float)alpha0;
    t.alpha = (float)alpha;
    if (alpha < 1e-12) t.mode = alpha0 == 0.0 ? 0 : 1;
    else if (alpha > 1.0 - 1e-12) t.mode = 2;
    else t.mode = alpha0 == 0.0 ? 3 : 4;
    return t;
}

template <typename T>
__device__ __forceinline__ float blend_val(const TBlendF& tb, const T* pa, const float* sa, const T* pb,
                                           const float* sb, const T* pt, const float* st, int row, long long n,
                                           int node) {
    switch (tb.mode) {
        case 0: return fval<T>(pa, sa, row, n, node);
        case 1: return (1.0f - tb.alpha0) * fval<T>(pa, sa, row, n, node) + tb.alpha0 * fval<T>(pb, sb, row, n, node);
        case 2: return fval<T>(pt, st, row, n, node);
        case 3: return (1.0f - tb.alpha) * fval<T>(pa, sa, row, n, node) + tb.alpha * fval<T>(pt, st, row, n, node);
        default: {
            const float a0 = (1.0f - tb.alpha0) * fval<T>(pa, sa, row, n, node) +
                             tb.alpha0 * fval<T>(pb, sb, row, n, node);
            return (1.0f - tb.alpha) * a0 + tb.alpha * fval<T>(pt, st, row, n, node);
        }
    }
}

template <typename T>
__device__ __forceinline__ float blend_u(const DBlend<T>& f, const TBlendF& tb, int row, int node) {
    return blend_val<T>(tb, f.a.u, f.a.su, f.b.u, f.b.su, f.t.u, f.t.su, row, f.n, node);
}
template <typename T>
__device__ __forceinline__ float blend_v(const DBlend<T>& f, const TBlendF& tb, int row, int node) {
    return blend_val<T>(tb, f.a.v, f.a.sv, f.b.v, f.b.sv, f.t.v, f.t.sv, row, f.n, node);
}
template <typename T>
__device__ __forceinline__ float blend_w(const DBlend<T>& f, const TBlendF& tb, int row, int node) {
    return blend_val<T>(tb, f.a.w, f.a.sw, f.b.w, f.b.sw, f.t.w, f.t.sw, row, f.n, node);
}

// Vertex weights of the point in element `elem` (its compacted ring, as
// load_ring compacts it), in float32 in the frame of the ring's first vertex:
// v[0..n-1] the vertex ids, w[0..n-1] their weights (w[3] = 0 for a
// triangle).  Only the float offsets stay live, never the double
// coordinates, and every array index is a compile-time constant.
__device__ __forceinline__ bool weights_f32(const DMesh& m, int elem, double xp, double yp, int* v, float* w,
                                            int& nv) {
    const int4 e = __ldg(&m.en[elem]);
    int n = 0, first = -1;
    v[0] = v[1] = v[2] = v[3] = -1;
    auto push = [&](int id) {
        if (n == 0) v[0] = id;
        else if (n == 1) v[1] = id;
        else if (n == 2) v[2] = id;
        else v[3] = id;
        ++n;
    };
    if (e.x >= 0) { push(e.x); first = e.x; }
    if (e.y >= 0 && !(n > 0 && e.y == first)) { push(e.y); if (first < 0) first = e.y; }
    if (e.z >= 0 && !(n > 0 && e.z == first)) { push(e.z); if (first < 0) first = e.z; }
    if (e.w >= 0 && !(n > 0 && e.w == first)) push(e.w);
    nv = n;
    if (n < 3) return false;
    if (n == 3) v[3] = v[0];
    const float cl = (float)__ldg(&m.ecos[elem]).y;
    const double2 a0 = __ldg(&m.ll[v[0]]);
    float x[4], y[4];
    x[0] = 0.0f;
    y[0] = 0.0f;
#pragma unroll
    for (int k = 1; k < 4; ++k) {
        const double2 a = __ldg(&m.ll[v[k]]);
        x[k] = (float)wrap180(a.x - a0.x) * cl;
        y[k] = (float)(a.y - a0.y);
    }
    const float px = (float)wrap180(xp - a0.x) * cl;
    const float py = (float)(yp - a0.y);
    if (n == 3) {
        const float denom = (y[1] - y[2]) * (x[0] - x[2]) + (x[2] - x[1]) * (y[0] - y[2]);
        if (!(fabsf(denom) > 0.0f)) return false;
        w[0] = ((y[1] - y[2]) * (px - x[2]) + (x[2] - x[1]) * (py - y[2])) / denom;
        w[1] = ((y[2] - y[0]) * (px - x[2]) + (x[0] - x[2]) * (py - y[2])) / denom;
        w[2] = 1.0f - w[0] - w[1];
        w[3] = 0.0f;
        return true;
    }
    float A[4], Cc[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int i1 = (k + 1) & 3, im = (k + 3) & 3;
        A[k] = (x[k] - px) * (y[i1] - py) - (x[i1] - px) * (y[k] - py);
        Cc[k] = (x[k] - x[im]) * (y[i1] - y[im]) - (x[i1] - x[im]) * (y[k] - y[im]);
    }
    float sum = 0.0f;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        w[k] = Cc[k] * A[(k + 1) & 3] * A[(k + 2) & 3];
        sum += w[k];
    }
    const float inv = 1.0f / sum;
#pragma unroll
    for (int k = 0; k < 4; ++k) w[k] *= inv;
    return true;
}

// W of one node at depth z (the location decided in float64 by w_locate),
// z clamped to the node's depth as the barycentric W reads its vertices.
template <typename T>
__device__ __forceinline__ float w_node_f32(const DMesh& m, const DBlend<T>& f, const TBlendF& tb, double z,
                                            const WLoc& Lz, int nd, bool clamp) {
    const double zc = clamp ? pymin(z, __ldg(&m.depth[nd])) : z;
    const WLoc L = zc == z ? Lz : w_locate(m, zc);
    const float lo = blend_w<T>(f, tb, L.k, nd);
    if (L.a < 0.0) return lo;
    const float a = (float)L.a;
    return (1.0f - a) * lo + a * blend_w<T>(f, tb, L.k + 1, nd);
}

// One 2-D or 3-D stage of the mixed form at (xp, yp, z) with anchor nn:
// containment and the vertical decisions in float64, values in float32.
// DIMS 2 reads u/v row 0 and no W; DL: depth-linear u/v (uv_vertical level /
// layer_linear).  One function per combination, so each keeps only its own
// values live across its calls.
template <typename T, int DIMS, bool DL>
__device__ __forceinline__ bool stage_f32(const DMesh& m, const DBlend<T>& f, const DStep& s, double xp,
                                       double yp, int nn, int hint, int whint, double z, double alpha, double& U,
                                       double& V, double& W) {
    U = 0.0;
    V = 0.0;
    W = 0.0;
    const TBlendF tb = tblend_mode(f.alpha0, alpha);
    const float td = (float)s.time_dir;
    int w_elem = -1;
    bool w_unsure = false;
    // the W bookkeeping of the scan only where a barycentric W reads it; a
    // carried scan (hint, whint >= -2) replaces it, an edge-walk element
    // (hint, whint -3) replaces the u/v scan and the W search then runs
    int elem;
    if (hint >= 0) {
        elem = hint;
        if (whint >= -2) {
            w_elem = whint >= 0 ? whint : -1;
            w_unsure = whint == -2;
        } else {
            w_unsure = true;
        }
    } else {
        elem = (DIMS == 3 && s.w_code == 1) ? contain_local_w(m, xp, yp, nn, w_elem, w_unsure)
                                            : contain_local(m, xp, yp, nn);
    }
    int rv[4], rn = 0;
    float w[4];
    const bool ok = elem >= 0 && weights_f32(m, elem, xp, yp, rv, w, rn);
    if constexpr (DIMS == 3) {
        const WLoc Lz = w_locate(m, z);
        float Wf;
        if (s.w_code == 1) {
            // the barycentric W's own element (the reference's search
            // decides it; the containment scan usually already has)
            if (w_unsure) w_elem = w_search_elem(m, xp, yp, nn);
            if (w_elem >= 0) {
                Wf = 0.0f;
                if (ok && w_elem == elem) {   // the u/v weights
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        if (k < rn) Wf += w[k] * w_node_f32<T>(m, f, tb, z, Lz, rv[k], true);
                } else {
                    int wv[4], wn = 0;
                    float ww[4];
                    if (weights_f32(m, w_elem, xp, yp, wv, ww, wn)) {
#pragma unroll
                        for (int k = 0; k < 4; ++k)
                            if (k < wn) Wf += ww[k] * w_node_f32<T>(m, f, tb, z, Lz, wv[k], true);
                    } else {
                        Wf = w_node_f32<T>(m, f, tb, z, Lz, nn, true);
                    }
                }
            } else {
                Wf = w_node_f32<T>(m, f, tb, z, Lz, nn, true);   // its nodal fallback, z clamped
            }
        } else {
            Wf = w_node_f32<T>(m, f, tb, z, Lz, nn, false);      // W nearest: the anchor at z
        }
        W = (double)(td * Wf);
    }
    if (!ok) return false;
    float Us = 0.0f, Vs = 0.0f;
    if constexpr (DIMS == 3 && DL) {
        // depth-linear u/v with the wall rule (interpolate.py:1879-1971)
        double zq = z;
        if (isnan(zq)) zq = INFINITY;
        bool wet[4];
        int n_wet = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            wet[k] = k < rn && zq <= __ldg(&m.dl_bed[rv[k]]);
            n_wet += wet[k] ? 1 : 0;
        }
        if (n_wet == 0) {
            int nd = rv[0];
            double bd = __ldg(&m.dl_bed[rv[0]]);
#pragma unroll
            for (int k = 1; k < 4; ++k)
                if (k < rn) {
                    const double b = __ldg(&m.dl_bed[rv[k]]);
                    if (b > bd) { bd = b; nd = rv[k]; }
                }
            const int row = __ldg(&m.dl_last[nd]);
            U = (double)(td * blend_u<T>(f, tb, row, nd));
            V = (double)(td * blend_v<T>(f, tb, row, nd));
            return true;
        }
        float den = 1.0f;
        if (n_wet < rn) {
            float wsum = 0.0f;
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (wet[k]) {
                    if (w[k] < 0.0f) w[k] = 0.0f;
                    wsum += w[k];
                }
            if (wsum < 1e-12f) {
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if (wet[k]) w[k] = 1.0f;
                den = (float)n_wet;
            } else {
                den = wsum;
            }
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (k >= rn || (n_wet < rn && !wet[k])) continue;
            const int nd = rv[k];
            int kb;
            double ab;
            uv_bracket(m.dl_p, __ldg(&m.dl_last[nd]), zq, kb, ab);
            float un = blend_u<T>(f, tb, kb, nd), vn = blend_v<T>(f, tb, kb, nd);
            if (!(ab < 0.0)) {
                const float a = (float)ab;
                un = (1.0f - a) * un + a * blend_u<T>(f, tb, kb + 1, nd);
                vn = (1.0f - a) * vn + a * blend_v<T>(f, tb, kb + 1, nd);
            }
            Us += w[k] * un;
            Vs += w[k] * vn;
        }
        if (n_wet < rn) {
            Us /= den;
            Vs /= den;
        }
    } else {
        const int row = DIMS == 3 ? find_layer(m, z, nn) : 0;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (k < rn) {
                Us += w[k] * blend_u<T>(f, tb, row, rv[k]);
                Vs += w[k] * blend_v<T>(f, tb, row, rv[k]);
            }
    }
    U = (double)(td * Us);
    V = (double)(td * Vs);
    return true;
}

// The same stage behind a call boundary: the unfused 3-D RK4 / Euler step
// evaluates four stages, and four inlined copies of both vertical variants
// (eight in all) cost more in instruction fetch than the calls.
template <typename T, int DIMS, bool DL>
__device__ __noinline__ bool stage_f32_call(const DMesh& m, const DBlend<T>& f, const DStep& s, double xp, double yp,
                                            int nn, int hint, int whint, double z, double alpha, double& U,
                                            double& V, double& W) {
    return stage_f32<T, DIMS, DL>(m, f, s, xp, yp, nn, hint, whint, z, alpha, U, V, W);
}

// The mixed form as a step-body policy (see PlainForm in kc_step.cuh).  INL:
// the stage inlined into the kernel (the fused 3-D RK2 and the 2-D steps,
// measured 11 % faster on the 3-D RK2 step) or called (the unfused 3-D
// steps, UnfusedFormOf).
template <typename T, bool INL = true>
struct MixedForm {
    static constexpr bool kExact = false;   // CUDA's sincos for sites and draws
    static __device__ __forceinline__ Site site(double lon, double lat) { return make_site_fast(lon, lat); }
    static __device__ __forceinline__ bool uv2(const DMesh& m, const DBlend<T>& f, const DStep& s, double lon,
                                               double lat, int nn, int hint, double alpha, double& U, double& V) {
        double W;
        if constexpr (INL) return stage_f32<T, 2, false>(m, f, s, lon, lat, nn, hint, -3, 0.0, alpha, U, V, W);
        else return stage_f32_call<T, 2, false>(m, f, s, lon, lat, nn, hint, -3, 0.0, alpha, U, V, W);
    }
    static __device__ __forceinline__ bool uvw3(const DMesh& m, const DBlend<T>& f, const DStep& s, double lon,
                                                double lat, int nn, int hint, int whint, double z, double alpha,
                                                double& U, double& V, double& W) {
        if constexpr (INL)
            return s.uv_dl ? stage_f32<T, 3, true>(m, f, s, lon, lat, nn, hint, whint, z, alpha, U, V, W)
                           : stage_f32<T, 3, false>(m, f, s, lon, lat, nn, hint, whint, z, alpha, U, V, W);
        else
            return s.uv_dl ? stage_f32_call<T, 3, true>(m, f, s, lon, lat, nn, hint, whint, z, alpha, U, V, W)
                           : stage_f32_call<T, 3, false>(m, f, s, lon, lat, nn, hint, whint, z, alpha, U, V, W);
    }
};

template <typename T>
struct UnfusedFormOf<MixedForm<T, true>> {
    using type = MixedForm<T, false>;
};

}  // namespace kc
