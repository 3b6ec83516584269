// Per-particle step bodies of the KELP time-stepping path: the fused 2-D
// barycentric Euler/RK2/RK4 steps with inline temporal blending, the fused
// 3-D RK2 step (z-level layers, W nearest/barycentric, surface/bottom clamp),
// and the split uniform-Kh random-walk kick applied to the particles that
// survived the deterministic step.  One thread owns one particle for the whole
// step, so every intermediate stays in registers; the searches, containment
// and interpolation are shared (non-inlined) device functions, which keeps
// the kernel's code footprint small under divergence.
#pragma once
#include <type_traits>
#include "kc_interp.cuh"

namespace kc {

// Structure-of-arrays particle state resident in HBM.
struct DState {
    double* lon;
    double* lat;
    double* z;
    int* status;
    int* nn;
    double* U;
    double* V;
    double* W;
    signed char* fr;
    const long long* pid;      // stable particle id (RNG key), index when null
    const int* rid;            // per-particle realization (RNG key), the step's real_id when null
    const int* release_step;   // delayed release (null: all released)
    int* prev;                 // status at the step's entry, for the beaching hook (null: not kept)
    unsigned char* nn_ok;      // bit 0: nn is the exact anchor of the current position; bit 1: el / wel hold
                               // its local containment scan (null: never trusted)
    int* elem;                 // carried containing element (elem_search walk), null: the local scan
    int* el;                   // the local scan's element at the current position and anchor
    int* wel;                  // what that scan implies for the barycentric W search: its element (>= 0),
                               // its nodal fallback (-1), undecided (-2), not evaluated (-3)
    long long P;
};

struct DStep {
    double dt, time_dir;
    double ak[4];              // stage alphas c_k * dt / dt_to_next
    int w_code;                // 3-D W: 0 nearest, 1 barycentric, 2 least squares, 3 inverse distance
    int uv_dl;                 // 3-D u/v: 0 layer, 1 depth-linear (level / layer_linear)
    int kick;                  // split uniform-Kh kick on/off
    double kh_x, kh_y;
    unsigned long long seed, real_id, step_i, pid_offset;
    long long global_step;     // for delayed release activation (-1: none)
    int az_on, az_field;       // vertical Az kick; Az from the snapshots' (K, N) az rows
    double az_const;
    double Dmin, z0b_min;      // sigma column floor and bed clearance
    double alpha_end;          // blend fraction of the end-of-step surface (sigma)
    int edge_bc;               // edge least-squares u/v: 0 freeslip, 1 noslip ghost values
    const double* eta_s;       // sigma: the tracking layer's surface at the step's start (N), or null
    const double* eta_e;       // sigma: the tracking layer's surface at the step's end (N), or null
    int sig_steady;            // sigma: a steady step (stage surfaces blend from start to end)
};

// displacement metric z0 = max(cos(lat) * 111120, 1) (integrators.py:2563-2565),
// cos(lat) from the site anchored at that latitude
// EXACT (the plain forms): cos(lat) correctly rounded, as the site of the
// anchor search may carry CUDA's value.
template <bool EXACT>
__device__ __forceinline__ double metric_z0f(const Site& q) {
    double z0 = (EXACT ? cr::cos_cr_k(q.lat * DEG2RAD) : q.cos_lat) * SLM;
    if (z0 < 1.0) z0 = 1.0;
    return z0;
}

__device__ __forceinline__ double metric_z0(const Site& q) {
    double z0 = q.cos_lat * SLM;
    if (z0 < 1.0) z0 = 1.0;
    return z0;
}

__device__ __forceinline__ double clamp_lat(double lat) {
    if (lat > 90.0) return 90.0;
    if (lat < -90.0) return -90.0;
    return lat;
}

// The anchor of the step's start position: the carried one when a kernel of
// this library computed it for exactly this position (the reference searches
// it afresh; the search is a pure function of the position, so the result is
// the same), else the exact search.
__device__ __forceinline__ int start_anchor(const DMesh& m, const DState& st, const Site& q0, int pre_nn,
                                            long long i) {
    if (st.nn_ok && (st.nn_ok[i] & 1) && pre_nn >= 0) return pre_nn;
    return site_anchor(m, q0);
}

// After a step: an ALIVE particle carries the anchor of its new position; a
// failed one sits at its start position and carries the start anchor, except
// after a reverted kick, which restores the carried anchor (trusted only when
// it equals the start anchor).
__device__ __forceinline__ void mark_anchor(const DState& st, long long i, int status, int nn_out, int node_i) {
    if (st.nn_ok) st.nn_ok[i] = (status == ALIVE || nn_out == node_i) ? 1 : 0;
}

// The containment scan of a step's start (position and anchor unchanged
// since the last step of this library computed it): the scan is a pure
// function of the two, so stage 1 reuses the end-of-step scan instead of
// repeating it.  eh = -1 / wh = -3 when nothing is carried.
__device__ __forceinline__ void carried_scan(const DState& st, long long i, int& eh, int& wh) {
    eh = -1;
    wh = -3;
    if (st.el && st.nn_ok && (st.nn_ok[i] & 2)) {
        eh = st.el[i];
        wh = st.wel[i];
    }
}

// After mark_anchor: keep the scan of the particle's final position (el >= 0).
__device__ __forceinline__ void mark_scan(const DState& st, long long i, int status, int el, int wel) {
    if (st.el && st.nn_ok && status == ALIVE && el >= 0) {
        st.el[i] = el;
        st.wel[i] = wel;
        st.nn_ok[i] |= 2;
    }
}

// The end-of-step containment in local mode: the scan at the new position and
// its exact anchor, with the barycentric W search's information when the
// step reads W that way (wel, for the next step's first stage).
__device__ __forceinline__ int end_scan(const DMesh& m, bool want_w, double lon, double lat, int nn, int& wel) {
    if (want_w) {
        int we;
        bool wu;
        const int e = contain_local_w(m, lon, lat, nn, we, wu);
        wel = wu ? -2 : we;
        return e;
    }
    wel = -3;
    return contain_local(m, lon, lat, nn);
}

// The realization key of particle i: its own when the particles carry one
// (several ensemble members in one array), else the step's.
__device__ __forceinline__ unsigned long long realization_of(const DState& st, const DStep& s, long long i) {
    return st.rid ? (unsigned long long)st.rid[i] : s.real_id;
}

// Walk mode (elem_search: walk, integrators.py:5019-5147, :5415-5608,
// :5792-6011): the containing element of a stage position walked from the
// previous stage's, handed to the interpolation in place of its local scan;
// -1 (no hint) in local mode.
template <bool WALK>
__device__ __forceinline__ int stage_elem(const DMesh& m, double lon, double lat, int from, int nn) {
    if constexpr (WALK) return walk_locate(m, lon, lat, from, nn);
    else return -1;
}

// The end-of-step containment: the walk from the last stage's element, or the
// local scan around the exact anchor of the new position.
template <bool WALK>
__device__ __forceinline__ int end_elem(const DMesh& m, double lon, double lat, int from, int nn) {
    if constexpr (WALK) return walk_locate(m, lon, lat, from, nn);
    else return contain_local(m, lon, lat, nn);
}

// integrators.py:673-818 _apply_split_diffusion_kick for one particle that is
// ALIVE after the deterministic step (site qn = its position): counter-RNG
// kick (diffusion.py:485-529, :261-298), great-circle move, exact re-anchor
// and containment re-check, revert to the pre-step state on leaving the
// domain; 3-D reclamp in the new column.
template <bool EXACT>
static __device__ KC_INL_KICK void apply_kick(const DMesh& m, const DStep& s, long long pid, unsigned long long rid,
                                        const Site& qn,
                                        double pre_lon, double pre_lat, double pre_z, int pre_nn, bool is3d,
                                        double& lon, double& lat, double& z, int& status, int& nn, signed char& fr,
                                        bool want_w, int& kel, int& kwel) {
    double g1, g2;
    normal_pair<EXACT>(m.rx, s.seed, rid, (unsigned long long)pid + s.pid_offset, s.step_i, 0ull, g1, g2);
    double abs_dt = s.dt >= 0.0 ? s.dt : -s.dt;
    double sq = sqrt(abs_dt);
    double sx = sqrt(2.0 * s.kh_x);
    double sy = sqrt(2.0 * s.kh_y);
    double dx = sx * sq * g1;
    double dy = sy * sq * g2;
    if (s.kh_x != s.kh_y) {
        double la = lat;
        if (la < -89.9) la = -89.9;
        if (la > 89.9) la = 89.9;
        double corr = (s.kh_x - s.kh_y) * tan(la * DEG2RAD) / R_METRIC * abs_dt;
        dy = dy + corr;
    }
    double lk, lak;
    if constexpr (EXACT) sphere_displace<true>(make_site(qn.lon, qn.lat), dx, dy, lk, lak);   // correctly rounded trig
    else sphere_displace<false>(qn, dx, dy, lk, lak);
    Site qk = make_site_fast(lk, lak);   // the anchor search of the kicked position only
    int nk = site_anchor(m, qk);
    kel = end_scan(m, want_w, lk, lak, nk, kwel);
    if (kel < 0) {
        status = OUTSIDE;
        lon = pre_lon;
        lat = pre_lat;
        z = pre_z;
        nn = pre_nn;
        fr = (signed char)FR_OOB;
        return;
    }
    lon = lk;
    lat = lak;
    nn = nk;
    if (is3d) {
        double zv = z;
        if (zv < m.zlev[0]) zv = m.zlev[0];
        double bottom = m.depth[nk];
        if (zv > bottom) zv = bottom;
        z = zv;
    }
}

// diffusion.py:333-352 reflect_depth: specular fold into [top, bot] (Python's
// float % for the positive divisor 2L).
__device__ __forceinline__ double reflect_depth(double z, double top, double bot) {
    const double L = bot - top;
    if (L <= 0.0) return top;
    const double L2 = 2.0 * L;
    double y = fmod(z - top, L2);
    if (y != 0.0) {
        if (y < 0.0) y += L2;
    } else {
        y = 0.0;
    }
    if (y < 0.0) y += L2;
    if (y > L) y = L2 - y;
    return top + y;
}

// The payload's Az at interface k of node: the step-start field, a single
// snapshot or the pair blended at alpha0 (io.py:68-117).
template <typename T>
__device__ __forceinline__ double az_at(const DBlend<T>& f, int k, int node) {
    const long long idx = (long long)k * f.n + node;
    const double a = (double)__ldg(&f.a.az[idx]);
    if (f.alpha0 == 0.0) return a;
    const double b = (double)__ldg(&f.b.az[idx]);
    return (1.0 - f.alpha0) * a + f.alpha0 * b;
}

// integrators.py:842-938 _apply_split_az_kick for one particle ALIVE after
// the deterministic step and the horizontal kick: Az and dAz/dz on the
// anchor's column (diffusion.py:357-423, the evaluation depth clamped to the
// wet column, the slope of the segment holding it), or the constant; the
// Euler-Maruyama increment with the Ito drift, both on |dt| (:302-330), the
// vertical counter-RNG component; reflective bounds [z_levels[0],
// depth[anchor]] (:426-455).
template <typename T, bool EXACT>
__device__ __noinline__ void apply_az(const DMesh& m, const DBlend<T>& f, const DStep& s, long long pid,
                                      unsigned long long rid, int nn, double& z) {
    double az = s.az_const, g = 0.0;
    const double bottom = __ldg(&m.depth[nn]);
    if (s.az_field) {
        const int K = m.K;
        const double* zl = m.zlev;
        const double top = __ldg(&zl[0]);
        double bot = bottom < __ldg(&zl[K - 1]) ? bottom : __ldg(&zl[K - 1]);
        if (bot < top) bot = top;
        double ze = z;
        if (ze < top) ze = top;
        if (ze > bot) ze = bot;
        // first segment k with ze <= zl[k + 1] (K - 2 when none)
        int k = K - 2;
        if (K >= 2) {
            int lo = 0, hi = K - 2;
            if (!(ze <= __ldg(&zl[K - 1]))) lo = hi;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (ze <= __ldg(&zl[mid + 1])) hi = mid;
                else lo = mid + 1;
            }
            k = lo;
        }
        if (K < 2 || ze <= __ldg(&zl[0])) az = az_at(f, 0, nn);
        else if (ze >= __ldg(&zl[K - 1])) az = az_at(f, K - 1, nn);
        else {
            const double dzl = __ldg(&zl[k + 1]) - __ldg(&zl[k]);
            if (dzl <= 0.0) az = az_at(f, k, nn);
            else {
                const double frac = (ze - __ldg(&zl[k])) / dzl;
                az = (1.0 - frac) * az_at(f, k, nn) + frac * az_at(f, k + 1, nn);
            }
        }
        if (K >= 2) {
            const double dz = __ldg(&zl[k + 1]) - __ldg(&zl[k]);
            if (dz > 0.0) {
                if (std::is_same<T, float>::value && f.alpha0 == 0.0) {
                    // an unblended float32 snapshot: the difference of two
                    // float32 values rounds in float32 (numpy promotion)
                    const float d = (float)az_at(f, k + 1, nn) - (float)az_at(f, k, nn);
                    g = (double)d / dz;
                } else {
                    g = (az_at(f, k + 1, nn) - az_at(f, k, nn)) / dz;
                }
            }
        }
    }
    if (az < 0.0) {
        az = 0.0;
        g = 0.0;
    }
    double xi, unused;
    normal_pair<EXACT>(m.rx, s.seed, rid, (unsigned long long)pid + s.pid_offset, s.step_i, 1ull, xi, unused);
    const double sdt = s.time_dir * s.dt;
    const double abs_dt = sdt >= 0.0 ? sdt : -sdt;
    const double dz = g * abs_dt + sqrt(2.0 * az * abs_dt) * xi;
    z = reflect_depth(z + dz, __ldg(&m.zlev[0]), bottom);
}

// integrators.py:2521-2638 (RK2), :2641-2816 (RK4); Euler follows the
// per-particle arithmetic of the unfused path (integrators.py:4997-5147):
// one stage at the start, move, re-anchor, domain check.
template <typename T, int SCHEME, typename Form, bool WALK = false>
__device__ __forceinline__ void step2d_particle(const DMesh& m, const DBlend<T>& f, const DState& st,
                                                const DStep& s, long long i) {
    int status = st.status[i];
    if (status != ALIVE) {
        st.U[i] = 0.0;
        st.V[i] = 0.0;
        return;
    }
    const double lon0 = st.lon[i], lat0 = st.lat[i];
    const int pre_nn = st.nn[i];
    const double dt = s.dt, td = s.time_dir;
    double lon_new = lon0, lat_new = lat0;
    int nn_out = pre_nn;
    signed char fr = st.fr[i];
    bool failed = false;
    const Site q0 = Form::site(lon0, lat0);
    const int node_i = start_anchor(m, st, q0, pre_nn, i);
    const int e1 = stage_elem<WALK>(m, lon0, lat0, WALK ? st.elem[i] : -1, node_i);
    int e_last = e1, e_out = e1;
    int eh = e1, wh = -3;
    if constexpr (!WALK) carried_scan(st, i, eh, wh);
    int sc_el = -1, sc_wel = -3;   // the scan of the final position

    double U1, V1;
    bool ok1 = Form::uv2(m, f, s, lon0, lat0, node_i, eh, s.ak[0], U1, V1);
    st.U[i] = U1;
    st.V[i] = V1;
    if (!ok1) {
        status = OUTSIDE; fr = FR_INTERP; nn_out = node_i; failed = true;
    } else if (SCHEME == 0) {
        lon_new = wrap180(lon0 + dt * U1 / metric_z0f<Form::kExact>(q0));
        lat_new = clamp_lat(lat0 + dt * V1 / SLM);
    } else if (SCHEME == 1) {
        double lon_mid = wrap180(lon0 + 0.5 * dt * U1 / metric_z0f<Form::kExact>(q0));
        double lat_mid = clamp_lat(lat0 + 0.5 * dt * V1 / SLM);
        const Site qm = Form::site(lon_mid, lat_mid);
        int nn_mid = site_anchor(m, qm);
        e_last = stage_elem<WALK>(m, lon_mid, lat_mid, e1, nn_mid);
        double U2, V2;
        if (!Form::uv2(m, f, s, lon_mid, lat_mid, nn_mid, e_last, s.ak[1], U2, V2)) {
            status = OUTSIDE; fr = FR_INTERP; nn_out = node_i; failed = true;
        } else {
            lon_new = wrap180(lon0 + dt * U2 / metric_z0f<Form::kExact>(qm));
            lat_new = clamp_lat(lat0 + dt * V2 / SLM);
        }
    } else {
        double dlon1 = dt * U1 / metric_z0f<Form::kExact>(q0);
        double dlat1 = dt * V1 / SLM;
        double lon2 = wrap180(lon0 + 0.5 * dlon1);
        double lat2 = clamp_lat(lat0 + 0.5 * dlat1);
        const Site q2 = Form::site(lon2, lat2);
        const int n2 = site_anchor(m, q2);
        const int e2 = stage_elem<WALK>(m, lon2, lat2, e1, n2);
        double U2, V2;
        if (!Form::uv2(m, f, s, lon2, lat2, n2, e2, s.ak[1], U2, V2)) {
            status = OUTSIDE; fr = FR_INTERP; nn_out = node_i; failed = true;
        } else {
            double dlon2 = dt * U2 / metric_z0f<Form::kExact>(q2);
            double dlat2 = dt * V2 / SLM;
            double lon3 = wrap180(lon0 + 0.5 * dlon2);
            double lat3 = clamp_lat(lat0 + 0.5 * dlat2);
            const Site q3 = Form::site(lon3, lat3);
            const int n3 = site_anchor(m, q3);
            const int e3 = stage_elem<WALK>(m, lon3, lat3, e2, n3);
            double U3, V3;
            if (!Form::uv2(m, f, s, lon3, lat3, n3, e3, s.ak[2], U3, V3)) {
                status = OUTSIDE; fr = FR_INTERP; nn_out = node_i; failed = true;
            } else {
                double dlon3 = dt * U3 / metric_z0f<Form::kExact>(q3);
                double dlat3 = dt * V3 / SLM;
                double lon4 = wrap180(lon0 + dlon3);
                double lat4 = clamp_lat(lat0 + dlat3);
                const Site q4 = Form::site(lon4, lat4);
                const int n4 = site_anchor(m, q4);
                e_last = stage_elem<WALK>(m, lon4, lat4, e3, n4);
                double U4, V4;
                if (!Form::uv2(m, f, s, lon4, lat4, n4, e_last, s.ak[3], U4, V4)) {
                    status = OUTSIDE; fr = FR_INTERP; nn_out = node_i; failed = true;
                } else {
                    double dlon4 = dt * U4 / metric_z0f<Form::kExact>(q4);
                    double dlat4 = dt * V4 / SLM;
                    double dlon = (dlon1 + 2.0 * dlon2 + 2.0 * dlon3 + dlon4) / 6.0;
                    double dlat = (dlat1 + 2.0 * dlat2 + 2.0 * dlat3 + dlat4) / 6.0;
                    lon_new = wrap180(lon0 + dlon);
                    lat_new = clamp_lat(lat0 + dlat);
                }
            }
        }
    }
    if (!failed) {
        const Site qn = Form::site(lon_new, lat_new);
        int nn_new = site_anchor(m, qn);
        int ein;
        if constexpr (WALK) ein = walk_locate(m, lon_new, lat_new, e_last, nn_new);
        else ein = end_scan(m, false, lon_new, lat_new, nn_new, sc_wel);
        sc_el = ein;
        if (ein < 0) {
            status = OUTSIDE; fr = FR_OOB; nn_out = node_i;
            lon_new = lon0; lat_new = lat0;
        } else {
            status = ALIVE;
            nn_out = nn_new;
            e_out = ein;
            if (s.kick) {
                double zz = 0.0;
                long long pid = st.pid ? st.pid[i] : i;
                apply_kick<Form::kExact>(m, s, pid, realization_of(st, s, i), qn, lon0, lat0, 0.0, pre_nn, false, lon_new, lat_new,
                           zz, status, nn_out, fr, false, sc_el, sc_wel);
            }
        }
    } else {
        lon_new = lon0;
        lat_new = lat0;
    }
    st.lon[i] = lon_new;
    st.lat[i] = lat_new;
    st.status[i] = status;
    st.nn[i] = nn_out;
    st.fr[i] = fr;
    if constexpr (WALK) st.elem[i] = e_out;
    mark_anchor(st, i, status, nn_out, node_i);
    if constexpr (!WALK) mark_scan(st, i, status, sc_el, sc_wel);
}

// u/v of one 3-D stage: the layer rule (the particle's layer at the anchor,
// integrators.py:3668-3676) or the depth-linear rule at the stage depth
// (:4071-4098).
template <typename T>
__device__ __forceinline__ bool stage_uv(const DMesh& m, const DBlend<T>& f, const DStep& s, double lon,
                                         double lat, int nn, int hint, double z, double alpha, double& U,
                                         double& V) {
    if (s.uv_dl) return interp_uv_bary_dl<T>(m, f, lon, lat, nn, hint, z, s.time_dir, alpha, U, V);
    const int layer = find_layer(m, z, nn);
    return interp_uv_bary<T>(m, f, lon, lat, nn, hint, s.time_dir, layer, alpha, U, V);
}

// The plain form: the reference's float64 interpolation, bit for bit.
// uvw3 evaluates W even where u/v failed (the caller then discards it).
// hint >= 0 is the stage's containing element from the edge walk, which
// replaces the u/v element search; the barycentric W keeps its own search.
// Element-layout u/v by element-centre least squares (the 2-D fused
// kernels of integrators.py:1490-2520 and their PCHIP twins :2820-3100):
// the stage reads the anchor's element ring, no containment; plain float64
// arithmetic, 2-D only.
// The form an unfused 3-D step (four stages) runs with: the form itself,
// unless a form says otherwise (MixedForm: its stage behind a call).
template <typename Form>
struct UnfusedFormOf {
    using type = Form;
};

// 3-D (interpolate.py:644-750 interp_leastsq with the per-particle layer of
// _compute_layers): the same fit on the layer's row of element values, W of
// the nodes by the step's W method.  A 3-D field's u/v (K-1, E) and w (K, N)
// rows share one stride, max(E, N).
template <typename T>
struct LsqForm {
    static constexpr bool kExact = true;
    static __device__ __forceinline__ Site site(double lon, double lat) { return make_site_fast(lon, lat); }
    static __device__ __forceinline__ bool uv2(const DMesh& m, const DBlend<T>& f, const DStep& s, double lon,
                                               double lat, int nn, int hint, double alpha, double& U, double& V) {
        return interp_uv_lsq<T>(m, f, lon, lat, nn, s.time_dir, alpha, U, V);
    }
    static __device__ __forceinline__ bool uvw3(const DMesh& m, const DBlend<T>& f, const DStep& s, double lon,
                                                double lat, int nn, int hint, int whint, double z, double alpha,
                                                double& U, double& V, double& W) {
        const bool ok = interp_uv_lsq<T>(m, f, lon, lat, nn, s.time_dir, alpha, U, V, find_layer(m, z, nn));
        if (s.w_code == 0) W = w_linear<T>(m, f, alpha, z, nn, s.time_dir);
        else if (s.w_code == 1) W = w_bary<T>(m, f, alpha, lon, lat, z, nn, s.time_dir);
        else W = w_ring<T>(m, f, s.w_code, alpha, lon, lat, z, nn, s.time_dir);
        return ok;
    }
};

// Element-centre u/v by the edge-neighbour least squares
// (interpolate.py:2588-2747 _interp_edge_leastsq_core, uv_interp
// "edge_leastsq"): 2-D and 3-D layer fields, node W by the step's W method.
template <typename T>
struct EdgeLsqForm {
    static constexpr bool kExact = true;
    static __device__ __forceinline__ Site site(double lon, double lat) { return make_site_fast(lon, lat); }
    static __device__ __forceinline__ bool uv2(const DMesh& m, const DBlend<T>& f, const DStep& s, double lon,
                                               double lat, int nn, int hint, double alpha, double& U, double& V) {
        return interp_uv_edge_lsq<T>(m, f, lon, lat, nn, s.edge_bc, s.time_dir, alpha, 0, U, V);
    }
    static __device__ __forceinline__ bool uvw3(const DMesh& m, const DBlend<T>& f, const DStep& s, double lon,
                                                double lat, int nn, int hint, int whint, double z, double alpha,
                                                double& U, double& V, double& W) {
        const bool ok = interp_uv_edge_lsq<T>(m, f, lon, lat, nn, s.edge_bc, s.time_dir, alpha, find_layer(m, z, nn),
                                              U, V);
        if (s.w_code == 0) W = w_linear<T>(m, f, alpha, z, nn, s.time_dir);
        else if (s.w_code == 1) W = w_bary<T>(m, f, alpha, lon, lat, z, nn, s.time_dir);
        else W = w_ring<T>(m, f, s.w_code, alpha, lon, lat, z, nn, s.time_dir);
        return ok;
    }
};

template <typename T>
// kExact: the displacement metric, the kick's move and the draws take the
// correctly rounded trigonometry (the reference's values but where the C
// library misrounds) and the table-corrected draws; sites carry CUDA's
// sincos, as they only feed the anchor search.
struct PlainForm {
    static constexpr bool kExact = true;
    static __device__ __forceinline__ Site site(double lon, double lat) { return make_site_fast(lon, lat); }
    static __device__ __forceinline__ bool uv2(const DMesh& m, const DBlend<T>& f, const DStep& s, double lon,
                                               double lat, int nn, int hint, double alpha, double& U, double& V) {
        return interp_uv_bary<T>(m, f, lon, lat, nn, hint, s.time_dir, 0, alpha, U, V);
    }
    static __device__ __forceinline__ bool uvw3(const DMesh& m, const DBlend<T>& f, const DStep& s, double lon,
                                                double lat, int nn, int hint, int whint, double z, double alpha,
                                                double& U, double& V, double& W) {
        if (s.w_code != 1) {   // W nearest (0), least squares (2), inverse distance (3)
            const bool ok = stage_uv<T>(m, f, s, lon, lat, nn, hint, z, alpha, U, V);
            W = s.w_code == 0 ? w_linear<T>(m, f, alpha, z, nn, s.time_dir)
                              : w_ring<T>(m, f, s.w_code, alpha, lon, lat, z, nn, s.time_dir);
            return ok;
        }
        // W barycentric: one containment scan decides the u/v element and,
        // almost always, the element the W search would stop at (a carried
        // scan, whint >= -2, gives both; a walk element, whint -3, leaves the
        // W search to run)
        int w_elem = -1;
        bool w_unsure = true;
        int elem = hint;
        if (hint >= 0) {
            if (whint >= -2) {
                w_elem = whint >= 0 ? whint : -1;
                w_unsure = whint == -2;
            }
        } else {
            elem = contain_local_w(m, lon, lat, nn, w_elem, w_unsure);
        }
        bool ok = false;
        U = 0.0;
        V = 0.0;
        if (elem >= 0) {
            ok = s.uv_dl ? interp_uv_dl_at<T>(m, f, elem, lon, lat, z, s.time_dir, alpha, U, V)
                         : interp_uv_at<T>(m, f, elem, lon, lat, s.time_dir, find_layer(m, z, nn), alpha, U, V);
        }
        if (w_unsure) W = w_bary<T>(m, f, alpha, lon, lat, z, nn, s.time_dir);
        else if (w_elem >= 0) W = w_bary_at<T>(m, f, alpha, lon, lat, z, w_elem, s.time_dir);
        else W = w_vertex<T>(m, f, alpha, z, w_locate(m, z), nn, s.time_dir);
        return ok;
    }
};

// One 3-D stage of the unfused paths: exact anchor at the stage position,
// u/v at the stage depth, W from the stage blend.
template <typename T, typename Form, bool WALK>
__device__ __forceinline__ bool stage3d(const DMesh& m, const DBlend<T>& f, const DStep& s, int k, double lon,
                                        double lat, double z, const Site& q, int from, int& e, double& U,
                                        double& V, double& W) {
    const int nn = site_anchor(m, q);
    e = stage_elem<WALK>(m, lon, lat, from, nn);
    return Form::uvw3(m, f, s, lon, lat, nn, e, -3, z, s.ak[k], U, V, W);
}

// 3-D Euler (integrators.py:4997-5147) and RK4 (:5760-6011): the reference's
// unfused multi-pass paths restated per particle -- the batch exact anchor of
// every stage position, the layer at the stage depth, the whole-field stage
// lerps of _make_stage_vels (:1187-1237) reproduced per vertex, W at the stage
// position; a failure reverts to the start with the start anchor.
template <typename T, int SCHEME, typename Form, bool WALK = false>
__device__ __forceinline__ void step3d_unfused_particle(const DMesh& m, const DBlend<T>& f, const DState& st,
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
    const double dt = s.dt, td = s.time_dir;
    signed char fr = st.fr[i];
    double lon_new = lon0, lat_new = lat0, z_new = z0p;

    const Site q0 = Form::site(lon0, lat0);
    const int node_i = start_anchor(m, st, q0, pre_nn, i);
    int nn_out = node_i;
    const int e1 = stage_elem<WALK>(m, lon0, lat0, WALK ? st.elem[i] : -1, node_i);
    int e_last = e1, e_out = e1;
    int eh = e1, wh = -3;
    if constexpr (!WALK) carried_scan(st, i, eh, wh);
    int sc_el = -1, sc_wel = -3;
    double U1, V1, W1;
    bool ok = Form::uvw3(m, f, s, lon0, lat0, node_i, eh, wh, z0p, s.ak[0], U1, V1, W1);
    st.U[i] = U1;
    st.V[i] = V1;
    st.W[i] = W1;
    double a = lon0, b = lat0, c = z0p;
    if (ok) {
        if (SCHEME == 0) {
            a = wrap180(lon0 + dt * U1 / metric_z0f<Form::kExact>(q0));
            b = clamp_lat(lat0 + dt * V1 / SLM);
            c = z0p + W1 * dt;
        } else {
            const double dl1 = dt * U1 / metric_z0f<Form::kExact>(q0), dd1 = dt * V1 / SLM, dz1 = dt * W1;
            const double l2 = wrap180(lon0 + 0.5 * dl1), t2 = clamp_lat(lat0 + 0.5 * dd1), z2 = z0p + 0.5 * dz1;
            const Site q2 = Form::site(l2, t2);
            double U2, V2, W2;
            int e2, e3;
            ok = stage3d<T, Form, WALK>(m, f, s, 1, l2, t2, z2, q2, e1, e2, U2, V2, W2);
            if (ok) {
                const double dl2 = dt * U2 / metric_z0f<Form::kExact>(q2), dd2 = dt * V2 / SLM, dz2 = dt * W2;
                const double l3 = wrap180(lon0 + 0.5 * dl2), t3 = clamp_lat(lat0 + 0.5 * dd2), z3 = z0p + 0.5 * dz2;
                const Site q3 = Form::site(l3, t3);
                double U3, V3, W3;
                ok = stage3d<T, Form, WALK>(m, f, s, 2, l3, t3, z3, q3, e2, e3, U3, V3, W3);
                if (ok) {
                    const double dl3 = dt * U3 / metric_z0f<Form::kExact>(q3), dd3 = dt * V3 / SLM, dz3 = dt * W3;
                    const double l4 = wrap180(lon0 + dl3), t4 = clamp_lat(lat0 + dd3), z4 = z0p + dz3;
                    const Site q4 = Form::site(l4, t4);
                    double U4, V4, W4;
                    ok = stage3d<T, Form, WALK>(m, f, s, 3, l4, t4, z4, q4, e3, e_last, U4, V4, W4);
                    if (ok) {
                        const double dl4 = dt * U4 / metric_z0f<Form::kExact>(q4), dd4 = dt * V4 / SLM, dz4 = dt * W4;
                        const double dl = (dl1 + 2.0 * dl2 + 2.0 * dl3 + dl4) / 6.0;
                        const double dd = (dd1 + 2.0 * dd2 + 2.0 * dd3 + dd4) / 6.0;
                        const double dz = (dz1 + 2.0 * dz2 + 2.0 * dz3 + dz4) / 6.0;
                        a = wrap180(lon0 + dl);
                        b = clamp_lat(lat0 + dd);
                        c = z0p + dz;
                    }
                }
            }
        }
    }
    if (!ok) {
        status = OUTSIDE; fr = FR_INTERP;
    } else {
        const Site qn = Form::site(a, b);
        const int nn_new = site_anchor(m, qn);
        int ein;
        if constexpr (WALK) ein = walk_locate(m, a, b, e_last, nn_new);
        else ein = end_scan(m, s.w_code == 1, a, b, nn_new, sc_wel);
        sc_el = ein;
        if (ein < 0) {
            status = OUTSIDE; fr = FR_OOB;
        } else {
            if (c < m.zlev[0]) c = m.zlev[0];
            const double bottom = m.depth[nn_new];
            if (c > bottom) c = bottom;
            lon_new = a; lat_new = b; z_new = c;
            status = ALIVE;
            nn_out = nn_new;
            e_out = ein;
            if (s.kick) {
                long long pid = st.pid ? st.pid[i] : i;
                apply_kick<Form::kExact>(m, s, pid, realization_of(st, s, i), qn, lon0, lat0, z0p, pre_nn, true, lon_new, lat_new, z_new,
                           status, nn_out, fr, s.w_code == 1, sc_el, sc_wel);
            }
            if (s.az_on && status == ALIVE)
                apply_az<T, Form::kExact>(m, f, s, st.pid ? st.pid[i] : i, realization_of(st, s, i), nn_out, z_new);
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
    if constexpr (!WALK) mark_scan(st, i, status, sc_el, sc_wel);
}

// integrators.py:3647-3856 _fused_rk2_step_3d_bary_tinterp (layer u/v,
// z-level), with the exact stage-1 anchor of its runner (:4766-4770) and the
// split kick epilogue.
template <typename T, typename Form, bool WALK = false>
__device__ __forceinline__ void step3d_rk2_particle(const DMesh& m, const DBlend<T>& f, const DState& st,
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
    const double dt = s.dt, td = s.time_dir;
    signed char fr = st.fr[i];
    double lon_new = lon0, lat_new = lat0, z_new = z0p;

    const Site q0 = Form::site(lon0, lat0);
    const int node_i = start_anchor(m, st, q0, pre_nn, i);
    int nn_out = node_i;
    const int e1 = stage_elem<WALK>(m, lon0, lat0, WALK ? st.elem[i] : -1, node_i);
    int e_out = e1;
    int eh = e1, wh = -3;
    if constexpr (!WALK) carried_scan(st, i, eh, wh);
    int sc_el = -1, sc_wel = -3;
    double U1, V1, W1;
    const bool ok1 = Form::uvw3(m, f, s, lon0, lat0, node_i, eh, wh, z0p, s.ak[0], U1, V1, W1);
    st.U[i] = U1;
    st.V[i] = V1;
    st.W[i] = W1;
    if (!ok1) {
        status = OUTSIDE; fr = FR_INTERP;
    } else {
        const double lon_mid = wrap180(lon0 + 0.5 * dt * U1 / metric_z0f<Form::kExact>(q0));
        const double lat_mid = clamp_lat(lat0 + 0.5 * dt * V1 / SLM);
        const double z_mid = z0p + W1 * 0.5 * dt;
        const Site qm = Form::site(lon_mid, lat_mid);
        const int nn_mid = site_anchor(m, qm);
        const int em = stage_elem<WALK>(m, lon_mid, lat_mid, e1, nn_mid);
        double U2, V2, W2;
        if (!Form::uvw3(m, f, s, lon_mid, lat_mid, nn_mid, em, -3, z_mid, s.ak[1], U2, V2, W2)) {
            status = OUTSIDE; fr = FR_INTERP;
        } else {
            const double ln = wrap180(lon0 + dt * U2 / metric_z0f<Form::kExact>(qm));
            const double lt = clamp_lat(lat0 + dt * V2 / SLM);
            double zn = z0p + W2 * dt;
            const Site qn = Form::site(ln, lt);
            const int nn_new = site_anchor(m, qn);
            int ein;
            if constexpr (WALK) ein = walk_locate(m, ln, lt, em, nn_new);
            else ein = end_scan(m, s.w_code == 1, ln, lt, nn_new, sc_wel);
            sc_el = ein;
            if (ein < 0) {
                status = OUTSIDE; fr = FR_OOB;
            } else {
                if (zn < m.zlev[0]) zn = m.zlev[0];
                const double bottom = m.depth[nn_new];
                if (zn > bottom) zn = bottom;
                lon_new = ln; lat_new = lt; z_new = zn;
                status = ALIVE;
                nn_out = nn_new;
                e_out = ein;
                if (s.kick) {
                    long long pid = st.pid ? st.pid[i] : i;
                    apply_kick<Form::kExact>(m, s, pid, realization_of(st, s, i), qn, lon0, lat0, z0p, pre_nn, true, lon_new, lat_new,
                               z_new, status, nn_out, fr, s.w_code == 1, sc_el, sc_wel);
                }
                if (s.az_on && status == ALIVE)
                    apply_az<T, Form::kExact>(m, f, s, st.pid ? st.pid[i] : i, realization_of(st, s, i), nn_out, z_new);
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
    if constexpr (!WALK) mark_scan(st, i, status, sc_el, sc_wel);
}

}  // namespace kc
