// Per-particle step bodies of the KELP time-stepping path: the fused 2-D
// barycentric Euler/RK2/RK4 steps with inline temporal blending, the fused
// 3-D RK2 step (z-level layers, W nearest/barycentric, surface/bottom clamp),
// and the split uniform-Kh random-walk kick applied to the particles that
// survived the deterministic step.  One thread owns one particle for the whole
// step, so every intermediate stays in registers.
#pragma once
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
    const int* release_step;   // delayed release (null: all released)
    long long P;
};

struct DStep {
    double dt, time_dir;
    double ak[4];              // stage alphas c_k * dt / dt_to_next
    int w_code;                // 0 nearest, 1 barycentric (3-D)
    int kick;                  // split uniform-Kh kick on/off
    double kh_x, kh_y;
    unsigned long long seed, real_id, step_i, pid_offset;
    long long global_step;     // for delayed release activation (-1: none)
};

// displacement metric z0 = max(cos(lat) * 111120, 1) (integrators.py:2563-2565)
__device__ __forceinline__ double metric_z0(double lat) {
    double z0 = cos(lat * DEG2RAD) * SLM;
    if (z0 < 1.0) z0 = 1.0;
    return z0;
}

__device__ __forceinline__ double clamp_lat(double lat) {
    if (lat > 90.0) return 90.0;
    if (lat < -90.0) return -90.0;
    return lat;
}

// integrators.py:673-818 _apply_split_diffusion_kick for one particle that is
// ALIVE after the deterministic step: counter-RNG kick (diffusion.py:485-529,
// :261-298), great-circle move, exact re-anchor and containment re-check,
// revert to the pre-step state on leaving the domain; 3-D reclamp in the new
// column.  Returns the new status.
template <bool IS3D>
__device__ __forceinline__ void apply_kick(const DMesh& m, const DStep& s, long long i, long long pid,
                                           double pre_lon, double pre_lat, double pre_z, int pre_nn,
                                           double& lon, double& lat, double& z, int& status, int& nn,
                                           signed char& fr) {
    double g1, g2;
    normal_pair(s.seed, s.real_id, (unsigned long long)pid + s.pid_offset, s.step_i, 0ull, g1, g2);
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
    sphere_displace(lon, lat, dx, dy, lk, lak);
    int nk = site_anchor(m, lk, lak);
    bool in_dom = contain_local(m, lk, lak, nk) >= 0;
    if (!in_dom) {
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
    if (IS3D) {
        double zv = z;
        if (zv < m.zlev[0]) zv = m.zlev[0];
        double bottom = m.depth[nk];
        if (zv > bottom) zv = bottom;
        z = zv;
    }
}

// integrators.py:2521-2638 (RK2), :2641-2816 (RK4); Euler follows the
// per-particle arithmetic of the unfused path (integrators.py:4997-5147):
// one stage at the start, move, re-anchor, domain check.
template <typename T, int SCHEME>
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
    signed char fr = st.fr ? st.fr[i] : 0;
    bool failed = false;
    int node_i = site_anchor(m, lon0, lat0);

    double U1, V1;
    bool ok1 = interp_uv_bary<T>(m, f, lon0, lat0, node_i, td, 0, s.ak[0], U1, V1);
    st.U[i] = U1;
    st.V[i] = V1;
    if (!ok1) {
        status = OUTSIDE; fr = FR_INTERP; nn_out = node_i; failed = true;
    } else if (SCHEME == 0) {
        double z0 = metric_z0(lat0);
        double ln = lon0 + dt * U1 / z0;
        double lt = lat0 + dt * V1 / SLM;
        ln = wrap180(ln);
        lt = clamp_lat(lt);
        lon_new = ln;
        lat_new = lt;
    } else if (SCHEME == 1) {
        double z0 = metric_z0(lat0);
        double lon_mid = lon0 + 0.5 * dt * U1 / z0;
        double lat_mid = lat0 + 0.5 * dt * V1 / SLM;
        lon_mid = wrap180(lon_mid);
        lat_mid = clamp_lat(lat_mid);
        int nn_mid = site_anchor(m, lon_mid, lat_mid);
        double U2, V2;
        bool ok2 = interp_uv_bary<T>(m, f, lon_mid, lat_mid, nn_mid, td, 0, s.ak[1], U2, V2);
        if (!ok2) {
            status = OUTSIDE; fr = FR_INTERP; nn_out = node_i; failed = true;
        } else {
            double z0m = metric_z0(lat_mid);
            double ln = lon0 + dt * U2 / z0m;
            double lt = lat0 + dt * V2 / SLM;
            lon_new = wrap180(ln);
            lat_new = clamp_lat(lt);
        }
    } else {
        double z0_1 = metric_z0(lat0);
        double dlon1 = dt * U1 / z0_1;
        double dlat1 = dt * V1 / SLM;
        double lon2 = wrap180(lon0 + 0.5 * dlon1);
        double lat2 = clamp_lat(lat0 + 0.5 * dlat1);
        int nn2 = site_anchor(m, lon2, lat2);
        double U2, V2;
        if (!interp_uv_bary<T>(m, f, lon2, lat2, nn2, td, 0, s.ak[1], U2, V2)) {
            status = OUTSIDE; fr = FR_INTERP; nn_out = node_i; failed = true;
        } else {
            double z0_2 = metric_z0(lat2);
            double dlon2 = dt * U2 / z0_2;
            double dlat2 = dt * V2 / SLM;
            double lon3 = wrap180(lon0 + 0.5 * dlon2);
            double lat3 = clamp_lat(lat0 + 0.5 * dlat2);
            int nn3 = site_anchor(m, lon3, lat3);
            double U3, V3;
            if (!interp_uv_bary<T>(m, f, lon3, lat3, nn3, td, 0, s.ak[2], U3, V3)) {
                status = OUTSIDE; fr = FR_INTERP; nn_out = node_i; failed = true;
            } else {
                double z0_3 = metric_z0(lat3);
                double dlon3 = dt * U3 / z0_3;
                double dlat3 = dt * V3 / SLM;
                double lon4 = wrap180(lon0 + dlon3);
                double lat4 = clamp_lat(lat0 + dlat3);
                int nn4 = site_anchor(m, lon4, lat4);
                double U4, V4;
                if (!interp_uv_bary<T>(m, f, lon4, lat4, nn4, td, 0, s.ak[3], U4, V4)) {
                    status = OUTSIDE; fr = FR_INTERP; nn_out = node_i; failed = true;
                } else {
                    double z0_4 = metric_z0(lat4);
                    double dlon4 = dt * U4 / z0_4;
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
        int nn_new = site_anchor(m, lon_new, lat_new);
        if (contain_local(m, lon_new, lat_new, nn_new) < 0) {
            status = OUTSIDE; fr = FR_OOB; nn_out = node_i;
            lon_new = lon0; lat_new = lat0;
        } else {
            status = ALIVE;
            nn_out = nn_new;
        }
    } else {
        lon_new = lon0;
        lat_new = lat0;
    }
    if (s.kick && status == ALIVE) {
        double zz = 0.0;
        long long pid = st.pid ? st.pid[i] : i;
        apply_kick<false>(m, s, i, pid, lon0, lat0, 0.0, pre_nn, lon_new, lat_new, zz, status, nn_out, fr);
    }
    st.lon[i] = lon_new;
    st.lat[i] = lat_new;
    st.status[i] = status;
    st.nn[i] = nn_out;
    if (st.fr) st.fr[i] = fr;
}


template <typename T>
__device__ __forceinline__ double stage_w(const DMesh& m, const DBlend<T>& f, int w_code, double alpha,
                                          double xp, double yp, double z, int node, double td) {
    if (w_code == 0) return w_linear<T>(m, f, alpha, z, node, td);
    return w_bary<T>(m, f, alpha, xp, yp, z, node, td);
}

// integrators.py:3647-3856 _fused_rk2_step_3d_bary_tinterp (layer u/v,
// z-level), with the exact stage-1 anchor of its runner (:4766-4770) and the
// split kick epilogue.
template <typename T>
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
    int nn_out;
    bool failed = true;

    int node_i = site_anchor(m, lon0, lat0);
    nn_out = node_i;
    int layer1 = find_layer(m, z0p, m.depth[node_i]);
    double U1, V1;
    bool ok1 = interp_uv_bary<T>(m, f, lon0, lat0, node_i, td, layer1, s.ak[0], U1, V1);
    double W1 = stage_w<T>(m, f, s.w_code, s.ak[0], lon0, lat0, z0p, node_i, td);
    st.U[i] = U1;
    st.V[i] = V1;
    st.W[i] = W1;
    if (!ok1) {
        status = OUTSIDE; fr = FR_INTERP;
    } else {
        double z0 = metric_z0(lat0);
        double lon_mid = wrap180(lon0 + 0.5 * dt * U1 / z0);
        double lat_mid = clamp_lat(lat0 + 0.5 * dt * V1 / SLM);
        double z_mid = z0p + W1 * 0.5 * dt;
        int nn_mid = site_anchor(m, lon_mid, lat_mid);
        int layer2 = find_layer(m, z_mid, m.depth[nn_mid]);
        double U2, V2;
        if (!interp_uv_bary<T>(m, f, lon_mid, lat_mid, nn_mid, td, layer2, s.ak[1], U2, V2)) {
            status = OUTSIDE; fr = FR_INTERP;
        } else {
            double W2 = stage_w<T>(m, f, s.w_code, s.ak[1], lon_mid, lat_mid, z_mid, nn_mid, td);
            double z0m = metric_z0(lat_mid);
            double ln = wrap180(lon0 + dt * U2 / z0m);
            double lt = clamp_lat(lat0 + dt * V2 / SLM);
            double zn = z0p + W2 * dt;
            int nn_new = site_anchor(m, ln, lt);
            if (contain_local(m, ln, lt, nn_new) < 0) {
                status = OUTSIDE; fr = FR_OOB;
            } else {
                if (zn < m.zlev[0]) zn = m.zlev[0];
                double bottom = m.depth[nn_new];
                if (zn > bottom) zn = bottom;
                lon_new = ln; lat_new = lt; z_new = zn;
                status = ALIVE;
                nn_out = nn_new;
                failed = false;
            }
        }
    }
    (void)failed;
    if (s.kick && status == ALIVE) {
        long long pid = st.pid ? st.pid[i] : i;
        apply_kick<true>(m, s, i, pid, lon0, lat0, z0p, pre_nn, lon_new, lat_new, z_new, status, nn_out, fr);
    }
    st.lon[i] = lon_new;
    st.lat[i] = lat_new;
    st.z[i] = z_new;
    st.status[i] = status;
    st.nn[i] = nn_out;
    st.fr[i] = fr;
}

}  // namespace kc
