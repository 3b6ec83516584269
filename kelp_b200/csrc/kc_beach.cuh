// Beaching and resuspension of one particle after its step: the on_failure
// remap, the depth / coastal-element / stochastic criteria and the automatic /
// stochastic resuspension of KELP's tracking._apply_beaching_hook
// (src/kelp/tracking.py:199-364) and numerics.beaching.evaluate_beaching
// (src/kelp/numerics/beaching.py:95-181), one thread per particle.
#pragma once
#include "kc_step.cuh"

namespace kc {

constexpr int RESUSP_NEVER = 0, RESUSP_AUTO = 1, RESUSP_STOCH = 2, RESUSP_BOTH = 3;
constexpr unsigned long long COMP_BEACH = 10, COMP_RESUSP = 11;

struct DBeach {
    int use_depth, use_coastal, use_stochastic, on_failure, need_topo, resuspension, min_wet_steps;
    double depth_min, zone_depth, rewet_level;   // rewet_level = depth_min + rewet_hysteresis
    double p_beach, p_resusp;                    // 1 - exp(-|dt| / t), evaluated by the host
    unsigned long long seed, real_id, step_i, pid_offset;
    const unsigned char* coastal;                // (E) coastal element flags, null without topology
    const double* eta;                           // (N) the payload's free surface (use_eta), or null
    const double* dry;                           // (N) the payload's dry mask (dry_mask_var), or null
    const int* prev;                             // (P) status at the step's entry
    int* wet_streak;                             // (P) consecutive wet steps of a beached particle
};

// beaching.py:46-56 _u01: the top 53 bits of the counter hash.
__device__ __forceinline__ double u01(unsigned long long seed, unsigned long long real_id, unsigned long long pid,
                                      unsigned long long step, unsigned long long comp) {
    uint64_t h = key_hash(seed, real_id, pid, step, comp);
    return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

__device__ __forceinline__ void beach_particle(const DMesh& m, const DState& st, const DBeach& b, long long N,
                                               long long i) {
    int status = st.status[i];
    const int prev = b.prev[i];
    int nn = st.nn[i];
    if (nn >= N || nn < -N) {   // the reference's indexing would raise; flag it and leave the particle
        atomicOr(m.err, ERR_BAD_ANCHOR);
        return;
    }
    signed char fr = st.fr[i];
    const bool newly = status == OUTSIDE && prev == ALIVE;
    // tracking.py:253-261: a particle that failed on its first step may still
    // carry the unknown anchor -1; its reverted position's anchor replaces it
    if (newly && nn < 0) {
        nn = site_anchor(m, make_site(st.lon[i], st.lat[i]));
        st.nn[i] = nn;
        if (st.nn_ok) st.nn_ok[i] = 1;
    }
    const bool alive0 = status == ALIVE, beached0 = status == BEACHED;
    int contained = -1;
    if (b.need_topo && (alive0 || beached0 || newly)) {
        // a -1 anchor indexes the last node, as the reference's wraparound does
        const int a = nn < 0 ? (int)(nn + N) : nn;
        contained = contain_local(m, st.lon[i], st.lat[i], a);
    }
    // the unclamped column height, with the free surface when use_eta
    // (beaching.py:112-117, tracking.py:290-297); a node the dry mask marks
    // (> 0.5) is dry for the depth criterion and never wet (:124-129, :151-159)
    double h_raw = INFINITY;
    if (nn >= 0) {
        h_raw = m.depth[nn];
        if (b.eta) h_raw = h_raw + b.eta[nn];
    }
    const bool masked = b.dry && nn >= 0 && b.dry[nn] > 0.5;
    const bool coastal_contact = contained >= 0 && b.coastal && b.coastal[contained];
    const long long pid = st.pid ? st.pid[i] : i;
    const unsigned long long key = (unsigned long long)pid + b.pid_offset;
    const unsigned long long rid = st.rid ? (unsigned long long)st.rid[i] : b.real_id;
    // 1. on_failure context-gated remap (tracking.py:279-307)
    if (b.on_failure && newly) {
        bool context = h_raw < b.zone_depth;
        if (b.need_topo && b.coastal) context = context || coastal_contact;
        if (context) {
            status = BEACHED;
            fr = 0;
        }
    }
    // 2. criteria (beaching.py:118-140)
    const bool alive = status == ALIVE, beached = status == BEACHED;
    bool to_beach = false;
    if (b.use_depth) to_beach = to_beach || (h_raw < b.depth_min) || masked;
    if (b.use_coastal) to_beach = to_beach || coastal_contact;
    if (b.use_stochastic && alive) {
        bool in_zone = h_raw < b.zone_depth;
        if (b.need_topo && b.coastal) in_zone = in_zone || coastal_contact;
        if (in_zone && u01(b.seed, rid, key, b.step_i, COMP_BEACH) < b.p_beach) to_beach = true;
    }
    to_beach = to_beach && alive;
    // resuspension (beaching.py:142-178)
    int ws = b.wet_streak[i];
    bool to_release = false;
    if (b.resuspension != RESUSP_NEVER && beached) {
        const bool rewet = h_raw > b.rewet_level && nn >= 0 && !masked;
        ws = rewet ? ws + 1 : 0;
        if (b.resuspension == RESUSP_AUTO || b.resuspension == RESUSP_BOTH)
            to_release = to_release || ws >= b.min_wet_steps;
        if ((b.resuspension == RESUSP_STOCH || b.resuspension == RESUSP_BOTH) && rewet &&
            u01(b.seed, rid, key, b.step_i, COMP_RESUSP) < b.p_resusp)
            to_release = true;
    }
    if (to_release) ws = 0;
    if (!beached) ws = 0;
    if (to_beach) status = BEACHED;
    if (to_release) {
        status = ALIVE;
        fr = 0;
    }
    st.status[i] = status;
    st.fr[i] = fr;
    b.wet_streak[i] = ws;
}

}  // namespace kc
