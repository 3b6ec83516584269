// Host routines of the C ABI that run on the CPU at set-up time.
//
// kc_node_xyz_fill restates KELP's _node_xyz_fill (src/kelp/core/mesh.py:712-737):
// the unit-sphere coordinates of every node, computed with the C library's
// cos/sin -- the functions Numba's lowering of np.cos / np.sin calls -- so the
// table is bit-identical to the reference's and nearest-node ties resolve the
// same way.  Compiled with -ffp-contract=off (no fused multiply-add).
#include <cmath>
#include "../../include/kelp_cuda.h"
#include "kc_host.h"

namespace kc_host {

// The mesh-only trigonometric tables of the step kernels, evaluated with the
// C library's sin/cos on the exact expressions the reference evaluates:
//   node_sc[n]  = (sin, cos)(lat_n * DEG2RAD)            mesh.py:1313-1315
//   elem_cos[e] = cos(lat0 * DEG2RAD), lat0 the running mean of the vertex
//                 latitudes in the containment set (x: mesh.py:2216-2236,
//                 :2036-2038) and in the compacted ring (y: interpolate.py
//                 :1368-1396, vertical.py:797-810)
//   max_layer[n] = the deepest layer above the node's bottom (vertical.py:74-81)
void mesh_tables(long long N, long long E, int max_v, const double* lat, const int* en, const double* depth,
                 const double* zl, int K, double* node_sc, double* elem_cos, int* max_layer) {
    const double deg2rad = 0.017453292519943295;
    for (long long n = 0; n < N; ++n) {
        double r = lat[n] * deg2rad;
        node_sc[2 * n] = std::sin(r);
        node_sc[2 * n + 1] = std::cos(r);
    }
    for (long long e = 0; e < E; ++e) {
        const int* v = en + e * max_v;
        // containment (mask) set: -1 slots dropped, slot 3 dropped when it repeats slot 0
        double s = 0.0;
        int n = 0;
        for (int k = 0; k < max_v; ++k) {
            bool keep = v[k] >= 0;
            if (k == 3 && max_v == 4 && v[3] == v[0] && v[0] >= 0) keep = false;
            if (keep) { s += lat[v[k]]; ++n; }
        }
        elem_cos[2 * e] = n > 0 ? std::cos((s / n) * deg2rad) : 1.0;
        // compacted ring: -1 slots and repeats of vertex 0 dropped
        double t = 0.0;
        int m = 0, first = -1;
        for (int k = 0; k < max_v; ++k) {
            int nd = v[k];
            if (nd < 0) continue;
            if (m > 0 && nd == first) continue;
            if (m == 0) first = nd;
            t += lat[nd];
            ++m;
        }
        double lat0 = m > 0 ? t / m : 0.0;
        elem_cos[2 * e + 1] = std::cos(lat0 * deg2rad);
    }
    if (max_layer && depth && zl) {
        for (long long nd = 0; nd < N; ++nd) {
            int ml = K - 2;
            for (int k = 0; k < K - 1; ++k) {
                if (zl[k + 1] > depth[nd]) {
                    ml = k - 1 > 0 ? k - 1 : 0;
                    break;
                }
            }
            max_layer[nd] = ml < 0 ? 0 : ml;
        }
    }
}

void cgrid_edge_lengths(long long E, const int* corners, const double* lon, const double* lat, double* out) {
    const double deg2rad = 0.017453292519943295, M = 111120.0;
    for (long long e = 0; e < E; ++e) {
        for (int k = 0; k < 4; ++k) {
            const int na = corners[4 * e + k], nb = corners[4 * e + (k + 1) % 4];
            // ((dlon + 180) % 360) - 180 with Python's float remainder
            double r = std::fmod(lon[nb] - lon[na] + 180.0, 360.0);
            if (r != 0.0) {
                if (r < 0.0) r += 360.0;
            } else {
                r = 0.0;
            }
            const double dl = r - 180.0;
            const double cm = std::cos(0.5 * (lat[na] + lat[nb]) * deg2rad);
            out[4 * e + k] = std::hypot(dl * cm * M, (lat[nb] - lat[na]) * M);
        }
    }
}

}  // namespace kc_host

extern "C" int kc_node_xyz_fill(const double* lon, const double* lat, long long n, double* out) {
    if (n < 0 || (n > 0 && (!lon || !lat || !out))) return KC_ERR_ARG;
    const double deg2rad = 0.017453292519943295;
    for (long long i = 0; i < n; ++i) {
        double lat_r = lat[i] * deg2rad;
        double lon_r = lon[i] * deg2rad;
        double c = std::cos(lat_r);
        out[3 * i] = c * std::cos(lon_r);
        out[3 * i + 1] = c * std::sin(lon_r);
        out[3 * i + 2] = std::sin(lat_r);
    }
    return KC_OK;
}
