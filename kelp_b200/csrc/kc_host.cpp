// Host routines of the C ABI that run on the CPU at set-up time.
//
// kc_node_xyz_fill restates KELP's _node_xyz_fill (src/kelp/core/mesh.py:712-737):
// the unit-sphere coordinates of every node, computed with the C library's
// cos/sin -- the functions Numba's lowering of np.cos / np.sin calls -- so the
// table is bit-identical to the reference's and nearest-node ties resolve the
// same way.  Compiled with -ffp-contract=off (no fused multiply-add).
#include <cmath>
#include "../../include/kelp_cuda.h"

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
