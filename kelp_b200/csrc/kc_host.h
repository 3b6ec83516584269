// Internal host routines of the native library (not part of the C ABI).
#pragma once
#include <cstddef>

namespace kc_host {

void mesh_tables(long long N, long long E, int max_v, const double* lat, const int* en, const double* depth,
                 const double* zl, int K, double* node_sc, double* elem_cos, int* max_layer);

// Plane lengths S, E, N, W of the F-point quads of a C-grid mesh, each edge at
// the cosine of its own mean latitude (numerics/nemo_cgrid.py:193-200, with
// the C library's cos and hypot): out is (E, 4).
void cgrid_edge_lengths(long long E, const int* corners, const double* lon, const double* lat, double* out);

// The Box-Muller exception tables embedded in the library (device layout of
// kc::DRngX; the pointers are into the library's read-only data, read them
// with memcpy): false when the embedded data is malformed.
struct RngTables {
    const unsigned* a_off;
    const unsigned short* a;
    const unsigned* b_off;
    const unsigned short* b;
    size_t n_off, na, nb;
};
bool rng_exception_tables(RngTables& t);

}  // namespace kc_host
