// Internal host routines of the native library (not part of the C ABI).
#pragma once

namespace kc_host {

void mesh_tables(long long N, long long E, int max_v, const double* lat, const int* en, const double* depth,
                 const double* zl, int K, double* node_sc, double* elem_cos, int* max_layer);

// Plane lengths S, E, N, W of the F-point quads of a C-grid mesh, each edge at
// the cosine of its own mean latitude (numerics/nemo_cgrid.py:193-200, with
// the C library's cos and hypot): out is (E, 4).
void cgrid_edge_lengths(long long E, const int* corners, const double* lon, const double* lat, double* out);

}  // namespace kc_host
