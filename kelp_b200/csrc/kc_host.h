// Internal host routines of the native library (not part of the C ABI).
#pragma once

namespace kc_host {

void mesh_tables(long long N, long long E, int max_v, const double* lat, const int* en, const double* depth,
                 const double* zl, int K, double* node_sc, double* elem_cos, int* max_layer);

}  // namespace kc_host
