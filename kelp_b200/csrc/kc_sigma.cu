// The sigma-mesh 3-D steps (plain form) on float64 and float32 snapshots.
#include "kc_launch.h"

void kc_launch_sigma_f64(const kc::DMesh& m, const kc::DBlend<double>& f, const kc::DState& st, const kc::DStep& s,
                         int scheme, cudaStream_t stream) {
    launch_sigma_kernel<double>(m, f, st, s, scheme, stream);
}

void kc_launch_sigma_f32(const kc::DMesh& m, const kc::DBlend<float>& f, const kc::DState& st, const kc::DStep& s,
                         int scheme, cudaStream_t stream) {
    launch_sigma_kernel<float>(m, f, st, s, scheme, stream);
}
