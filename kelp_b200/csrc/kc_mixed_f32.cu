// The mixed-precision step kernels on float32 snapshots (float32
// interpolation, float64 positions and element decisions).
#include "kc_mixed.cuh"
#include "kc_launch.h"

void kc_launch_mixed_f32(const kc::DMesh& m, const kc::DBlend<float>& f, const kc::DState& st, const kc::DStep& s,
                         int dims, int scheme, cudaStream_t stream) {
    launch_step_kernel<float, kc::MixedForm<float>>(m, f, st, s, dims, scheme, stream);
}

void kc_launch_multi_mixed_f32(const kc::DMesh& m, const MultiHead* head, const StepPack<float>* packs, long long P,
                               int dims, int scheme, int block, cudaStream_t stream) {
    launch_multi_kernel<float, kc::MixedForm<float>>(m, head, packs, P, dims, scheme, block, stream);
}
