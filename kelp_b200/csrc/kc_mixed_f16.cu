// The mixed-precision step kernels on float16 snapshots with per-row float32
// scales (float32 interpolation, float64 positions and element decisions).
#include "kc_mixed.cuh"
#include "kc_launch.h"

void kc_launch_mixed_f16(const kc::DMesh& m, const kc::DBlend<__half>& f, const kc::DState& st, const kc::DStep& s,
                         int dims, int scheme, cudaStream_t stream) {
    launch_step_kernel<__half, kc::MixedForm<__half>>(m, f, st, s, dims, scheme, stream);
}

void kc_launch_multi_mixed_f16(const kc::DMesh& m, const MultiHead* head, const StepPack<__half>* packs, long long P,
                               int dims, int scheme, int block, cudaStream_t stream) {
    launch_multi_kernel<__half, kc::MixedForm<__half>>(m, head, packs, P, dims, scheme, block, stream);
}
