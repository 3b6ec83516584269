// The mixed-precision step kernels (float32 interpolation on float32 or
// scaled float16 snapshots, float64 positions and element decisions), in
// their own translation unit so they compile beside the plain form's.
#include <cuda_runtime.h>
#include <cuda_fp16.h>

#include "kc_mixed.cuh"
#include "kc_kernels.cuh"

void kc_launch_mixed_f32(const kc::DMesh& m, const kc::DBlend<float>& f, const kc::DState& st, const kc::DStep& s,
                         int dims, int scheme, cudaStream_t stream) {
    launch_step_kernel<float, kc::MixedForm<float>>(m, f, st, s, dims, scheme, stream);
}

void kc_launch_mixed_f16(const kc::DMesh& m, const kc::DBlend<__half>& f, const kc::DState& st,
                         const kc::DStep& s, int dims, int scheme, cudaStream_t stream) {
    launch_step_kernel<__half, kc::MixedForm<__half>>(m, f, st, s, dims, scheme, stream);
}

void kc_launch_multi_mixed_f32(const kc::DMesh& m, const MultiHead* head, const StepPack<float>* packs, long long P,
                               int dims, int scheme, int block, cudaStream_t stream) {
    launch_multi_kernel<float, kc::MixedForm<float>>(m, head, packs, P, dims, scheme, block, stream);
}

void kc_launch_multi_mixed_f16(const kc::DMesh& m, const MultiHead* head, const StepPack<__half>* packs, long long P,
                               int dims, int scheme, int block, cudaStream_t stream) {
    launch_multi_kernel<__half, kc::MixedForm<__half>>(m, head, packs, P, dims, scheme, block, stream);
}
