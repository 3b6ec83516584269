// The plain form's step kernels on double snapshots (the reference's float64
// arithmetic), one launch per step and the fused multi-step launch.
#include "kc_launch.h"

void kc_launch_plain_f64(const kc::DMesh& m, const kc::DBlend<double>& f, const kc::DState& st, const kc::DStep& s,
                         int dims, int scheme, cudaStream_t stream) {
    launch_step_kernel<double, kc::PlainForm<double>>(m, f, st, s, dims, scheme, stream);
}

void kc_launch_multi_plain_f64(const kc::DMesh& m, const MultiHead* head, const StepPack<double>* packs, long long P,
                               int dims, int scheme, int block, cudaStream_t stream) {
    launch_multi_kernel<double, kc::PlainForm<double>>(m, head, packs, P, dims, scheme, block, stream);
}
