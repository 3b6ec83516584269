// The element-centre least-squares steps (plain form) on float64 and float32
// snapshots: the 2-D fused Euler / RK2 / RK4 and the 3-D RK2 / RK4 / Euler, for
// the element-centre fit and the edge-neighbour fit (DStep.edge_bc >= 0).
#include "kc_launch.h"

void kc_launch_lsq_f64(const kc::DMesh& m, const kc::DBlend<double>& f, const kc::DState& st, const kc::DStep& s,
                       int dims, int scheme, cudaStream_t stream) {
    if (s.edge_bc >= 0) launch_lsq_kernel<double, kc::EdgeLsqForm<double>>(m, f, st, s, dims, scheme, stream);
    else launch_lsq_kernel<double>(m, f, st, s, dims, scheme, stream);
}

void kc_launch_lsq_f32(const kc::DMesh& m, const kc::DBlend<float>& f, const kc::DState& st, const kc::DStep& s,
                       int dims, int scheme, cudaStream_t stream) {
    if (s.edge_bc >= 0) launch_lsq_kernel<float, kc::EdgeLsqForm<float>>(m, f, st, s, dims, scheme, stream);
    else launch_lsq_kernel<float>(m, f, st, s, dims, scheme, stream);
}
