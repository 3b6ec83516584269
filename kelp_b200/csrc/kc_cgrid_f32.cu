// The NEMO C-grid steps on float face rasters (plain form).
#include "kc_launch.h"

void kc_launch_cgrid_f32(const kc::DMesh& m, const kc::DBlend<float>& f, const kc::DState& st, const kc::DStep& s,
                         int dims, int scheme, cudaStream_t stream) {
    launch_cgrid_kernel<float>(m, f, st, s, dims, scheme, stream);
}
