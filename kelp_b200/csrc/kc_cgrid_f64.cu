// The NEMO C-grid steps on double face rasters (plain form).
#include "kc_launch.h"

void kc_launch_cgrid_f64(const kc::DMesh& m, const kc::DBlend<double>& f, const kc::DState& st, const kc::DStep& s,
                         int dims, int scheme, cudaStream_t stream) {
    launch_cgrid_kernel<double>(m, f, st, s, dims, scheme, stream);
}
