// The mixed form's 3-D C-grid step on float32 and scaled float16 face
// rasters (float32 values and fluxes, float64 geometry and positions).
#include "kc_launch.h"

void kc_launch_cgrid_mixed_f32(const kc::DMesh& m, const kc::DBlend<float>& f, const kc::DState& st,
                               const kc::DStep& s, int scheme, cudaStream_t stream) {
    launch_cgrid_mixed_kernel<float>(m, f, st, s, scheme, stream);
}

void kc_launch_cgrid_mixed_f16(const kc::DMesh& m, const kc::DBlend<__half>& f, const kc::DState& st,
                               const kc::DStep& s, int scheme, cudaStream_t stream) {
    launch_cgrid_mixed_kernel<__half>(m, f, st, s, scheme, stream);
}
