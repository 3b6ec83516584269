// Launchers of the step kernels, one set per translation unit so the kernel
// instantiations compile in parallel (kc_plain_f64.cu, kc_plain_f32.cu,
// kc_mixed_f32.cu, kc_mixed_f16.cu, kc_cgrid_f64.cu, kc_cgrid_f32.cu,
// kc_cgrid_mixed.cu, kc_sigma.cu).  kc_api.cu calls them; the kernels are kc_kernels.cuh.
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>

#include "kc_kernels.cuh"

// one step of every particle: dims 2 / 3, scheme 0 Euler, 1 RK2, 2 RK4
void kc_launch_plain_f64(const kc::DMesh& m, const kc::DBlend<double>& f, const kc::DState& st, const kc::DStep& s,
                         int dims, int scheme, cudaStream_t stream);
void kc_launch_plain_f32(const kc::DMesh& m, const kc::DBlend<float>& f, const kc::DState& st, const kc::DStep& s,
                         int dims, int scheme, cudaStream_t stream);
void kc_launch_mixed_f32(const kc::DMesh& m, const kc::DBlend<float>& f, const kc::DState& st, const kc::DStep& s,
                         int dims, int scheme, cudaStream_t stream);
void kc_launch_mixed_f16(const kc::DMesh& m, const kc::DBlend<__half>& f, const kc::DState& st,
                         const kc::DStep& s, int dims, int scheme, cudaStream_t stream);

// the fused multi-step launch (k_multi)
void kc_launch_multi_plain_f64(const kc::DMesh& m, const MultiHead* head, const StepPack<double>* packs, long long P,
                               int dims, int scheme, int block, cudaStream_t stream);
void kc_launch_multi_plain_f32(const kc::DMesh& m, const MultiHead* head, const StepPack<float>* packs, long long P,
                               int dims, int scheme, int block, cudaStream_t stream);
void kc_launch_multi_mixed_f32(const kc::DMesh& m, const MultiHead* head, const StepPack<float>* packs, long long P,
                               int dims, int scheme, int block, cudaStream_t stream);
void kc_launch_multi_mixed_f16(const kc::DMesh& m, const MultiHead* head, const StepPack<__half>* packs, long long P,
                               int dims, int scheme, int block, cudaStream_t stream);

// NEMO C-grid meshes, sigma meshes, element-centre least squares (plain form)
void kc_launch_cgrid_f64(const kc::DMesh& m, const kc::DBlend<double>& f, const kc::DState& st, const kc::DStep& s,
                         int dims, int scheme, cudaStream_t stream);
void kc_launch_cgrid_f32(const kc::DMesh& m, const kc::DBlend<float>& f, const kc::DState& st, const kc::DStep& s,
                         int dims, int scheme, cudaStream_t stream);
// the mixed form's 3-D C-grid step (kc_cgrid_mixed.cu)
void kc_launch_cgrid_mixed_f32(const kc::DMesh& m, const kc::DBlend<float>& f, const kc::DState& st,
                               const kc::DStep& s, int scheme, cudaStream_t stream);
void kc_launch_cgrid_mixed_f16(const kc::DMesh& m, const kc::DBlend<__half>& f, const kc::DState& st,
                               const kc::DStep& s, int scheme, cudaStream_t stream);
void kc_launch_sigma_f64(const kc::DMesh& m, const kc::DBlend<double>& f, const kc::DState& st, const kc::DStep& s,
                         int scheme, cudaStream_t stream);
void kc_launch_sigma_f32(const kc::DMesh& m, const kc::DBlend<float>& f, const kc::DState& st, const kc::DStep& s,
                         int scheme, cudaStream_t stream);
void kc_launch_lsq_f64(const kc::DMesh& m, const kc::DBlend<double>& f, const kc::DState& st, const kc::DStep& s,
                       int dims, int scheme, cudaStream_t stream);
void kc_launch_lsq_f32(const kc::DMesh& m, const kc::DBlend<float>& f, const kc::DState& st, const kc::DStep& s,
                       int dims, int scheme, cudaStream_t stream);
