// Launch shape and the step kernels of both numerical forms (one thread per
// particle), shared by the translation units that instantiate them.
#pragma once
#include "kc_beach.cuh"
#include "kc_sigma.cuh"
#include "kc_cgrid.cuh"

#ifndef KC_BLOCK
#define KC_BLOCK 128   // threads per block of every kernel (a build option)
#endif
#ifndef KC_STEP_MIN_BLOCKS
// resident blocks per SM the step kernels' register budget must allow: 8
// blocks of 128 threads cap them at 64 registers (measured fastest on the
// HEALPix 3-D step: the path is latency-bound, occupancy beats spills)
#define KC_STEP_MIN_BLOCKS 8
#endif
#ifndef KC_RK2_3D_MIN_BLOCKS
// the fused 3-D RK2 step (the HEALPix benchmark's kernel): 10 blocks of 128
// cap it at 48 registers, measured 2 % faster there than 64 (and 40
// registers no faster)
#define KC_RK2_3D_MIN_BLOCKS 10
#endif
#ifndef KC_UNFUSED_3D_MIN_BLOCKS
// the 3-D RK4 / Euler step likewise (depth-linear RK4 benchmark: 3-5 % faster
// at 48 registers; the 2-D and C-grid steps measured slower there)
#define KC_UNFUSED_3D_MIN_BLOCKS 10
#endif
constexpr int kBlock = KC_BLOCK;

// delayed release (release.py:112-129): NOT_RELEASED -> ALIVE at its step
__device__ __forceinline__ void activate(const kc::DState& st, const kc::DStep& s, long long i) {
    if (st.release_step && s.global_step >= 0 && st.status[i] == kc::NOT_RELEASED &&
        s.global_step >= (long long)st.release_step[i])
        st.status[i] = kc::ALIVE;
}

template <typename T, int SCHEME, typename Form, bool WALK>
__global__ void __launch_bounds__(kBlock, KC_STEP_MIN_BLOCKS) k_step2d(const __grid_constant__ kc::DMesh m, const __grid_constant__ kc::DBlend<T> f, const __grid_constant__ kc::DState st, const __grid_constant__ kc::DStep s) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= st.P) return;
    activate(st, s, i);
    if (st.prev) st.prev[i] = st.status[i];
    kc::step2d_particle<T, SCHEME, Form, WALK>(m, f, st, s, i);
}

template <typename T, typename Form, bool WALK>
__global__ void __launch_bounds__(kBlock, KC_RK2_3D_MIN_BLOCKS) k_step3d_rk2(const __grid_constant__ kc::DMesh m, const __grid_constant__ kc::DBlend<T> f, const __grid_constant__ kc::DState st, const __grid_constant__ kc::DStep s) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= st.P) return;
    activate(st, s, i);
    if (st.prev) st.prev[i] = st.status[i];
    kc::step3d_rk2_particle<T, Form, WALK>(m, f, st, s, i);
}

template <typename T, int SCHEME, typename Form, bool WALK>
__global__ void __launch_bounds__(kBlock, KC_UNFUSED_3D_MIN_BLOCKS) k_step3d_unfused(const __grid_constant__ kc::DMesh m,
                                                           const __grid_constant__ kc::DBlend<T> f,
                                                           const __grid_constant__ kc::DState st,
                                                           const __grid_constant__ kc::DStep s) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= st.P) return;
    activate(st, s, i);
    if (st.prev) st.prev[i] = st.status[i];
    kc::step3d_unfused_particle<T, SCHEME, Form, WALK>(m, f, st, s, i);
}


template <typename T, int SCHEME, bool WALK>
__global__ void __launch_bounds__(kBlock, KC_STEP_MIN_BLOCKS) k_step3d_sigma(const __grid_constant__ kc::DMesh m,
                                                                         const __grid_constant__ kc::DBlend<T> f,
                                                                         const __grid_constant__ kc::DState st,
                                                                         const __grid_constant__ kc::DStep s) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= st.P) return;
    activate(st, s, i);
    if (st.prev) st.prev[i] = st.status[i];
    kc::step3d_sigma_particle<T, SCHEME, WALK>(m, f, st, s, i);
}

// The 3-D step of a sigma mesh (plain form): scheme 0 Euler, 1 RK2, 2 RK4.
template <typename T>
void launch_sigma_kernel(const kc::DMesh& m, const kc::DBlend<T>& f, const kc::DState& st, const kc::DStep& s,
                         int scheme, cudaStream_t stream) {
    const unsigned g = (unsigned)((st.P + kBlock - 1) / kBlock);
    if (st.elem) {
        if (scheme == 0) k_step3d_sigma<T, 0, true><<<g, kBlock, 0, stream>>>(m, f, st, s);
        else if (scheme == 1) k_step3d_sigma<T, 1, true><<<g, kBlock, 0, stream>>>(m, f, st, s);
        else k_step3d_sigma<T, 2, true><<<g, kBlock, 0, stream>>>(m, f, st, s);
    } else {
        if (scheme == 0) k_step3d_sigma<T, 0, false><<<g, kBlock, 0, stream>>>(m, f, st, s);
        else if (scheme == 1) k_step3d_sigma<T, 1, false><<<g, kBlock, 0, stream>>>(m, f, st, s);
        else k_step3d_sigma<T, 2, false><<<g, kBlock, 0, stream>>>(m, f, st, s);
    }
}

template <typename T, int SCHEME, bool MIXED = false>
__global__ void __launch_bounds__(kBlock, KC_STEP_MIN_BLOCKS) k_step3d_cgrid(const __grid_constant__ kc::DMesh m,
                                                                         const __grid_constant__ kc::DBlend<T> f,
                                                                         const __grid_constant__ kc::DState st,
                                                                         const __grid_constant__ kc::DStep s) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= st.P) return;
    activate(st, s, i);
    if (st.prev) st.prev[i] = st.status[i];
    kc::step3d_cgrid_particle<T, SCHEME, MIXED>(m, f, st, s, i);
}

// The 3-D C-grid step of the mixed form (float32 or scaled float16 rasters).
template <typename T>
void launch_cgrid_mixed_kernel(const kc::DMesh& m, const kc::DBlend<T>& f, const kc::DState& st, const kc::DStep& s,
                               int scheme, cudaStream_t stream) {
    const unsigned g = (unsigned)((st.P + kBlock - 1) / kBlock);
    if (scheme == 0) k_step3d_cgrid<T, 0, true><<<g, kBlock, 0, stream>>>(m, f, st, s);
    else if (scheme == 1) k_step3d_cgrid<T, 1, true><<<g, kBlock, 0, stream>>>(m, f, st, s);
    else k_step3d_cgrid<T, 2, true><<<g, kBlock, 0, stream>>>(m, f, st, s);
}

// One step on a NEMO C-grid mesh (plain form): the 2-D steps read the
// surface faces through CgridForm (edge walk when the state carries
// elements); the 3-D step is the fractional-level one (elements untouched).
template <typename T>
void launch_cgrid_kernel(const kc::DMesh& m, const kc::DBlend<T>& f, const kc::DState& st, const kc::DStep& s,
                         int dims, int scheme, cudaStream_t stream) {
    const unsigned g = (unsigned)((st.P + kBlock - 1) / kBlock);
    using F = kc::CgridForm<T>;
    if (dims == 3) {
        if (scheme == 0) k_step3d_cgrid<T, 0><<<g, kBlock, 0, stream>>>(m, f, st, s);
        else if (scheme == 1) k_step3d_cgrid<T, 1><<<g, kBlock, 0, stream>>>(m, f, st, s);
        else k_step3d_cgrid<T, 2><<<g, kBlock, 0, stream>>>(m, f, st, s);
    } else if (st.elem) {
        if (scheme == 0) k_step2d<T, 0, F, true><<<g, kBlock, 0, stream>>>(m, f, st, s);
        else if (scheme == 1) k_step2d<T, 1, F, true><<<g, kBlock, 0, stream>>>(m, f, st, s);
        else k_step2d<T, 2, F, true><<<g, kBlock, 0, stream>>>(m, f, st, s);
    } else {
        if (scheme == 0) k_step2d<T, 0, F, false><<<g, kBlock, 0, stream>>>(m, f, st, s);
        else if (scheme == 1) k_step2d<T, 1, F, false><<<g, kBlock, 0, stream>>>(m, f, st, s);
        else k_step2d<T, 2, F, false><<<g, kBlock, 0, stream>>>(m, f, st, s);
    }
}

// Launch one step of every particle: dims 2 / 3, scheme 0 Euler, 1 RK2, 2 RK4;
// the walk-mode instantiations when the state carries elements.
template <typename T, typename Form, bool WALK>
void launch_step_kernel_t(const kc::DMesh& m, const kc::DBlend<T>& f, const kc::DState& st, const kc::DStep& s,
                          int dims, int scheme, cudaStream_t stream) {
    const unsigned g = (unsigned)((st.P + kBlock - 1) / kBlock);
    if (dims == 2) {
        if (scheme == 0) k_step2d<T, 0, Form, WALK><<<g, kBlock, 0, stream>>>(m, f, st, s);
        else if (scheme == 1) k_step2d<T, 1, Form, WALK><<<g, kBlock, 0, stream>>>(m, f, st, s);
        else k_step2d<T, 2, Form, WALK><<<g, kBlock, 0, stream>>>(m, f, st, s);
    } else {
        if (scheme == 1) k_step3d_rk2<T, Form, WALK><<<g, kBlock, 0, stream>>>(m, f, st, s);
        else if (scheme == 2) k_step3d_unfused<T, 2, typename kc::UnfusedFormOf<Form>::type, WALK><<<g, kBlock, 0, stream>>>(m, f, st, s);
        else k_step3d_unfused<T, 0, typename kc::UnfusedFormOf<Form>::type, WALK><<<g, kBlock, 0, stream>>>(m, f, st, s);
    }
}

template <typename T, typename Form>
void launch_step_kernel(const kc::DMesh& m, const kc::DBlend<T>& f, const kc::DState& st, const kc::DStep& s,
                        int dims, int scheme, cudaStream_t stream) {
    if (st.elem) launch_step_kernel_t<T, Form, true>(m, f, st, s, dims, scheme, stream);
    else launch_step_kernel_t<T, Form, false>(m, f, st, s, dims, scheme, stream);
}

// 2-D steps with element-centre least-squares u/v (LsqForm), local search
template <typename T, typename Form = kc::LsqForm<T>>
void launch_lsq_kernel(const kc::DMesh& m, const kc::DBlend<T>& f, const kc::DState& st, const kc::DStep& s,
                       int dims, int scheme, cudaStream_t stream) {
    const unsigned g = (unsigned)((st.P + kBlock - 1) / kBlock);
    if (dims == 3) {   // the 3-D RK2 (arithmetic of the unfused RK2) and the unfused RK4 / Euler
        if (scheme == 1) k_step3d_rk2<T, Form, false><<<g, kBlock, 0, stream>>>(m, f, st, s);
        else if (scheme == 2) k_step3d_unfused<T, 2, Form, false><<<g, kBlock, 0, stream>>>(m, f, st, s);
        else k_step3d_unfused<T, 0, Form, false><<<g, kBlock, 0, stream>>>(m, f, st, s);
        return;
    }
    if (scheme == 0) k_step2d<T, 0, Form, false><<<g, kBlock, 0, stream>>>(m, f, st, s);
    else if (scheme == 1) k_step2d<T, 1, Form, false><<<g, kBlock, 0, stream>>>(m, f, st, s);
    else k_step2d<T, 2, Form, false><<<g, kBlock, 0, stream>>>(m, f, st, s);
}

// ---------------------------------------------------------------------------
// Fused multi-step launch: each thread carries its particles through n steps
// (particles are independent within and across steps), running the beaching
// hook after a step where asked.  Everything that changes between calls is
// read from device memory: the state view (kc_sort swaps its buffers) and,
// per step, the snapshot blend, the step arguments and the beaching
// arguments.  So one launch can be captured in a CUDA graph and replayed with
// the next steps' arguments copied into the same device buffer.  Local
// element search only: a state that carries walk elements steps through the
// per-step kernels.
// ---------------------------------------------------------------------------

template <typename T>
struct StepPack {
    kc::DBlend<T> f;
    kc::DStep s;
    kc::DBeach b;
    int beach;   // run the beaching hook after this step
};

struct MultiHead {
    kc::DState st;
    long long N;   // mesh nodes (the beaching anchor wrap)
    int n_steps;
};

// BLOCK threads per block; the resident threads per SM those bounds ask for
// are the per-step kernels' (1024 for 2-D: 64 registers; 128 x
// KC_RK2_3D_MIN_BLOCKS / KC_UNFUSED_3D_MIN_BLOCKS for 3-D), so a fused
// launch gets the same register budget at either block size.
template <int DIMS, int SCHEME>
constexpr int multi_threads_per_sm() {
    return DIMS == 2 ? 1024 : 128 * (SCHEME == 1 ? KC_RK2_3D_MIN_BLOCKS : KC_UNFUSED_3D_MIN_BLOCKS);
}

template <typename T, int DIMS, int SCHEME, typename Form, int BLOCK>
__global__ void __launch_bounds__(BLOCK, multi_threads_per_sm<DIMS, SCHEME>() / BLOCK) k_multi(const __grid_constant__ kc::DMesh m,
                                                                     const MultiHead* __restrict__ head,
                                                                     const StepPack<T>* __restrict__ packs) {
    const kc::DState& st = head->st;
    const long long P = st.P;
    const long long N = head->N;
    const int n = head->n_steps;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < P;
         i += (long long)gridDim.x * blockDim.x) {
        for (int j = 0; j < n; ++j) {
            const StepPack<T>& pk = packs[j];
            activate(st, pk.s, i);
            if (st.prev) st.prev[i] = st.status[i];
            if (DIMS == 2) kc::step2d_particle<T, SCHEME, Form>(m, pk.f, st, pk.s, i);
            else if (SCHEME == 1) kc::step3d_rk2_particle<T, Form>(m, pk.f, st, pk.s, i);
            else kc::step3d_unfused_particle<T, SCHEME, typename kc::UnfusedFormOf<Form>::type>(m, pk.f, st, pk.s, i);
            if (pk.beach) kc::beach_particle(m, st, pk.b, N, i);
        }
    }
}

// Persistent grid: every SM's resident blocks, no more than the particles need.
template <typename K>
unsigned persistent_grid(K kernel, long long P, int block) {
    int dev = 0, sms = 1, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0);
    if (per_sm < 1) per_sm = 1;
    const long long need = (P + block - 1) / block;
    const long long cap = (long long)sms * per_sm;
    return (unsigned)(need < cap ? (need > 0 ? need : 1) : cap);
}

template <typename T, typename Form, int DIMS, int SCHEME>
void launch_multi_one(const kc::DMesh& m, const MultiHead* head, const StepPack<T>* packs, long long P, int block,
                      cudaStream_t stream) {
    if (block == 256) {
        auto kern = k_multi<T, DIMS, SCHEME, Form, 256>;
        kern<<<persistent_grid(kern, P, 256), 256, 0, stream>>>(m, head, packs);
    } else {
        auto kern = k_multi<T, DIMS, SCHEME, Form, 128>;
        kern<<<persistent_grid(kern, P, 128), 128, 0, stream>>>(m, head, packs);
    }
}

template <typename T, typename Form>
void launch_multi_kernel(const kc::DMesh& m, const MultiHead* head, const StepPack<T>* packs, long long P, int dims,
                         int scheme, int block, cudaStream_t stream) {
    if (dims == 2) {
        if (scheme == 0) launch_multi_one<T, Form, 2, 0>(m, head, packs, P, block, stream);
        else if (scheme == 1) launch_multi_one<T, Form, 2, 1>(m, head, packs, P, block, stream);
        else launch_multi_one<T, Form, 2, 2>(m, head, packs, P, block, stream);
    } else {
        if (scheme == 1) launch_multi_one<T, Form, 3, 1>(m, head, packs, P, block, stream);
        else if (scheme == 2) launch_multi_one<T, Form, 3, 2>(m, head, packs, P, block, stream);
        else launch_multi_one<T, Form, 3, 0>(m, head, packs, P, block, stream);
    }
}
