// Launch shape and the step kernels of both numerical forms (one thread per
// particle), shared by the translation units that instantiate them.
#pragma once
#include "kc_step.cuh"

#ifndef KC_BLOCK
#define KC_BLOCK 128   // threads per block of every kernel (a build option)
#endif
#ifndef KC_STEP_MIN_BLOCKS
// resident blocks per SM the step kernels' register budget must allow: 8
// blocks of 128 threads cap them at 64 registers (measured fastest on the
// HEALPix 3-D step: the path is latency-bound, occupancy beats spills)
#define KC_STEP_MIN_BLOCKS 8
#endif
constexpr int kBlock = KC_BLOCK;

// delayed release (release.py:112-129): NOT_RELEASED -> ALIVE at its step
__device__ __forceinline__ void activate(const kc::DState& st, const kc::DStep& s, long long i) {
    if (st.release_step && s.global_step >= 0 && st.status[i] == kc::NOT_RELEASED &&
        s.global_step >= (long long)st.release_step[i])
        st.status[i] = kc::ALIVE;
}

template <typename T, int SCHEME, typename Form>
__global__ void __launch_bounds__(kBlock, KC_STEP_MIN_BLOCKS) k_step2d(const __grid_constant__ kc::DMesh m, const __grid_constant__ kc::DBlend<T> f, const __grid_constant__ kc::DState st, const __grid_constant__ kc::DStep s) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= st.P) return;
    activate(st, s, i);
    if (st.prev) st.prev[i] = st.status[i];
    kc::step2d_particle<T, SCHEME, Form>(m, f, st, s, i);
}

template <typename T, typename Form>
__global__ void __launch_bounds__(kBlock, KC_STEP_MIN_BLOCKS) k_step3d_rk2(const __grid_constant__ kc::DMesh m, const __grid_constant__ kc::DBlend<T> f, const __grid_constant__ kc::DState st, const __grid_constant__ kc::DStep s) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= st.P) return;
    activate(st, s, i);
    if (st.prev) st.prev[i] = st.status[i];
    kc::step3d_rk2_particle<T, Form>(m, f, st, s, i);
}

template <typename T, int SCHEME, typename Form>
__global__ void __launch_bounds__(kBlock, KC_STEP_MIN_BLOCKS) k_step3d_unfused(const __grid_constant__ kc::DMesh m,
                                                           const __grid_constant__ kc::DBlend<T> f,
                                                           const __grid_constant__ kc::DState st,
                                                           const __grid_constant__ kc::DStep s) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= st.P) return;
    activate(st, s, i);
    if (st.prev) st.prev[i] = st.status[i];
    kc::step3d_unfused_particle<T, SCHEME, Form>(m, f, st, s, i);
}


// Launch one step of every particle: dims 2 / 3, scheme 0 Euler, 1 RK2, 2 RK4.
template <typename T, typename Form>
void launch_step_kernel(const kc::DMesh& m, const kc::DBlend<T>& f, const kc::DState& st, const kc::DStep& s,
                        int dims, int scheme, cudaStream_t stream) {
    const unsigned g = (unsigned)((st.P + kBlock - 1) / kBlock);
    if (dims == 2) {
        if (scheme == 0) k_step2d<T, 0, Form><<<g, kBlock, 0, stream>>>(m, f, st, s);
        else if (scheme == 1) k_step2d<T, 1, Form><<<g, kBlock, 0, stream>>>(m, f, st, s);
        else k_step2d<T, 2, Form><<<g, kBlock, 0, stream>>>(m, f, st, s);
    } else {
        if (scheme == 1) k_step3d_rk2<T, Form><<<g, kBlock, 0, stream>>>(m, f, st, s);
        else if (scheme == 2) k_step3d_unfused<T, 2, Form><<<g, kBlock, 0, stream>>>(m, f, st, s);
        else k_step3d_unfused<T, 0, Form><<<g, kBlock, 0, stream>>>(m, f, st, s);
    }
}
