// Device helpers shared by the solver kernels: deterministic block
// reductions, the device-resident iteration state and the partial-sum arrays.
#pragma once
#include "ofea_internal.cuh"

namespace ofea {

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block sum over kBlock threads, result in every thread, fixed order.
template <class T>
__device__ __forceinline__ T block_sum(T v, T *sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    T s = 0;
#pragma unroll
    for (int w = 0; w < kWarpsPerBlock; ++w) s += sh[w];
    return s;
}

template <class T>
__device__ __forceinline__ T sum_partials(const T *P, int cnt, T *sh) {
    T s = 0;
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) s += P[i];
    return block_sum(s, sh);
}

// Device-resident solver state.
struct Flags {
    int done;    // 1: stop (converged, breakdown)
    int status;  // OFEA_OK / OFEA_ERR_BREAKDOWN
    int itA;     // iteration index read by A (written by B)
    int itB;     // iteration index read by B (written by A)
    int iters;   // completed iterations
    int pad[3];
};

// The stop flag is written by CTA 0 of some kernels while other CTAs of the
// same kernel may be starting: read it once per CTA and broadcast, so every
// thread of a CTA takes the same path before any barrier.
__device__ __forceinline__ bool cta_done(const Flags *fl) {
    __shared__ int s_done;
    if (threadIdx.x == 0) s_done = *(volatile const int *)&fl->done;
    __syncthreads();
    return s_done != 0;
}

// Per-CTA partial sums, all arrays of kMaxGrid doubles.
struct Parts {
    double *pq, *rz0, *rz1, *rzo, *rr, *ff;
    int G;  // CTAs of every reducing kernel
};

__device__ __forceinline__ void block3_apply(const double *D, const double *v, double *o) {
    o[0] = D[0] * v[0] + D[1] * v[1] + D[2] * v[2];
    o[1] = D[3] * v[0] + D[4] * v[1] + D[5] * v[2];
    o[2] = D[6] * v[0] + D[7] * v[1] + D[8] * v[2];
}
__device__ __forceinline__ void block3_apply(const float *D, const float *v, float *o) {
    o[0] = D[0] * v[0] + D[1] * v[1] + D[2] * v[2];
    o[1] = D[3] * v[0] + D[4] * v[1] + D[5] * v[2];
    o[2] = D[6] * v[0] + D[7] * v[1] + D[8] * v[2];
}

}  // namespace ofea
