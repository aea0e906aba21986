// Block-level reduction helpers of the solver kernels: warp/block sums and the
// last-block-done pattern that finishes a grid-wide reduction without an extra launch.
#pragma once

#include "plato_internal.cuh"

namespace plato {

constexpr int kThreads = 256;

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sums NV per-thread values over the block; every thread of warp 0 gets the result.
template <int NV>
__device__ __forceinline__ void block_sum_n(double (&v)[NV], double (*sh)[32]) {
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = warp_sum(v[q]);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0)
#pragma unroll
        for (int q = 0; q < NV; ++q) sh[q][w] = v[q];
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
#pragma unroll
        for (int q = 0; q < NV; ++q) v[q] = warp_sum(l < nw ? sh[q][l] : 0.0);
    }
    __syncthreads();
}

// Stores the block's sums in partials[NV*block + q]; returns true in the block that
// arrives last (its view of partials is then complete).
template <int NV>
__device__ __forceinline__ bool publish_partials(const double (&v)[NV], double* partials,
                                                 unsigned int* ticket, bool* sh_last) {
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) partials[NV * blockIdx.x + q] = v[q];
        __threadfence();
        *sh_last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    return *sh_last;
}

// Sums the partials of every block in block order (deterministic).
template <int NV>
__device__ __forceinline__ void final_sums(double (&t)[NV], const double* partials, double (*sh)[32]) {
    __threadfence();
#pragma unroll
    for (int q = 0; q < NV; ++q) t[q] = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
#pragma unroll
        for (int q = 0; q < NV; ++q) t[q] += partials[NV * b + q];
    block_sum_n<NV>(t, sh);
}

}  // namespace plato
