// SELL-32 component-major block layout shared by the solver kernels (see sell.cu).
#pragma once

#include <cuda_bf16.h>

#include <cstdint>

namespace plato {

struct SellPattern {
    int32_t  nslices = 0;
    int32_t* width = nullptr;       // [nslices] blocks per row in the slice (max over its rows)
    int64_t* ptr = nullptr;         // [nslices+1] first slot of each slice
    int32_t* cols = nullptr;        // [total_slots] column node of each slot
    int16_t* dcols = nullptr;       // [total_slots] column - 32 * slice, when every one fits in 16 bits
    int64_t  total_slots = 0;
    int32_t  max_slice_blocks = 0;  // max CRS blocks in one slice (transpose tile size)
};

struct SellView {
    int32_t        num_rows;
    const int32_t* width;
    const int64_t* ptr;
    const int32_t* cols;
    const int16_t* dcols;  // nullptr unless the mesh numbering keeps every column within 16 bits
};

__device__ __forceinline__ float to_float(float v) { return v; }
__device__ __forceinline__ float to_float(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ double to_acc(double v) { return v; }

// y_r = sum_k A(r, k) x(col(r, k)) for one node row; TV = entry type, TA = accumulation type.
template <typename TA, typename TV, typename TX>
__device__ __forceinline__ void sell_row(const SellView& A, const TV* __restrict__ vals, const TX* __restrict__ x,
                                         int64_t r, TA& a0, TA& a1, TA& a2) {
    const int64_t s = r >> 5;
    const int l = int(r & 31);
    const int w = __ldg(A.width + s);
    const int64_t base = __ldg(A.ptr + s);
    const int32_t* __restrict__ c = A.cols + base + l;
    const TV* __restrict__ v = vals + 9 * base + l;
    a0 = a1 = a2 = TA(0);
#pragma unroll 4
    for (int k = 0; k < w; ++k) {
        const int64_t col = __ldg(c + 32 * k);
        const TA x0 = TA(__ldg(x + 3 * col)), x1 = TA(__ldg(x + 3 * col + 1)), x2 = TA(__ldg(x + 3 * col + 2));
        const TV* vk = v + 288 * k;
        a0 += TA(vk[0]) * x0 + TA(vk[32]) * x1 + TA(vk[64]) * x2;
        a1 += TA(vk[96]) * x0 + TA(vk[128]) * x1 + TA(vk[160]) * x2;
        a2 += TA(vk[192]) * x0 + TA(vk[224]) * x1 + TA(vk[256]) * x2;
    }
}

// BF16 entries are widened to FP32 before the multiply.
template <typename TX>
__device__ __forceinline__ void sell_row_bf16(const SellView& A, const __nv_bfloat16* __restrict__ vals,
                                              const TX* __restrict__ x, int64_t r, float& a0, float& a1,
                                              float& a2) {
    const int64_t s = r >> 5;
    const int l = int(r & 31);
    const int w = __ldg(A.width + s);
    const int64_t base = __ldg(A.ptr + s);
    const int32_t* __restrict__ c = A.cols + base + l;
    const __nv_bfloat16* __restrict__ v = vals + 9 * base + l;
    a0 = a1 = a2 = 0.f;
#pragma unroll 4
    for (int k = 0; k < w; ++k) {
        const int64_t col = __ldg(c + 32 * k);
        const float x0 = float(__ldg(x + 3 * col)), x1 = float(__ldg(x + 3 * col + 1)),
                    x2 = float(__ldg(x + 3 * col + 2));
        const __nv_bfloat16* vk = v + 288 * k;
        a0 += __bfloat162float(vk[0]) * x0 + __bfloat162float(vk[32]) * x1 + __bfloat162float(vk[64]) * x2;
        a1 += __bfloat162float(vk[96]) * x0 + __bfloat162float(vk[128]) * x1 + __bfloat162float(vk[160]) * x2;
        a2 += __bfloat162float(vk[192]) * x0 + __bfloat162float(vk[224]) * x1 + __bfloat162float(vk[256]) * x2;
    }
}

}  // namespace plato
