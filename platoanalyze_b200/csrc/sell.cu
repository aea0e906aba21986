// Solver-private sliced-ELL copy of the 3x3 block matrix (SELL-32, component-major).
//
// The API hands out the reference's block CRS (row-major 3x3 blocks, rows contiguous).  A
// warp-per-row CRS SpMV spends most of its time in shuffles and dependent loads, so the
// solver works on a second layout: node rows are grouped in slices of 32; slice s has
// width w_s = max blocks of its rows; block k of row 32s+l sits at slot ptr_s + 32k + l and
// its 9 entries are stored component-major, entry q at value index 9 ptr_s + 32(9k + q) + l.
// A thread owns one row: for each k it loads the column (one 128 B line per warp) and the 9
// entries (nine 256 B lines per warp), gathers x through L2, and accumulates its three row
// sums in registers.  Padding slots have value 0 and column = the row itself.
//
// The copy is made once per solve from the constrained CRS by a per-slice shared-memory
// transpose (both sides coalesced), which also extracts the Jacobi diagonal and can emit
// FP32 and BF16 copies of the entries for the mixed-precision preconditioner.
#include <mutex>

#include <cub/cub.cuh>
#include <cuda_bf16.h>

#include <cuda_fp16.h>

#include "plato_internal.cuh"
#include "sell.cuh"

namespace plato {
namespace {

__host__ __device__ __forceinline__ int64_t llmin(int64_t a, int64_t b) { return a < b ? a : b; }

constexpr int kSliceThreads = 256;

__global__ void k_slice_width(int32_t N, int32_t nslices, const int32_t* __restrict__ row_map,
                              int32_t* __restrict__ width, int64_t* __restrict__ slots,
                              int32_t* __restrict__ slice_nnz) {
    const int lane = threadIdx.x & 31;
    for (int64_t s = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; s < nslices;
         s += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int64_t r = 32 * s + lane;
        int nb = 0;
        if (r < N) nb = row_map[r + 1] - row_map[r];
        for (int o = 16; o > 0; o >>= 1) nb = max(nb, __shfl_xor_sync(0xffffffffu, nb, o));
        if (lane == 0) {
            width[s] = nb;
            slots[s] = 32 * (int64_t)nb;
            const int64_t r1 = llmin(32 * s + 32, N);
            slice_nnz[s] = row_map[r1] - row_map[32 * s];
        }
    }
}

__global__ void k_sell_cols(int32_t N, int32_t nslices, const int32_t* __restrict__ row_map,
                            const int32_t* __restrict__ cols, const int32_t* __restrict__ width,
                            const int64_t* __restrict__ ptr, int32_t* __restrict__ sell_cols) {
    for (int64_t s = blockIdx.x; s < nslices; s += gridDim.x) {
        const int w = width[s];
        const int64_t base = ptr[s];
        for (int t = threadIdx.x; t < 32 * w; t += blockDim.x) {
            const int k = t >> 5, l = t & 31;
            const int64_t r = 32 * s + l;
            int32_t c = 0;
            if (r < N) {
                const int32_t rs = row_map[r], nb = row_map[r + 1] - rs;
                c = (k < nb) ? cols[rs + k] : int32_t(r);
            }
            sell_cols[base + t] = c;
        }
    }
}

// Column offsets from the slice's first row, 16 bits each, for the FP16 sweep (whose
// column indices are otherwise 18 % of its bytes); `bad` counts offsets that do not fit.  The
// padding lanes past the last row (zero entries) point at the slice's first row.
__global__ void k_sell_dcols(int32_t N, int32_t nslices, const int64_t* __restrict__ ptr,
                             const int32_t* __restrict__ cols, int16_t* __restrict__ dcols,
                             int32_t* __restrict__ bad) {
    for (int64_t s = blockIdx.x; s < nslices; s += gridDim.x) {
        const int64_t base = ptr[s], end = ptr[s + 1];
        for (int64_t t = base + threadIdx.x; t < end; t += blockDim.x) {
            const int64_t r = 32 * s + ((t - base) & 31);
            const int64_t d = r < N ? int64_t(cols[t]) - 32 * s : 0;
            if (d < -32768 || d > 32767) {
                atomicAdd(bad, 1);
                dcols[t] = 0;
            } else {
                dcols[t] = int16_t(d);
            }
        }
    }
}

// Per-slice transpose CRS -> SELL (+ Jacobi diagonal, + optional FP32 / BF16 copies).
template <bool kSmem>
__global__ void __launch_bounds__(kSliceThreads)
k_crs_to_sell(int32_t N, int32_t nslices, const int32_t* __restrict__ row_map, const int32_t* __restrict__ diag,
              const int32_t* __restrict__ width, const int64_t* __restrict__ ptr,
              const double* __restrict__ crs, double* __restrict__ out64, float* __restrict__ out32,
              __nv_bfloat16* __restrict__ out16, double* __restrict__ dinv, float* __restrict__ dinv32) {
    extern __shared__ double tile[];
    __shared__ int32_t rs_sh[33];
    for (int64_t s = blockIdx.x; s < nslices; s += gridDim.x) {
        const int64_t r0 = 32 * s;
        const int nrows = int(llmin(32, N - r0));
        if (threadIdx.x <= 32) rs_sh[threadIdx.x] = row_map[llmin(r0 + threadIdx.x, N)];
        __syncthreads();
        const int64_t v0 = 9 * (int64_t)rs_sh[0];
        const int nvals = 9 * (rs_sh[nrows] - rs_sh[0]);
        if (kSmem)
            for (int t = threadIdx.x; t < nvals; t += blockDim.x) tile[t] = crs[v0 + t];
        __syncthreads();
        const double* src = kSmem ? tile : crs + v0;
        const int w = width[s];
        const int64_t base = 9 * ptr[s];
        for (int t = threadIdx.x; t < 9 * 32 * w; t += blockDim.x) {
            const int l = t & 31, kq = t >> 5;
            const int k = kq / 9, q = kq - 9 * k;
            double v = 0.0;
            if (l < nrows) {
                const int rs = rs_sh[l] - rs_sh[0], nb = rs_sh[l + 1] - rs_sh[l];
                if (k < nb) v = src[9 * (rs + k) + q];
            }
            if (out64) out64[base + t] = v;
            if (out32) out32[base + t] = float(v);
            if (out16) out16[base + t] = __float2bfloat16_rn(float(v));
        }
        if (threadIdx.x < 3 * nrows) {
            const int l = threadIdx.x / 3, i = threadIdx.x - 3 * l;
            const int64_t r = r0 + l;
            const double d = src[9 * (diag[r] - rs_sh[0]) + 4 * i];
            if (dinv) dinv[3 * r + i] = 1.0 / d;
            if (dinv32) dinv32[3 * r + i] = float(1.0 / d);
        }
        __syncthreads();
    }
}

// D^1/2, D^-1/2 (FP32) and the unit Jacobi diagonal of the scaled matrix, from dinv = 1/diag.
__global__ void k_scale_vectors(int64_t n, const double* __restrict__ dinv, float* __restrict__ sq,
                                float* __restrict__ isq, float* __restrict__ ones) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double di = dinv[i];
        sq[i] = float(1.0 / sqrt(di));
        isq[i] = float(sqrt(di));
        ones[i] = 1.0f;
    }
}

// FP16 copy of the Jacobi-scaled matrix: entry (a, b) of block k of row r, column node c,
// becomes A * isq[3r+a] * isq[3c+b] (isq = D^-1/2 in FP32, far finer than the FP16 result;
// the diagonal rounds to exactly 1), same slots as the FP64 SELL copy.  A thread owns one
// row of a slice: per block it loads the column once, the three isq of the column and the
// nine entries (coalesced across the warp), and stores nine halves.
__global__ void __launch_bounds__(256)
k_sell_scale16(int32_t N, int32_t nslices, const int32_t* __restrict__ width, const int64_t* __restrict__ ptr,
               const int32_t* __restrict__ cols, const double* __restrict__ sell64, const float* __restrict__ isq,
               __half* __restrict__ out16) {
    const int lane = threadIdx.x & 31;
    for (int64_t s = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; s < nslices;
         s += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int w = __ldg(width + s);
        const int64_t base = __ldg(ptr + s);
        const int64_t r = 32 * s + lane;
        float ir[3] = {0.f, 0.f, 0.f};
        if (r < N)
            for (int a = 0; a < 3; ++a) ir[a] = __ldg(isq + 3 * r + a);
        for (int k = 0; k < w; ++k) {
            const int64_t c = __ldg(cols + base + 32 * k + lane);
            const float ic0 = __ldg(isq + 3 * c), ic1 = __ldg(isq + 3 * c + 1), ic2 = __ldg(isq + 3 * c + 2);
            const double* v = sell64 + 9 * base + 32 * (9 * k) + lane;
            __half* o = out16 + 9 * base + 32 * (9 * k) + lane;
#pragma unroll
            for (int q = 0; q < 9; ++q) {
                const float ic = (q % 3) == 0 ? ic0 : ((q % 3) == 1 ? ic1 : ic2);
                o[32 * q] = __float2half_rn(float(__ldg(v + 32 * q)) * ir[q / 3] * ic);
            }
        }
    }
}

}  // namespace

int build_sell_pattern(plato_problem* h) {
    const int32_t N = h->N;
    const int32_t ns = (N + 31) / 32;
    cudaStream_t s = h->stream;
    SellPattern& P = h->sell;
    P.nslices = ns;
    PLATO_CUDA(h, cudaMalloc(&P.width, sizeof(int32_t) * ns));
    PLATO_CUDA(h, cudaMalloc(&P.ptr, sizeof(int64_t) * (ns + 1)));
    int64_t* slots = nullptr;
    int32_t* slice_nnz = nullptr;
    PLATO_CUDA(h, cudaMallocAsync(&slots, sizeof(int64_t) * (ns + 1), s));
    PLATO_CUDA(h, cudaMallocAsync(&slice_nnz, sizeof(int32_t) * ns, s));
    PLATO_CUDA(h, cudaMemsetAsync(slots, 0, sizeof(int64_t) * (ns + 1), s));
    k_slice_width<<<grid_for((int64_t)ns * 32, 256), 256, 0, s>>>(N, ns, h->row_map, P.width, slots, slice_nnz);
    PLATO_LAUNCH_CHECK(h);
    size_t tb = 0;
    PLATO_CUDA(h, cub::DeviceScan::ExclusiveSum(nullptr, tb, slots, P.ptr, ns + 1, s));
    void* tmp = nullptr;
    PLATO_CUDA(h, cudaMallocAsync(&tmp, tb, s));
    PLATO_CUDA(h, cub::DeviceScan::ExclusiveSum(tmp, tb, slots, P.ptr, ns + 1, s));
    size_t tb2 = 0;
    int32_t* d_max = nullptr;
    PLATO_CUDA(h, cudaMallocAsync(&d_max, sizeof(int32_t), s));
    PLATO_CUDA(h, cub::DeviceReduce::Max(nullptr, tb2, slice_nnz, d_max, ns, s));
    void* tmp2 = nullptr;
    PLATO_CUDA(h, cudaMallocAsync(&tmp2, tb2, s));
    PLATO_CUDA(h, cub::DeviceReduce::Max(tmp2, tb2, slice_nnz, d_max, ns, s));
    int32_t maxnnz = 0;
    PLATO_CUDA(h, cudaMemcpyAsync(&P.total_slots, P.ptr + ns, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    PLATO_CUDA(h, cudaMemcpyAsync(&maxnnz, d_max, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    PLATO_CUDA(h, cudaStreamSynchronize(s));
    P.max_slice_blocks = maxnnz;
    PLATO_CUDA(h, cudaMalloc(&P.cols, sizeof(int32_t) * (P.total_slots > 0 ? P.total_slots : 1)));
    k_sell_cols<<<grid_for(ns, 1, 148 * 64), 256, 0, s>>>(N, ns, h->row_map, h->cols, P.width, P.ptr, P.cols);
    PLATO_LAUNCH_CHECK(h);
    // the 16-bit column offsets (kept only when every column is within 32767 of its slice)
    PLATO_CUDA(h, cudaMalloc(&P.dcols, sizeof(int16_t) * (P.total_slots > 0 ? P.total_slots : 1)));
    PLATO_CUDA(h, cudaMemsetAsync(d_max, 0, sizeof(int32_t), s));
    k_sell_dcols<<<grid_for(ns, 1, 148 * 64), 256, 0, s>>>(N, ns, P.ptr, P.cols, P.dcols, d_max);
    PLATO_LAUNCH_CHECK(h);
    int32_t bad = 0;
    PLATO_CUDA(h, cudaMemcpyAsync(&bad, d_max, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    PLATO_CUDA(h, cudaFreeAsync(tmp, s));
    PLATO_CUDA(h, cudaFreeAsync(tmp2, s));
    PLATO_CUDA(h, cudaFreeAsync(d_max, s));
    PLATO_CUDA(h, cudaFreeAsync(slots, s));
    PLATO_CUDA(h, cudaFreeAsync(slice_nnz, s));
    PLATO_CUDA(h, cudaStreamSynchronize(s));
    if (bad) {
        PLATO_CUDA(h, cudaFree(P.dcols));
        P.dcols = nullptr;
    }
    return PLATO_OK;
}

int launch_crs_to_sell(plato_problem* h, const double* crs, double* out64, float* out32, void* out16,
                       double* dinv, float* dinv32) {
    const SellPattern& P = h->sell;
    const size_t smem = size_t(9) * P.max_slice_blocks * sizeof(double);
    const int grid = grid_for(P.nslices, 1, 148 * 16);
    if (smem <= 200 * 1024) {
        const int want = int(smem > 48 * 1024 ? smem : 48 * 1024);
        const int rc = ensure_smem_attribute(h, reinterpret_cast<const void*>(k_crs_to_sell<true>), want);
        if (rc) return rc;
        k_crs_to_sell<true><<<grid, kSliceThreads, smem, h->stream>>>(
            h->N, P.nslices, h->row_map, h->diag, P.width, P.ptr, crs, out64, out32,
            static_cast<__nv_bfloat16*>(out16), dinv, dinv32);
    } else {
        k_crs_to_sell<false><<<grid, kSliceThreads, 0, h->stream>>>(
            h->N, P.nslices, h->row_map, h->diag, P.width, P.ptr, crs, out64, out32,
            static_cast<__nv_bfloat16*>(out16), dinv, dinv32);
    }
    PLATO_LAUNCH_CHECK(h);
    return PLATO_OK;
}

int launch_sell_scale16(plato_problem* h, const double* sell64, const double* dinv, void* out16, float* sq,
                        float* isq, float* ones) {
    const SellPattern& P = h->sell;
    const int64_t n = 3 * int64_t(h->N);
    k_scale_vectors<<<grid_for(n, 256), 256, 0, h->stream>>>(n, dinv, sq, isq, ones);
    PLATO_LAUNCH_CHECK(h);
    k_sell_scale16<<<grid_for(int64_t(P.nslices) * 32, 256, 148 * 16), 256, 0, h->stream>>>(
        h->N, P.nslices, P.width, P.ptr, P.cols, sell64, isq, static_cast<__half*>(out16));
    PLATO_LAUNCH_CHECK(h);
    return PLATO_OK;
}

}  // namespace plato
