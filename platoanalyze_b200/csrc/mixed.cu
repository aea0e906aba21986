// Flexible CG in FP64 with a Chebyshev-Jacobi polynomial preconditioner applied in low
// precision (the mixed-precision solve of PLATO_PRECISION_MIXED_FP32 / _MIXED_BF16, and the
// FP64 polynomial-preconditioned variant).
//
// Outer method: flexible conjugate gradients with one-term A-orthogonalisation (Notay's
// FCG(1)): q = A p, alpha = (p.r)/(p.q), x += alpha p, r -= alpha q, z = M(r),
// beta = -(z.q)/(p.q), p = z + beta p.  Operator applications, the residual, the iterate,
// every dot product and step length are FP64; the stop test ||r|| <= tol ||b|| is FP64 and
// is confirmed on exit with the recomputed residual b - A x.
//
// Preconditioner M: `degree` steps of the Chebyshev iteration for D^-1 A on the interval
// [lambda_max / ratio, lambda_max] from a zero initial guess (Saad, Iterative Methods for
// Sparse Linear Systems, 2nd ed., Alg. 12.1), run on an FP32 (or BF16-stored, or
// matrix-free FP32) copy of the operator with FP32 vectors.  Only the preconditioner sees
// reduced precision, so it changes the iteration count, not the converged answer.
// lambda_max comes from a few Lanczos steps with a safety factor.
//
// Each Chebyshev step on the SELL copy is one fused kernel (gather SpMV, residual update,
// direction and iterate update; no reductions).  The matrix-free variant scatters with
// FP32 atomics and finishes the step in a vector kernel.
#include <algorithm>
#include <cmath>
#include <cuda_bf16.h>

#include <cuda_fp16.h>

#include "plato_internal.cuh"
#include "solver_common.cuh"

namespace plato {

int launch_assemble_sell(plato_problem* h, const double* z, double* v64, float* v32, void* v16, double* dinv,
                         float* dinv32);
int launch_assemble_sell32(plato_problem* h, const double* z, float* v32, float* dinv32);

int launch_axpby(plato_problem* h, int64_t n, double a, const double* x, double b, double* y);
int launch_dot(plato_problem* h, const double* a, const double* b, int64_t n, double* host_result);
int launch_crs_to_sell(plato_problem* h, const double* crs, double* out64, float* out32, void* out16,
                       double* dinv, float* dinv32);
int launch_sell_scale16(plato_problem* h, const double* sell64, const double* dinv, void* out16, float* sq,
                        float* isq, float* ones);
int launch_sell_spmv(plato_problem* h, const double* vals, const double* x, double* y);
int launch_ebe_apply64(plato_problem* h, const double* x, double* y, const PcgScalars* S);
int launch_ebe_apply32(plato_problem* h, const float* x, float* y, const PcgScalars* S);
int launch_mask_copy(plato_problem* h, const double* x, double* y);
int matfree_setup(plato_problem* h, const double* z);
SellView sell_view(const plato_problem* h);
int spmv_blocks(const plato_problem* h);
int timing_events(plato_problem* h, cudaEvent_t* e0, cudaEvent_t* e1);
int collect_timing(plato_problem* h, const std::vector<int64_t>& iters, int64_t executed);

namespace {

constexpr int kChunk = 16;
constexpr int kTimingStride = 8;
constexpr int kMaxRestarts = 8;  // restarts from the true residual (see the plain PCG)

enum InnerKind { INNER_SELL64 = 0, INNER_SELL32 = 1, INNER_SELL16 = 2, INNER_EBE32 = 3, INNER_EBE64 = 4,
                 INNER_SELL16S = 5 };

struct ChebCoef {
    float c0;      // first step: d = c0 Dinv r
    float c1[64];  // step k: d_k = c1[k] d_(k-1) + c2[k] Dinv res
    float c2[64];
};

// ---- outer operator: q = A p, then p.q -> alpha = (p.r)/(p.q) ------------------------------

__device__ __forceinline__ void finish_pq(PcgScalars* S, double pq) {
    S->pAp = pq;
    S->alpha = S->rz / pq;
    if (!isfinite(S->alpha) || pq <= 0.0) { S->nonfinite = 1; S->done = 1; }
}

__global__ void __launch_bounds__(kThreads)
k_fcg_sell_apply(SellView A, const double* __restrict__ vals, const double* __restrict__ p, double* __restrict__ q,
                 PcgScalars* S, double* partials) {
    __shared__ double sh[1][32];
    __shared__ bool last;
    pdl_wait();
    pdl_trigger();
    if (S->done) return;
    double dot = 0.0;
    const int64_t padded = ((int64_t)A.num_rows + 31) & ~int64_t(31);
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < padded; r += (int64_t)gridDim.x * blockDim.x) {
        double a0, a1, a2;
        sell_row<double>(A, vals, p, r, a0, a1, a2);
        if (r < A.num_rows) {
            q[3 * r] = a0;
            q[3 * r + 1] = a1;
            q[3 * r + 2] = a2;
            dot += p[3 * r] * a0 + p[3 * r + 1] * a1 + p[3 * r + 2] * a2;
        }
    }
    double v[1] = {dot};
    block_sum_n<1>(v, sh);
    if (publish_partials<1>(v, partials, &S->ticket, &last)) {
        double t[1];
        final_sums<1>(t, partials, sh);
        if (threadIdx.x == 0) {
            finish_pq(S, t[0]);
            S->ticket = 0u;
        }
    }
}

// After a matrix-free apply: constrained rows of q take p (identity rows), then p.q.
__global__ void __launch_bounds__(kThreads)
k_fcg_mask_dot(int64_t n, const uint8_t* __restrict__ mask, const double* __restrict__ p, double* __restrict__ q,
               PcgScalars* S, double* partials) {
    __shared__ double sh[1][32];
    __shared__ bool last;
    if (S->done) return;
    double v[1] = {0.0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double qi = q[i];
        if (mask[i]) { qi = p[i]; q[i] = qi; }
        v[0] += p[i] * qi;
    }
    block_sum_n<1>(v, sh);
    if (publish_partials<1>(v, partials, &S->ticket, &last)) {
        double t[1];
        final_sums<1>(t, partials, sh);
        if (threadIdx.x == 0) {
            finish_pq(S, t[0]);
            S->ticket = 0u;
        }
    }
}

// x += alpha p; r -= alpha q; r.r and the stop test; starts the preconditioner:
// res = r (FP32), d = c0 Dinv r, y = d.
__global__ void __launch_bounds__(kThreads)
k_fcg_update(int64_t n, double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
             const double* __restrict__ q, const float* __restrict__ dinv32, const float* __restrict__ res_scale,
             float* __restrict__ res, float* __restrict__ d, float* __restrict__ y, float c0, PcgScalars* S,
             double* partials, int32_t max_it) {
    __shared__ double sh[1][32];
    __shared__ bool last;
    pdl_wait();
    pdl_trigger();
    if (S->done) return;
    const double alpha = S->alpha;
    double v[1] = {0.0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        x[i] += alpha * p[i];
        const double ri = r[i] - alpha * q[i];
        r[i] = ri;
        v[0] += ri * ri;
        const float rf = res_scale ? res_scale[i] * float(ri) : float(ri);
        const float di = c0 * dinv32[i] * rf;
        res[i] = rf;
        d[i] = di;
        y[i] = di;
    }
    block_sum_n<1>(v, sh);
    if (publish_partials<1>(v, partials, &S->ticket, &last)) {
        double t[1];
        final_sums<1>(t, partials, sh);
        if (threadIdx.x == 0) {
            S->rr = t[0];
            S->iter += 1;
            if (!isfinite(t[0])) { S->nonfinite = 1; S->done = 1; }
            if (t[0] <= S->tol2 || S->iter >= max_it) S->done = 1;
            S->ticket = 0u;
        }
    }
}

// One Chebyshev step on a SELL copy (entries TV): w = A d_cur, res -= w,
// d_next = c1 d_cur + c2 Dinv res, y += d_next.
template <int KIND>
__global__ void __launch_bounds__(kThreads)
k_cheb_sell(SellView A, const void* __restrict__ vals, const float* __restrict__ dinv32, float* __restrict__ res,
            const float* __restrict__ dcur, float* __restrict__ dnext, float* __restrict__ y, float c1, float c2,
            const PcgScalars* S) {
    if (S->done) return;
    const int64_t padded = ((int64_t)A.num_rows + 31) & ~int64_t(31);
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < padded; r += (int64_t)gridDim.x * blockDim.x) {
        float w0, w1, w2;
        if (KIND == INNER_SELL16)
            sell_row_bf16(A, static_cast<const __nv_bfloat16*>(vals), dcur, r, w0, w1, w2);
        else if (KIND == INNER_SELL32)
            sell_row<float>(A, static_cast<const float*>(vals), dcur, r, w0, w1, w2);
        else {
            double a0, a1, a2;
            sell_row<double>(A, static_cast<const double*>(vals), dcur, r, a0, a1, a2);
            w0 = float(a0); w1 = float(a1); w2 = float(a2);
        }
        if (r < A.num_rows) {
            const float w[3] = {w0, w1, w2};
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const int64_t k = 3 * r + i;
                const float rs = res[k] - w[i];
                res[k] = rs;
                const float dn = c1 * dcur[k] + c2 * dinv32[k] * rs;
                dnext[k] = dn;
                y[k] += dn;
            }
        }
    }
}

// FP16 Jacobi-scaled matrix (INNER_SELL16S), two rows per thread: rows 2m and 2m+1 of a
// slice share each (k, q) entry pair as one __half2 and their column indices as one int2,
// so a thread loads 4 bytes per entry load (2-byte loads would halve the bytes in flight of
// this latency-bound loop).  Entry (k, q) of the pair at (9 ptr_s) / 2 + 16 (9k + q) + m.
// kShort: the pair's two column indices come as 16-bit offsets from the slice's first row
// (one 4-byte load instead of 8; 20 instead of 22 bytes per block pair entry).
// kConstX: x is read-only for the whole kernel (read through the non-coherent path); the
// multi-step sweep reads directions written by other CTAs of the same launch with plain
// loads instead, ordered after its acquire of their completion flags.
template <bool kShort, bool kConstX>
__device__ __forceinline__ void sell16s_pair(const SellView& A, const __half* __restrict__ vals, const float* x,
                                             int64_t pr, float (&wv)[6]) {
    const int64_t sl = pr >> 4;
    const int m = int(pr & 15);
    const int w = __ldg(A.width + sl);
    const int64_t base = __ldg(A.ptr + sl);
    const int2* __restrict__ cp = reinterpret_cast<const int2*>(A.cols + base) + m;
    const short2* __restrict__ dp = reinterpret_cast<const short2*>(A.dcols + base) + m;
    const int32_t row0 = int32_t(32 * sl);
    const __half2* __restrict__ vp = reinterpret_cast<const __half2*>(vals + 9 * base) + m;
    float a0 = 0.f, a1 = 0.f, a2 = 0.f, b0 = 0.f, b1 = 0.f, b2 = 0.f;
#pragma unroll 4
    for (int k = 0; k < w; ++k) {
        int2 c;
        if (kShort) {
            const short2 d = __ldg(dp + 16 * k);
            c = make_int2(row0 + d.x, row0 + d.y);
        } else {
            c = __ldg(cp + 16 * k);
        }
        const float* xa = x + 3 * (int64_t)c.x;
        const float* xb = x + 3 * (int64_t)c.y;
        const float x0 = kConstX ? __ldg(xa) : xa[0], x1 = kConstX ? __ldg(xa + 1) : xa[1],
                    x2 = kConstX ? __ldg(xa + 2) : xa[2];
        const float z0 = kConstX ? __ldg(xb) : xb[0], z1 = kConstX ? __ldg(xb + 1) : xb[1],
                    z2 = kConstX ? __ldg(xb + 2) : xb[2];
        const __half2* vk = vp + 144 * k;
        float2 e[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) e[q] = __half22float2(vk[16 * q]);
        a0 += e[0].x * x0 + e[1].x * x1 + e[2].x * x2;
        a1 += e[3].x * x0 + e[4].x * x1 + e[5].x * x2;
        a2 += e[6].x * x0 + e[7].x * x1 + e[8].x * x2;
        b0 += e[0].y * z0 + e[1].y * z1 + e[2].y * z2;
        b1 += e[3].y * z0 + e[4].y * z1 + e[5].y * z2;
        b2 += e[6].y * z0 + e[7].y * z1 + e[8].y * z2;
    }
    wv[0] = a0; wv[1] = a1; wv[2] = a2; wv[3] = b0; wv[4] = b1; wv[5] = b2;
}

// The pair's vector update after w = A^ x.  MODE 0: Chebyshev step in scaled variables (unit
// diagonal): res -= w, d_next = c1 x + c2 res, y += d_next;  MODE 1: res -= w;  MODE 2: y = w.
template <int MODE>
__device__ __forceinline__ void sell16s_update(int64_t num_rows, int64_t pr, const float (&wv)[6],
                                               const float* __restrict__ x, float* __restrict__ res,
                                               float* __restrict__ dnext, float* __restrict__ y, float c1, float c2,
                                               bool vec2) {
    const int64_t r0 = 32 * (pr >> 4) + 2 * (pr & 15);
    // both rows of the pair: their 6 entries start at 3 r0 = 6 (16 sl + m), 8-byte aligned
    // when the vectors are, so the update runs on float2 (half the memory instructions)
    if (MODE != 2 && vec2 && r0 + 1 < num_rows) {
        float2* rp = reinterpret_cast<float2*>(res + 3 * r0);
#pragma unroll
        for (int u = 0; u < 3; ++u) {
            const float2 rr = rp[u];
            const float rs0 = rr.x - wv[2 * u], rs1 = rr.y - wv[2 * u + 1];
            rp[u] = make_float2(rs0, rs1);
            if (MODE == 0) {
                const float2 xx = reinterpret_cast<const float2*>(x + 3 * r0)[u];
                float2* yp = reinterpret_cast<float2*>(y + 3 * r0) + u;
                const float2 yy = *yp;
                const float d0 = c1 * xx.x + c2 * rs0, d1 = c1 * xx.y + c2 * rs1;
                reinterpret_cast<float2*>(dnext + 3 * r0)[u] = make_float2(d0, d1);
                *yp = make_float2(yy.x + d0, yy.y + d1);
            }
        }
        return;
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        if (r0 + h >= num_rows) break;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const int64_t k = 3 * (r0 + h) + i;
            const float wi = wv[3 * h + i];
            if (MODE == 0) {
                const float rs = res[k] - wi;
                res[k] = rs;
                const float dn = c1 * x[k] + c2 * rs;
                dnext[k] = dn;
                y[k] += dn;
            } else if (MODE == 1) {
                res[k] -= wi;
            } else {
                y[k] = wi;
            }
        }
    }
}

// One application of the FP16 scaled matrix per launch (sell16s_pair + sell16s_update).
template <int MODE, bool kShort>
__global__ void __launch_bounds__(kThreads, 4)
k_sell16s(SellView A, const __half* __restrict__ vals, const float* __restrict__ x, float* __restrict__ res,
          float* __restrict__ dnext, float* __restrict__ y, float c1, float c2, const PcgScalars* S) {
    pdl_wait();
    pdl_trigger();
    if (S && S->done) return;
    const int64_t npairs = (((int64_t)A.num_rows + 31) & ~int64_t(31)) >> 1;
    const uintptr_t vbits = reinterpret_cast<uintptr_t>(res) |
                            (MODE == 0 ? reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(dnext) |
                                             reinterpret_cast<uintptr_t>(y)
                                       : uintptr_t(0));
    const bool vec2 = (vbits & 7) == 0;
    for (int64_t pr = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; pr < npairs;
         pr += (int64_t)gridDim.x * blockDim.x) {
        float wv[6];
        sell16s_pair<kShort, true>(A, vals, x, pr, wv);
        sell16s_update<MODE>(A.num_rows, pr, wv, x, res, dnext, y, c1, c2, vec2);
    }
}

// Staged form of k_sell16s (16-bit column offsets): each warp covers two slices (lanes 0-15
// and 16-31, two rows per lane as above) and streams their FP16 entries and column offsets
// through shared memory in chunks of kStK slots: cp.async copies chunk c + 1 (16-byte pieces;
// a slice's slots are contiguous, 576 B of entries and 64 B of offsets per slot) while the lanes
// compute chunk c from shared memory.  The direction gathers then wait only on L2 (the offsets
// are already on chip) instead of on a DRAM round trip followed by an L2 round trip.
// Measured on the 160x80x80 bench mesh (sweep launch): 74.4 us with 2 slots x 2 stages (43 KB
// per CTA, 4 CTAs per SM), 77.2 us with 3 stages (3 CTAs per SM), 79.0 us with 4 slots x 2
// stages (2 CTAs per SM), 77.1 us with 1 slot x 3 stages, 78.7 us with 5 CTAs per SM (launch
// bound 5; 78.4 us with 1 slot x 3 stages), 80.3 us for the register-fed k_sell16s.
constexpr int kStK = 2;       // slots per chunk
constexpr int kStStages = 2;  // chunks in the ring (kStStages - 1 in flight)
// one slice's chunk: entries, then offsets; padded by 64 B so that the two half-warps' regions
// start 16 banks apart
constexpr int kStHalfBytes = kStK * (576 + 64) + 64;
constexpr int kStWarpBytes = kStStages * 2 * kStHalfBytes;
constexpr int kStSmem = (kThreads / 32) * kStWarpBytes;

__device__ __forceinline__ void sweep_cp16(uint32_t dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}

template <int MODE>
__global__ void __launch_bounds__(kThreads, 4)
k_sell16s_st(SellView A, const __half* __restrict__ vals, const float* __restrict__ x, float* __restrict__ res,
             float* __restrict__ dnext, float* __restrict__ y, float c1, float c2, const PcgScalars* S) {
    extern __shared__ __align__(16) uint8_t st_smem[];
    pdl_wait();
    pdl_trigger();
    if (S && S->done) return;
    const int64_t npairs = (((int64_t)A.num_rows + 31) & ~int64_t(31)) >> 1;
    const uintptr_t vbits = reinterpret_cast<uintptr_t>(res) |
                            (MODE == 0 ? reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(dnext) |
                                             reinterpret_cast<uintptr_t>(y)
                                       : uintptr_t(0));
    const bool vec2 = (vbits & 7) == 0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, half = lane >> 4, m = lane & 15;
    const uint8_t* wsm = st_smem + warp * kStWarpBytes;
    const uint32_t wsm_s = static_cast<uint32_t>(__cvta_generic_to_shared(wsm));
    // a warp's 32 pairs are 32 consecutive pairs starting at a multiple of 32: two whole slices
    for (int64_t pb = blockIdx.x * (int64_t)blockDim.x + 32 * warp; pb < npairs;
         pb += (int64_t)gridDim.x * blockDim.x) {
        const int64_t pr = pb + lane;
        const bool active = pr < npairs;  // npairs is a multiple of 16: half-warps are all or none
        const int64_t sl = pr >> 4;
        int w = 0;
        int64_t base = 0;
        if (active) {
            w = __ldg(A.width + sl);
            base = __ldg(A.ptr + sl);
        }
        int wmax = w;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) wmax = max(wmax, __shfl_xor_sync(0xffffffffu, wmax, o));
        const int nch = (wmax + kStK - 1) / kStK;
        const uint8_t* gv = reinterpret_cast<const uint8_t*>(vals + 9 * base);  // 576 B per slot
        const uint8_t* gc = reinterpret_cast<const uint8_t*>(A.dcols + base);  // 64 B per slot
        // chunk c of this half-warp's slice into ring stage stg (nothing past the slice's width)
        auto copy = [&](int c, int stg) {
            const int k0 = c * kStK, kn = min(kStK, w - k0);
            if (kn > 0) {
                const uint32_t dst = wsm_s + uint32_t((stg * 2 + half) * kStHalfBytes);
                for (int u = m; u < kn * 36; u += 16) sweep_cp16(dst + 16u * u, gv + 576 * int64_t(k0) + 16 * u);
                for (int u = m; u < kn * 4; u += 16)
                    sweep_cp16(dst + uint32_t(kStK * 576) + 16u * u, gc + 64 * int64_t(k0) + 16 * u);
            }
        };
        const int32_t row0 = int32_t(32 * sl);
        float a0 = 0.f, a1 = 0.f, a2 = 0.f, b0 = 0.f, b1 = 0.f, b2 = 0.f;
#pragma unroll
        for (int c = 0; c < kStStages - 1; ++c) {
            if (c < nch) copy(c, c);
            asm volatile("cp.async.commit_group;" ::: "memory");
        }
        for (int c = 0; c < nch; ++c) {
            if (c + kStStages - 1 < nch) copy(c + kStStages - 1, (c + kStStages - 1) % kStStages);
            asm volatile("cp.async.commit_group;" ::: "memory");
            asm volatile("cp.async.wait_group %0;" ::"n"(kStStages - 1) : "memory");  // chunk c is in
            __syncwarp();
            const uint8_t* sv = wsm + ((c % kStStages) * 2 + half) * kStHalfBytes;
            const __half2* sh = reinterpret_cast<const __half2*>(sv) + m;
            const short2* sd = reinterpret_cast<const short2*>(sv + kStK * 576) + m;
#pragma unroll
            for (int kk = 0; kk < kStK; ++kk) {
                if (c * kStK + kk < w) {
                    const short2 d = sd[16 * kk];
                    const float* xa = x + 3 * (int64_t)(row0 + d.x);
                    const float* xb = x + 3 * (int64_t)(row0 + d.y);
                    const float x0 = __ldg(xa), x1 = __ldg(xa + 1), x2 = __ldg(xa + 2);
                    const float z0 = __ldg(xb), z1 = __ldg(xb + 1), z2 = __ldg(xb + 2);
                    float2 e[9];
#pragma unroll
                    for (int q = 0; q < 9; ++q) e[q] = __half22float2(sh[144 * kk + 16 * q]);
                    a0 += e[0].x * x0 + e[1].x * x1 + e[2].x * x2;
                    a1 += e[3].x * x0 + e[4].x * x1 + e[5].x * x2;
                    a2 += e[6].x * x0 + e[7].x * x1 + e[8].x * x2;
                    b0 += e[0].y * z0 + e[1].y * z1 + e[2].y * z2;
                    b1 += e[3].y * z0 + e[4].y * z1 + e[5].y * z2;
                    b2 += e[6].y * z0 + e[7].y * z1 + e[8].y * z2;
                }
            }
            __syncwarp();  // every lane has read stage c before a later copy refills it
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
        if (active) {
            const float wv[6] = {a0, a1, a2, b0, b1, b2};
            sell16s_update<MODE>(A.num_rows, pr, wv, x, res, dnext, y, c1, c2, vec2);
        }
    }
}

// ---- multi-step sweep: several Chebyshev steps per launch, the matrix re-read from L2 ------
//
// Step g of a preconditioner call reads the whole FP16 matrix (280 MB on the 160x80x80 mesh)
// to apply it to d_(g-1).  A row of step g needs d_(g-1) only at its columns, which lie within
// the row's tile +- `halo` tiles (tiles of kWaveRows consecutive rows; halo from the mesh's
// numbering, 14 tiles of 512 rows on the bench mesh), so step g can start on a tile as soon as
// step g-1 has finished that neighbourhood.  One launch runs `nsteps` consecutive steps as
// tasks (step, tile) issued in the order of tile + lag * step (lag = halo + 1 + slack): step g
// trails step g-1 by `lag` tiles, so the rows a step reads were read by the step before a few
// tens of MB earlier and are still in the 126 MB L2 -- the matrix comes from HBM once per
// launch instead of once per step.  Each CTA takes the next task from a ticket counter (only
// running CTAs take tickets, and every task depends only on tasks issued before it, so the
// launch cannot deadlock whatever the residency), waits until the completion stamps of its
// dependencies -- step g-1 on tiles t-halo..t+halo -- carry this launch's epoch (acquire:
// the SM's L1 holds no stale line of the direction vector after it), runs the same row-pair
// arithmetic as k_sell16s, and stamps its own completion (release).  d_g alternates between
// two buffers: step g overwrites d_(g-2) on tile t only after step g-1 finished every tile
// that reads it.  Every wait is bounded: after kWavePolls polls the CTA raises `abort`, the
// others stop taking tasks and stop waiting, the launch ends, and `fail` stays set for the
// host.  The last CTA to leave resets the ticket counters for the next launch.
constexpr int kWaveRows = 2 * kThreads;  // rows per tile: one row pair per thread
constexpr int kWaveMaxSteps = 16;        // steps per launch
constexpr uint32_t kWavePolls = 1u << 21;

struct WaveCtl {
    uint32_t ticket;  // next task
    uint32_t exits;   // CTAs that left the task loop
    int32_t  abort;   // a wait ran out during this launch
    int32_t  fail;    // sticky for the host: some launch aborted
};

struct WaveStep {
    float c1[kWaveMaxSteps], c2[kWaveMaxSteps];
    int32_t first;     // global step number of local step 0 (d_(first-1) is the launch's input)
    int32_t nsteps;    // steps in this launch
    int32_t nupdate;   // local steps < nupdate are Chebyshev steps, the rest residual-only (MODE 1)
};

__device__ __forceinline__ int32_t ld_acquire_s32(const int32_t* p) {
    int32_t v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_s32(int32_t* p, int32_t v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

template <bool kShort>
__global__ void __launch_bounds__(kThreads, 4)
k_sell16s_wave(SellView A, const __half* __restrict__ vals, float* __restrict__ res, float* d_even, float* d_odd,
               float* __restrict__ y, WaveStep st, const int32_t* __restrict__ order, int32_t ntasks, int32_t ntiles,
               int32_t halo, int32_t epoch, int32_t wait_epoch, int32_t* flags, WaveCtl* ctl,
               const PcgScalars* S) {
    if (S && S->done) return;
    __shared__ uint32_t sh_task, sh_next;
    const int64_t npairs = (((int64_t)A.num_rows + 31) & ~int64_t(31)) >> 1;
    const uintptr_t vbits = reinterpret_cast<uintptr_t>(res) | reinterpret_cast<uintptr_t>(d_even) |
                            reinterpret_cast<uintptr_t>(d_odd) | reinterpret_cast<uintptr_t>(y);
    const bool vec2 = (vbits & 7) == 0;
    if (threadIdx.x == 0) sh_next = atomicAdd(&ctl->ticket, 1u);
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) {
            sh_task = sh_next;  // take the next ticket now, so its latency hides behind this task
            const bool stop = sh_task >= uint32_t(ntasks) || *reinterpret_cast<volatile int32_t*>(&ctl->abort);
            sh_next = stop ? uint32_t(ntasks) : atomicAdd(&ctl->ticket, 1u);
            if (stop) sh_task = uint32_t(ntasks);
        }
        __syncthreads();
        const uint32_t task = sh_task;
        if (task >= uint32_t(ntasks)) break;
        const int32_t code = __ldg(order + task);
        const int j = code >> 24, t = code & 0xFFFFFF;  // local step, tile
        if (j > 0) {
            // step j-1 finished on tiles t-halo .. t+halo (a thread per tile)
            int ok = 1;
            for (int q = max(0, t - halo) + int(threadIdx.x); ok && q <= min(ntiles - 1, t + halo);
                 q += blockDim.x) {
                const int32_t* f = flags + (int64_t)(j - 1) * ntiles + q;
                uint32_t polls = 0;
                while (ld_acquire_s32(f) < wait_epoch) {
                    if (++polls > kWavePolls || *reinterpret_cast<volatile int32_t*>(&ctl->abort)) {
                        ok = 0;
                        break;
                    }
                    __nanosleep(128);
                }
            }
            if (!__syncthreads_and(ok)) {
                if (threadIdx.x == 0) atomicExch(&ctl->abort, 1);
                break;
            }
        }
        const int g = st.first + j;  // global step: reads d_(g-1), writes d_g
        const float* x = ((g - 1) & 1) ? d_odd : d_even;
        float* dn = (g & 1) ? d_odd : d_even;
        const int64_t pr = (int64_t)t * kThreads + threadIdx.x;
        if (pr < npairs) {
            float wv[6];
            if (kShort) sell16s_pair<true, false>(A, vals, x, pr, wv);
            else sell16s_pair<false, false>(A, vals, x, pr, wv);
            if (j < st.nupdate)
                sell16s_update<0>(A.num_rows, pr, wv, x, res, dn, y, st.c1[j], st.c2[j], vec2);
            else
                sell16s_update<1>(A.num_rows, pr, wv, x, res, nullptr, nullptr, 0.f, 0.f, vec2);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            st_release_s32(flags + (int64_t)j * ntiles + t, epoch);
        }
    }
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&ctl->exits, 1u) == gridDim.x - 1) {
            if (ctl->abort) ctl->fail = 1;
            ctl->abort = 0;
            ctl->ticket = 0u;
            ctl->exits = 0u;
            __threadfence();
        }
    }
}

// Largest distance in tiles between a row and one of its columns (padding lanes excluded).
__global__ void k_wave_halo(SellView A, int32_t* __restrict__ out) {
    int32_t m = 0;
    const int32_t nslices = (A.num_rows + 31) >> 5;
    for (int64_t sl = blockIdx.x; sl < nslices; sl += gridDim.x) {
        const int64_t base = A.ptr[sl];
        const int w = A.width[sl];
        for (int e = threadIdx.x; e < 32 * w; e += blockDim.x) {
            const int32_t r = int32_t(32 * sl + (e & 31));
            if (r >= A.num_rows) continue;
            const int32_t c = A.cols[base + e];
            const int32_t d = abs(c / kWaveRows - r / kWaveRows);
            m = max(m, d);
        }
    }
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// Chebyshev step after a matrix-free apply (w holds P A P d_cur; constrained rows are identity).
__global__ void __launch_bounds__(kThreads)
k_cheb_vec(int64_t n, const uint8_t* __restrict__ mask, const float* __restrict__ w, const float* __restrict__ dinv32,
           float* __restrict__ res, const float* __restrict__ dcur, float* __restrict__ dnext, float* __restrict__ y,
           float c1, float c2, const PcgScalars* S) {
    if (S->done) return;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float wi = mask[i] ? dcur[i] : w[i];
        const float rs = res[i] - wi;
        res[i] = rs;
        const float dn = c1 * dcur[i] + c2 * dinv32[i] * rs;
        dnext[i] = dn;
        y[i] += dn;
    }
}

// res -= A x on a SELL copy (FP32 vectors).
template <int KIND>
__global__ void __launch_bounds__(kThreads)
k_res_sub_sell(SellView A, const void* __restrict__ vals, const float* __restrict__ x, float* __restrict__ res,
               const PcgScalars* S) {
    if (S->done) return;
    const int64_t padded = ((int64_t)A.num_rows + 31) & ~int64_t(31);
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < padded; r += (int64_t)gridDim.x * blockDim.x) {
        float w0, w1, w2;
        if (KIND == INNER_SELL16)
            sell_row_bf16(A, static_cast<const __nv_bfloat16*>(vals), x, r, w0, w1, w2);
        else if (KIND == INNER_SELL32)
            sell_row<float>(A, static_cast<const float*>(vals), x, r, w0, w1, w2);
        else {
            double a0, a1, a2;
            sell_row<double>(A, static_cast<const double*>(vals), x, r, a0, a1, a2);
            w0 = float(a0); w1 = float(a1); w2 = float(a2);
        }
        if (r < A.num_rows) {
            res[3 * r] -= w0;
            res[3 * r + 1] -= w1;
            res[3 * r + 2] -= w2;
        }
    }
}

// res -= P A P x + (I - P) x after a matrix-free apply into w.
__global__ void __launch_bounds__(kThreads)
k_res_sub_vec(int64_t n, const uint8_t* __restrict__ mask, const float* __restrict__ x, const float* __restrict__ w,
              float* __restrict__ res, const PcgScalars* S) {
    if (S->done) return;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        res[i] -= mask[i] ? x[i] : w[i];
}

// z = y (widened; times z_scale when the preconditioner ran in scaled variables), z.q ->
// beta = -(z.q)/(p.q); then p = z + beta p and p.r in k_fcg_direction.
__global__ void __launch_bounds__(kThreads)
k_fcg_zq(int64_t n, const float* __restrict__ y, const float* __restrict__ z_scale, double* __restrict__ z,
         const double* __restrict__ q, PcgScalars* S, double* partials, int first) {
    __shared__ double sh[1][32];
    __shared__ bool last;
    pdl_wait();
    pdl_trigger();
    if (S->done) return;
    if (first) {  // initial direction: only widen z = y
        for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
            z[i] = double(z_scale ? z_scale[i] * y[i] : y[i]);
        return;
    }
    double v[1] = {0.0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double zi = double(z_scale ? z_scale[i] * y[i] : y[i]);
        z[i] = zi;
        v[0] += zi * q[i];
    }
    block_sum_n<1>(v, sh);
    if (publish_partials<1>(v, partials, &S->ticket, &last)) {
        double t[1];
        final_sums<1>(t, partials, sh);
        if (threadIdx.x == 0) {
            S->zq = t[0];
            S->beta = -t[0] / S->pAp;
            if (!isfinite(S->beta)) { S->nonfinite = 1; S->done = 1; }
            S->ticket = 0u;
        }
    }
}

__global__ void __launch_bounds__(kThreads)
k_fcg_direction(int64_t n, const double* __restrict__ z, double* __restrict__ p, const double* __restrict__ r,
                PcgScalars* S, double* partials, int first) {
    __shared__ double sh[1][32];
    __shared__ bool last;
    pdl_wait();
    pdl_trigger();
    if (S->done) return;
    const double beta = first ? 0.0 : S->beta;
    double v[1] = {0.0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double pi = z[i] + beta * (first ? 0.0 : p[i]);
        p[i] = pi;
        v[0] += pi * r[i];
    }
    block_sum_n<1>(v, sh);
    if (publish_partials<1>(v, partials, &S->ticket, &last)) {
        double t[1];
        final_sums<1>(t, partials, sh);
        if (threadIdx.x == 0) {
            S->rz = t[0];  // p.r
            if (!isfinite(t[0])) { S->nonfinite = 1; S->done = 1; }
            S->ticket = 0u;
        }
    }
}

// r = b - A x (A x in r on entry), r.r and b.b; starts the preconditioner like k_fcg_update.
__global__ void __launch_bounds__(kThreads)
k_fcg_start(int64_t n, const double* __restrict__ b, double* __restrict__ r, const float* __restrict__ dinv32,
            const float* __restrict__ res_scale, float* __restrict__ res, float* __restrict__ d, float* __restrict__ y,
            float c0, PcgScalars* S, double* partials, double tol, int keep_bb) {
    __shared__ double sh[2][32];
    __shared__ bool last;
    double v[2] = {0.0, 0.0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double ri = b[i] - r[i];
        r[i] = ri;
        v[0] += ri * ri;
        v[1] += b[i] * b[i];
        const float rf = res_scale ? res_scale[i] * float(ri) : float(ri);
        const float di = c0 * dinv32[i] * rf;
        res[i] = rf;
        d[i] = di;
        y[i] = di;
    }
    block_sum_n<2>(v, sh);
    if (publish_partials<2>(v, partials, &S->ticket, &last)) {
        double t[2];
        final_sums<2>(t, partials, sh);
        if (threadIdx.x == 0) {
            S->rr = t[0];
            if (!keep_bb) {
                S->bb = t[1];
                S->tol2 = tol * tol * t[1];
                S->iter = 0;
            }
            S->nonfinite = (!isfinite(t[0]) || !isfinite(t[1])) ? 1 : 0;
            S->done = (t[0] <= S->tol2 || S->nonfinite) ? 1 : 0;
            S->ticket = 0u;
        }
    }
}

__global__ void k_power_init(int64_t n, float* __restrict__ v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        uint32_t h = uint32_t(i) * 2654435761u;
        h ^= h >> 15;
        h *= 2246822519u;
        h ^= h >> 13;
        v[i] = float(h & 0xffffff) / float(0x1000000) + 0.5f;
    }
}

int inner_kind(const plato_problem* h) {
    const plato_solver_opts& o = h->opts;
    if (o.operator_kind == PLATO_OPERATOR_MATRIX_FREE) {
        if (o.precision == PLATO_PRECISION_MIXED_FP32_ASSEMBLED) return INNER_SELL32;  // FP32 element assembly
        return o.precision == PLATO_PRECISION_FP64 ? INNER_EBE64 : INNER_EBE32;
    }
    if (o.precision == PLATO_PRECISION_MIXED_BF16) return INNER_SELL16;
    if (o.precision == PLATO_PRECISION_MIXED_FP16) return INNER_SELL16S;
    if (o.precision == PLATO_PRECISION_MIXED_FP32) return INNER_SELL32;
    return INNER_SELL64;
}

}  // namespace

// Inner SELL product for the Lanczos estimate (plain w = A d, FP32 out).
namespace {
template <int KIND>
__global__ void __launch_bounds__(kThreads)
k_sell_apply32(SellView A, const void* __restrict__ vals, const float* __restrict__ x, float* __restrict__ y) {
    const int64_t padded = ((int64_t)A.num_rows + 31) & ~int64_t(31);
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < padded; r += (int64_t)gridDim.x * blockDim.x) {
        float w0, w1, w2;
        if (KIND == INNER_SELL16)
            sell_row_bf16(A, static_cast<const __nv_bfloat16*>(vals), x, r, w0, w1, w2);
        else if (KIND == INNER_SELL32)
            sell_row<float>(A, static_cast<const float*>(vals), x, r, w0, w1, w2);
        else {
            double a0, a1, a2;
            sell_row<double>(A, static_cast<const double*>(vals), x, r, a0, a1, a2);
            w0 = float(a0); w1 = float(a1); w2 = float(a2);
        }
        if (r < A.num_rows) {
            y[3 * r] = w0;
            y[3 * r + 1] = w1;
            y[3 * r + 2] = w2;
        }
    }
}
}  // namespace

static const void* inner_vals(const plato_problem* h, int kind) {
    if (kind == INNER_SELL16S) return h->sell16s;
    if (kind == INNER_SELL16) return h->sell16;
    if (kind == INNER_SELL32) return h->sell32;
    return h->sell64;
}

static int apply_inner_plain(plato_problem* h, int kind, const float* x, float* y) {
    if (kind == INNER_EBE32 || kind == INNER_EBE64) return launch_ebe_apply32(h, x, y, nullptr);
    const SellView V = sell_view(h);
    const void* vals = inner_vals(h, kind);
    const int B = spmv_blocks(h);
    if (kind == INNER_SELL16S)
        if (V.dcols)
            k_sell16s<2, true><<<B, kThreads, 0, h->stream>>>(V, static_cast<const __half*>(vals), x, nullptr, nullptr,
                                                              y, 0.f, 0.f, nullptr);
        else
            k_sell16s<2, false><<<B, kThreads, 0, h->stream>>>(V, static_cast<const __half*>(vals), x, nullptr, nullptr,
                                                               y, 0.f, 0.f, nullptr);
    else if (kind == INNER_SELL16) k_sell_apply32<INNER_SELL16><<<B, kThreads, 0, h->stream>>>(V, vals, x, y);
    else if (kind == INNER_SELL32) k_sell_apply32<INNER_SELL32><<<B, kThreads, 0, h->stream>>>(V, vals, x, y);
    else k_sell_apply32<INNER_SELL64><<<B, kThreads, 0, h->stream>>>(V, vals, x, y);
    PLATO_LAUNCH_CHECK(h);
    return PLATO_OK;
}

// ---- Lanczos estimate of lambda_max(Dinv A) (see estimate_lambda_max) ----------------------
// lz layout: alpha_k at [k-1], beta_k at [kLanczosMax + k-1], |v_0|_D^2 at [2 kLanczosMax]
constexpr int kLanczosMax = 16;
constexpr int kLanczosSteps = 8;

__global__ void __launch_bounds__(kThreads)
k_lanczos_norm(int64_t n, const float* __restrict__ v, const float* __restrict__ dinv32, double* partials,
               unsigned int* ticket, double* lz) {
    __shared__ double sh[1][32];
    __shared__ bool last;
    double s[1] = {0.0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        s[0] += double(v[i]) * v[i] / dinv32[i];
    block_sum_n<1>(s, sh);
    if (publish_partials<1>(s, partials, ticket, &last)) {
        double t[1];
        final_sums<1>(t, partials, sh);
        if (threadIdx.x == 0) {
            lz[2 * kLanczosMax] = t[0];
            *ticket = 0u;
        }
    }
}

__global__ void k_lanczos_scale(int64_t n, float* __restrict__ v, const double* __restrict__ lz) {
    const float scale = float(1.0 / sqrt(lz[2 * kLanczosMax]));
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        v[i] *= scale;
}

// alpha_k = q.u and beta_k = sqrt(|Dinv u|_D^2 - alpha_k^2 - beta_(k-1)^2), u = A q (masked rows: q)
__global__ void __launch_bounds__(kThreads)
k_lanczos_step(int64_t n, const uint8_t* __restrict__ mask, const float* __restrict__ q, const float* __restrict__ w,
               const float* __restrict__ dinv32, double* partials, unsigned int* ticket, double* lz, int k) {
    __shared__ double sh[2][32];
    __shared__ bool last;
    double s[2] = {0.0, 0.0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double ui = (mask && mask[i]) ? q[i] : w[i];
        s[0] += double(q[i]) * ui;
        s[1] += double(dinv32[i]) * ui * ui;
    }
    block_sum_n<2>(s, sh);
    if (publish_partials<2>(s, partials, ticket, &last)) {
        double t[2];
        final_sums<2>(t, partials, sh);
        if (threadIdx.x == 0) {
            const double a = t[0], bp = k > 1 ? lz[kLanczosMax + k - 2] : 0.0;
            lz[k - 1] = a;
            lz[kLanczosMax + k - 1] = sqrt(fmax(t[1] - a * a - bp * bp, 0.0));
            *ticket = 0u;
        }
    }
}

// q_(k+1) = (Dinv u - alpha_k q_k - beta_(k-1) q_(k-1)) / beta_k (zero after a breakdown)
__global__ void k_lanczos_next(int64_t n, const uint8_t* __restrict__ mask, const float* __restrict__ q,
                               const float* __restrict__ w, const float* __restrict__ qp,
                               const float* __restrict__ dinv32, const double* __restrict__ lz, int k,
                               float* __restrict__ qn) {
    const double a = lz[k - 1], b = lz[kLanczosMax + k - 1], bp = k > 1 ? lz[kLanczosMax + k - 2] : 0.0;
    const float inv = b > 0.0 ? float(1.0 / b) : 0.f;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float ui = (mask && mask[i]) ? q[i] : w[i];
        float r = dinv32[i] * ui - float(a) * q[i];
        if (k > 1) r -= float(bp) * qp[i];
        qn[i] = r * inv;
    }
}

// Largest eigenvalue of the symmetric tridiagonal matrix with diagonal a[0..m) and off-diagonal
// b[0..m-1), by Sturm-sequence bisection (count of eigenvalues below x from the LDL^T pivots).
static double tridiag_max_eigenvalue(const double* a, const double* b, int m) {
    double lo = a[0], hi = a[0];
    for (int i = 0; i < m; ++i) {
        const double r = (i > 0 ? std::fabs(b[i - 1]) : 0.0) + (i + 1 < m ? std::fabs(b[i]) : 0.0);
        lo = std::min(lo, a[i] - r);
        hi = std::max(hi, a[i] + r);
    }
    auto below = [&](double x) {
        int c = 0;
        double d = 1.0;
        for (int i = 0; i < m; ++i) {
            d = a[i] - x - (i > 0 ? b[i - 1] * b[i - 1] / d : 0.0);
            if (d == 0.0) d = -1e-300;
            if (d < 0.0) ++c;
        }
        return c;
    };
    for (int it = 0; it < 200 && hi - lo > 1e-12 * std::max(1.0, std::fabs(hi)); ++it) {
        const double mid = 0.5 * (lo + hi);
        if (below(mid) < m) lo = mid; else hi = mid;
    }
    return hi;
}

// Largest eigenvalue of Dinv A (the preconditioner's operator, D = 1 / dinv) by `steps` Lanczos
// steps in the D inner product, which is what makes Dinv A self-adjoint: q_1 = v / |v|_D; per
// step u = A q_k, alpha_k = q_k . u, beta_k^2 = |Dinv u|_D^2 - alpha_k^2 - beta_(k-1)^2 (both
// sums in one pass), q_(k+1) = (Dinv u - alpha_k q_k - beta_(k-1) q_(k-1)) / beta_k; the
// estimate is the largest eigenvalue of the tridiagonal T_k.  8 steps give what 20 steps of the
// power iteration's Rayleigh quotient gave (40x20x20 cantilever, nodal U[0.01, 1] density:
// 2.556 against 2.545; exact 2.720).
// Constrained rows of the matrix-free operator are identity rows (u_i = q_i).
static int estimate_lambda_max(plato_problem* h, int kind, int steps, double* lmax) {
    const int64_t n = 3 * (int64_t)h->N;
    const int VB = grid_for(n, kThreads, 148 * 16);
    const uint8_t* mask = (kind == INNER_EBE32 || kind == INNER_EBE64) ? h->bc_mask : nullptr;
    steps = std::max(1, std::min(steps, kLanczosMax));
    if (!h->lanczos) PLATO_CUDA(h, cudaMalloc(&h->lanczos, sizeof(double) * 3 * kLanczosMax));
    k_power_init<<<VB, kThreads, 0, h->stream>>>(n, h->f_d0);
    k_lanczos_norm<<<VB, kThreads, 0, h->stream>>>(n, h->f_d0, h->f_dinv, h->partials, h->red_ticket, h->lanczos);
    k_lanczos_scale<<<VB, kThreads, 0, h->stream>>>(n, h->f_d0, h->lanczos);
    PLATO_LAUNCH_CHECK(h);
    // q_(k-1), q_k, q_(k+1) rotate through three FP32 vectors the solve overwrites afterwards
    float* qs[3] = {h->f_d1, h->f_d0, h->f_y};
    int prev = 0, cur = 1, next = 2;
    for (int k = 1; k <= steps; ++k) {
        int rc = apply_inner_plain(h, kind, qs[cur], h->f_w);
        if (rc) return rc;
        k_lanczos_step<<<VB, kThreads, 0, h->stream>>>(n, mask, qs[cur], h->f_w, h->f_dinv, h->partials,
                                                      h->red_ticket, h->lanczos, k);
        PLATO_LAUNCH_CHECK(h);
        if (k < steps) {
            k_lanczos_next<<<VB, kThreads, 0, h->stream>>>(n, mask, qs[cur], h->f_w, qs[prev], h->f_dinv, h->lanczos, k,
                                                          qs[next]);
            PLATO_LAUNCH_CHECK(h);
            const int t = prev;
            prev = cur;
            cur = next;
            next = t;
        }
    }
    double host[3 * kLanczosMax];
    PLATO_CUDA(h, cudaMemcpyAsync(host, h->lanczos, sizeof(host), cudaMemcpyDeviceToHost, h->stream));
    PLATO_CUDA(h, cudaStreamSynchronize(h->stream));
    // stop at a breakdown (beta ~ 0: the Krylov space is invariant)
    int m = steps;
    for (int k = 0; k + 1 < steps; ++k)
        if (!(host[kLanczosMax + k] > 1e-12 * std::fabs(host[k]))) { m = k + 1; break; }
    for (int k = 0; k < m; ++k)
        if (!std::isfinite(host[k]) || (k + 1 < m && !std::isfinite(host[kLanczosMax + k])))
            return plato_fail(h, PLATO_NONFINITE, "Lanczos estimate of the Chebyshev interval failed");
    const double lam = tridiag_max_eigenvalue(host, host + kLanczosMax, m);
    if (!std::isfinite(lam) || !(lam > 0.0))
        return plato_fail(h, PLATO_NONFINITE, "Lanczos estimate of the Chebyshev interval failed");
    *lmax = lam;
    return PLATO_OK;
}

// Chebyshev coefficients for `degree` steps on [lmax/ratio, lmax] (first kind), or -- kind
// 4 -- the fourth-kind polynomial on (0, lmax] (Lottes, "Optimal polynomial smoothers for
// multigrid V-cycles", Numer. Linear Algebra Appl. 2023): d_0 = 4/(3 lmax) Dinv r,
// d_k = (2k-1)/(2k+3) d_(k-1) + (8k+4)/((2k+3) lmax) Dinv r_k, whose error polynomial E
// satisfies max sqrt(lambda/lmax) |E(lambda)| = 1/(2 degree + 1) on (0, lmax].
static ChebCoef chebyshev(double lmax, double ratio, int degree, int kind) {
    ChebCoef c{};
    if (kind == 4) {
        c.c0 = float(4.0 / (3.0 * lmax));
        for (int k = 1; k < degree && k < 64; ++k) {
            c.c1[k] = float((2.0 * k - 1.0) / (2.0 * k + 3.0));
            c.c2[k] = float((8.0 * k + 4.0) / ((2.0 * k + 3.0) * lmax));
        }
        return c;
    }
    const double lmin = lmax / ratio;
    const double theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin), sigma = theta / delta;
    double rho = 1.0 / sigma;
    c.c0 = float(1.0 / theta);
    for (int k = 1; k < degree && k < 64; ++k) {
        const double rn = 1.0 / (2.0 * sigma - rho);
        c.c1[k] = float(rn * rho);
        c.c2[k] = float(2.0 * rn / delta);
        rho = rn;
    }
    return c;
}

// Prepares the operators for a polynomial-preconditioned solve with control z.  Assembled
// operator: from the constrained CRS matrix crs, or -- crs == nullptr -- assembled straight
// into the solver's SELL copies from z (thread-per-row assembly with the constraints applied).
int prepare_mixed(plato_problem* h, const double* crs, const double* z) {
    const int64_t n = 3 * (int64_t)h->N;
    for (float** v : {&h->f_res, &h->f_d0, &h->f_d1, &h->f_y, &h->f_w, &h->f_dinv})
        if (!*v) PLATO_CUDA(h, cudaMalloc(v, sizeof(float) * n));
    if (!h->v_q) PLATO_CUDA(h, cudaMalloc(&h->v_q, sizeof(double) * n));
    const int kind = inner_kind(h);
    if (h->opts.operator_kind == PLATO_OPERATOR_MATRIX_FREE) {
        int rc = matfree_setup(h, z);
        if (rc || kind != INNER_SELL32) return rc;
        // the preconditioner's matrix by FP32 element assembly (no FP64 matrix)
        if (!h->sell32) PLATO_CUDA(h, cudaMalloc(&h->sell32, sizeof(float) * 9 * size_t(h->sell.total_slots)));
        return launch_assemble_sell32(h, z, h->sell32, h->f_dinv);
    }
    const size_t slots = 9 * size_t(h->sell.total_slots);
    if (!h->sell64) PLATO_CUDA(h, cudaMalloc(&h->sell64, sizeof(double) * slots));
    float* o32 = nullptr;
    void* o16 = nullptr;
    if (kind == INNER_SELL32) {
        if (!h->sell32) PLATO_CUDA(h, cudaMalloc(&h->sell32, sizeof(float) * slots));
        o32 = h->sell32;
    } else if (kind == INNER_SELL16) {
        if (!h->sell16) PLATO_CUDA(h, cudaMalloc(&h->sell16, sizeof(__nv_bfloat16) * slots));
        o16 = h->sell16;
    } else if (kind == INNER_SELL16S) {
        if (!h->sell16s) PLATO_CUDA(h, cudaMalloc(&h->sell16s, sizeof(__half) * slots));
        for (float** v : {&h->f_sq, &h->f_isq})
            if (!*v) PLATO_CUDA(h, cudaMalloc(v, sizeof(float) * n));
        int rc = crs ? launch_crs_to_sell(h, crs, h->sell64, nullptr, nullptr, h->v_dinv, nullptr)
                     : launch_assemble_sell(h, z, h->sell64, nullptr, nullptr, h->v_dinv, nullptr);
        if (rc) return rc;
        // the Jacobi diagonal of the scaled matrix is 1: f_dinv = ones
        return launch_sell_scale16(h, h->sell64, h->v_dinv, h->sell16s, h->f_sq, h->f_isq, h->f_dinv);
    }
    return crs ? launch_crs_to_sell(h, crs, h->sell64, o32, o16, h->v_dinv, h->f_dinv)
               : launch_assemble_sell(h, z, h->sell64, o32, o16, h->v_dinv, h->f_dinv);
}

// Mesh-level coarse data (once per grid) and the start mark of the next per-solve set-up.
int prepare_coarse_start(plato_problem* h) {
    if (h->opts.coarse_cells[0] <= 0) return PLATO_OK;
    int rc = coarse_setup_mesh(h);
    if (rc) return rc;
    return coarse_mark_start(h);
}

// Two-level preconditioner data for control z (mesh buckets once, Galerkin operator per solve).
int prepare_coarse(plato_problem* h, const double* z) {
    if (h->opts.coarse_cells[0] <= 0 || !z) return PLATO_OK;
    int rc = coarse_setup_mesh(h);
    if (rc) return rc;
    rc = coarse_setup_operator(h, z, nullptr, 1);  // overlapped with the fine-level set-up
    if (rc) return rc;
    h->coarse.active = 1;
    return PLATO_OK;
}

// Multi-step sweep set-up (once per handle and launch length): the column reach in tiles, the
// stamp and counter arrays, and the task order of an `nsteps`-step launch; *steps = the steps
// per launch to use (0: one launch per step).  Measured on the 160x80x80 bench mesh (halo 13
// tiles, 592 CTAs in flight): a step trails the one before by at least (592 / steps) tiles or
// the tasks serialise on their waits (2 steps, slack 0: 223 us per step; 4 steps: 514 us);
// with that slack the rows between the first and the last front approach half the matrix, so
// little of the L2 reuse survives: 7 steps per launch, slack 130: 81 us per step against 88 us
// with one launch per step, 41.8 against 42.4 ms per solve+adjoint.  The sweep is bound by
// load latency rather than HBM bandwidth, so automatic mode (sweep_steps 0) keeps one launch
// per step and the multi-step form is an option.
constexpr int kWaveSlackCtas = 600;  // default slack: this many tasks between a task and its deps

int wave_steps(plato_problem* h, int* steps, int* lag) {
    *steps = 0;
    if (h->opts.sweep_steps <= 1 || h->wave_halo == -2 || !h->sell.dcols) return PLATO_OK;
    const int32_t nslices = h->sell.nslices;
    const int32_t tiles = int32_t((int64_t(nslices) * 16 + kThreads - 1) / kThreads);
    if (h->wave_halo == -1 || h->wave_tiles != tiles) {
        int32_t* d = nullptr;
        PLATO_CUDA(h, cudaMallocAsync(&d, sizeof(int32_t), h->stream));
        PLATO_CUDA(h, cudaMemsetAsync(d, 0, sizeof(int32_t), h->stream));
        k_wave_halo<<<grid_for(nslices, 1, 148 * 8), 256, 0, h->stream>>>(sell_view(h), d);
        PLATO_LAUNCH_CHECK(h);
        int32_t halo = 0;
        PLATO_CUDA(h, cudaMemcpyAsync(&halo, d, sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream));
        PLATO_CUDA(h, cudaFreeAsync(d, h->stream));
        PLATO_CUDA(h, cudaStreamSynchronize(h->stream));
        if (h->wave_flags) PLATO_CUDA(h, cudaFree(h->wave_flags));
        h->wave_flags = nullptr;
        for (int k = 0; k <= kWaveMaxSteps; ++k) {
            if (h->wave_order[k]) PLATO_CUDA(h, cudaFree(h->wave_order[k]));
            h->wave_order[k] = nullptr;
        }
        PLATO_CUDA(h, cudaMalloc(&h->wave_flags, sizeof(int32_t) * kWaveMaxSteps * size_t(tiles)));
        PLATO_CUDA(h, cudaMemset(h->wave_flags, 0, sizeof(int32_t) * kWaveMaxSteps * size_t(tiles)));
        if (!h->wave_ctl) {
            PLATO_CUDA(h, cudaMalloc(&h->wave_ctl, sizeof(WaveCtl)));
            PLATO_CUDA(h, cudaMemset(h->wave_ctl, 0, sizeof(WaveCtl)));
        }
        h->wave_epoch = 0;
        h->wave_tiles = tiles;
        h->wave_halo = halo;
    }
    const int S = h->opts.sweep_steps;
    *lag = h->wave_halo + 1 + (h->opts.sweep_lag > 0 ? h->opts.sweep_lag : (kWaveSlackCtas + S - 1) / S);
    if (h->wave_tiles < 2 * (h->wave_halo + 1)) return PLATO_OK;  // too few tiles to pipeline
    *steps = S;
    return PLATO_OK;
}

int wave_order(plato_problem* h, int nsteps, int lag) {
    if (h->wave_order[nsteps] && h->wave_order_lag[nsteps] == lag) return PLATO_OK;
    const int32_t tiles = h->wave_tiles;
    std::vector<std::pair<int64_t, int32_t>> key;
    key.reserve(size_t(nsteps) * tiles);
    for (int j = 0; j < nsteps; ++j)
        for (int32_t t = 0; t < tiles; ++t)
            key.push_back({(int64_t(t) + int64_t(lag) * j) * 64 + (63 - j), (j << 24) | t});
    std::sort(key.begin(), key.end());
    std::vector<int32_t> codes(key.size());
    for (size_t i = 0; i < key.size(); ++i) codes[i] = key[i].second;
    if (h->wave_order[nsteps]) PLATO_CUDA(h, cudaFree(h->wave_order[nsteps]));
    h->wave_order[nsteps] = nullptr;
    PLATO_CUDA(h, cudaMalloc(&h->wave_order[nsteps], sizeof(int32_t) * codes.size()));
    PLATO_CUDA(h, cudaMemcpy(h->wave_order[nsteps], codes.data(), sizeof(int32_t) * codes.size(),
                             cudaMemcpyHostToDevice));
    h->wave_order_lag[nsteps] = lag;
    return PLATO_OK;
}

// Global steps [first, first + nsteps) of a preconditioner call in one launch; steps below
// `cheb_end` are Chebyshev steps (coefficients cc), the others residual-only.
int wave_launch(plato_problem* h, const ChebCoef& cc, int first, int nsteps, int cheb_end, int lag, int grid) {
    int rc = wave_order(h, nsteps, lag);
    if (rc) return rc;
    WaveStep st{};
    st.first = first;
    st.nsteps = nsteps;
    st.nupdate = std::max(0, std::min(nsteps, cheb_end - first));
    for (int j = 0; j < nsteps && first + j < 64; ++j) {
        st.c1[j] = cc.c1[first + j];
        st.c2[j] = cc.c2[first + j];
    }
    const int32_t ntasks = nsteps * h->wave_tiles;
    const int32_t epoch = ++h->wave_epoch;
    // test hook (plato_test_stall_next_sweep): the launch waits for a later epoch than its
    // tasks stamp, so its first dependency wait runs out
    const int32_t wait_epoch = h->wave_stall ? epoch + 1 : epoch;
    h->wave_stall = 0;
    k_sell16s_wave<true><<<std::min(grid, ntasks), kThreads, 0, h->stream>>>(
        sell_view(h), static_cast<const __half*>(h->sell16s), h->f_res, h->f_d0, h->f_d1, h->f_y, st,
        h->wave_order[nsteps], ntasks, h->wave_tiles, h->wave_halo, epoch, wait_epoch, h->wave_flags,
        reinterpret_cast<WaveCtl*>(h->wave_ctl), h->scal);
    PLATO_LAUNCH_CHECK(h);
    h->launches += 1;
    return PLATO_OK;
}

// Flexible CG with the Chebyshev preconditioner: A x = b, x holds the initial guess.
int fcg_poly(plato_problem* h, const double* b, double* x, plato_solve_stats* stats) {
    const int64_t n = 3 * (int64_t)h->N;
    cudaStream_t s = h->stream;
    const double tol = h->opts.tolerance;
    const int32_t max_it = h->opts.max_iterations;
    const int degree = h->opts.chebyshev_degree < 1 ? 1 : (h->opts.chebyshev_degree > 64 ? 64 : h->opts.chebyshev_degree);
    const int kind = inner_kind(h);
    const bool mf = h->opts.operator_kind == PLATO_OPERATOR_MATRIX_FREE;       // FP64 outer operator
    const bool mf_inner = kind == INNER_EBE32 || kind == INNER_EBE64;          // preconditioner operator
    const int VB = grid_for(n, kThreads, 148 * 16);
    const int SB = spmv_blocks(h);
    const SellView V = sell_view(h);
    // The FP16 sweep runs as one resident wave that strides over the row pairs (every CTA
    // takes 3-4 pairs per thread on the bench mesh): 8 % faster per step than a grid of one
    // pair per thread, whose last partial wave leaves SMs idle.
    int CB = SB, CBst = SB;
    if (kind == INNER_SELL16S) {
        int sms = 0, per_sm = 0;
        PLATO_CUDA(h, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
        PLATO_CUDA(h, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sell16s<0, false>, kThreads, 0));
        CB = std::min(SB, std::max(1, per_sm) * std::max(1, sms));
        if (V.dcols) {  // the staged form, one resident wave as well
            int per_st = 0;
            PLATO_CUDA(h, cudaFuncSetAttribute(k_sell16s_st<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, kStSmem));
            PLATO_CUDA(h, cudaFuncSetAttribute(k_sell16s_st<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kStSmem));
            PLATO_CUDA(h, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_st, k_sell16s_st<0>, kThreads, kStSmem));
            CBst = std::min(SB, std::max(1, per_st) * std::max(1, sms));
        }
    }
    // multi-step sweep (FP16 scaled matrix, numbering with a short column reach)
    int wave_S = 0, wave_lag = 0, wave_grid = 0;
    if (kind == INNER_SELL16S) {
        const int wrc = wave_steps(h, &wave_S, &wave_lag);
        if (wrc) return wrc;
        if (wave_S > 0) {
            int sms = 0, per_sm = 0;
            PLATO_CUDA(h, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
            PLATO_CUDA(h, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sell16s_wave<true>, kThreads, 0));
            wave_grid = std::max(1, per_sm) * std::max(1, sms);
        }
    }
    h->sweep_steps_used = wave_S > 0 ? wave_S : 1;

    double lmax = 0.0;
    int rc = estimate_lambda_max(h, kind, kLanczosSteps, &lmax);
    if (rc) return rc;
    const double safety = kind == INNER_SELL16 ? 1.15 : 1.10;
    const ChebCoef cc = chebyshev(lmax * safety, h->opts.chebyshev_ratio > 1.0 ? h->opts.chebyshev_ratio : 30.0, degree,
                                   h->opts.chebyshev_kind);
    // The coarse set-up runs on its own stream meanwhile; the handle's stream waits for it only
    // at the first coarse solve (after the first residual and Chebyshev sweep), so the set-up
    // overlaps that work too.
    bool coarse_waited = false;

    auto outer_apply = [&](const double* in, double* out) -> int {
        if (mf) {
            int r2 = launch_ebe_apply64(h, in, out, nullptr);
            if (r2) return r2;
            return launch_mask_copy(h, in, out);
        }
        return launch_sell_spmv(h, h->sell64, in, out);
    };
    const bool coarse = h->coarse.active != 0;
    // FP16 scaled inner matrix: the preconditioner works on D^-1/2 r and returns D^1/2 z
    const bool scaled = kind == INNER_SELL16S;
    const float* res_scale = scaled ? h->f_isq : nullptr;
    // res -= A_inner xin (FP32)
    auto inner_apply_sub = [&](const float* xin) -> int {
        if (mf_inner) {
            int r2 = launch_ebe_apply32(h, xin, h->f_w, h->scal);
            if (r2) return r2;
            k_res_sub_vec<<<VB, kThreads, 0, s>>>(n, h->bc_mask, xin, h->f_w, h->f_res, h->scal);
        } else if (kind == INNER_SELL16S) {
            if (V.dcols)
                PLATO_CUDA(h, launch_pdl_smem(k_sell16s_st<1>, CBst, kThreads, size_t(kStSmem), s, V,
                                              static_cast<const __half*>(h->sell16s), xin, h->f_res, nullptr, nullptr,
                                              0.f, 0.f, (const PcgScalars*)h->scal));
            else
                PLATO_CUDA(h, launch_pdl(k_sell16s<1, false>, CB, kThreads, s, V, static_cast<const __half*>(h->sell16s),
                                         xin, h->f_res, nullptr, nullptr, 0.f, 0.f, (const PcgScalars*)h->scal));
        } else if (kind == INNER_SELL16) {
            k_res_sub_sell<INNER_SELL16><<<SB, kThreads, 0, s>>>(V, h->sell16, xin, h->f_res, h->scal);
        } else if (kind == INNER_SELL32) {
            k_res_sub_sell<INNER_SELL32><<<SB, kThreads, 0, s>>>(V, h->sell32, xin, h->f_res, h->scal);
        } else {
            k_res_sub_sell<INNER_SELL64><<<SB, kThreads, 0, s>>>(V, h->sell64, xin, h->f_res, h->scal);
        }
        PLATO_LAUNCH_CHECK(h);
        return PLATO_OK;
    };
    float* dlast = h->f_d0;
    int wave_first_len = 0;  // steps in the first launch of a multi-step sweep (timing)
    std::vector<int64_t> timed_iters;  // timing records of the current pass (see collect_timing)
    int64_t inner_record = -1;  // >= 0: time the first step of this sweep (record 2*iter+1)
    // The multi-step sweep runs the Chebyshev steps 1 .. degree-1 and, with a coarse space, the
    // residual step res -= A^ d_(degree-1) of the two-level form as step `degree`, in launches
    // of at most wave_S steps of as even a length as possible.
    auto wave_sweep = [&]() -> int {
        const int total = (degree - 1) + (coarse ? 1 : 0);
        const int launches_n = (total + wave_S - 1) / wave_S;
        int first = 1;
        for (int L = 0; L < launches_n; ++L) {
            const int len = (total - (first - 1) + (launches_n - L) - 1) / (launches_n - L);
            cudaEvent_t t0 = nullptr, t1 = nullptr;
            if (L == 0 && inner_record >= 0) {
                int r2 = timing_events(h, &t0, &t1);
                if (r2) return r2;
                timed_iters.push_back(inner_record);
                PLATO_CUDA(h, cudaEventRecord(t0, s));
            }
            int r2 = wave_launch(h, cc, first, len, degree, wave_lag, wave_grid);
            if (r2) return r2;
            if (t1) PLATO_CUDA(h, cudaEventRecord(t1, s));
            if (L == 0) wave_first_len = len;
            first += len;
        }
        dlast = ((degree - 1) & 1) ? h->f_d1 : h->f_d0;
        return PLATO_OK;
    };
    auto chebyshev_steps = [&]() -> int {
        if (wave_S > 0) return wave_sweep();
        float* dcur = h->f_d0;
        float* dnext = h->f_d1;
        // a sampled call times its whole run of degree - 1 consecutive step launches between one
        // event pair (collect_timing counts it as that many steps)
        cudaEvent_t t0 = nullptr, t1 = nullptr;
        for (int k = 1; k < degree; ++k) {
            if (k == 1 && inner_record >= 0) {
                int r2 = timing_events(h, &t0, &t1);
                if (r2) return r2;
                timed_iters.push_back(inner_record);
                PLATO_CUDA(h, cudaEventRecord(t0, s));
            }
            if (mf_inner) {
                int r2 = launch_ebe_apply32(h, dcur, h->f_w, h->scal);
                if (r2) return r2;
                k_cheb_vec<<<VB, kThreads, 0, s>>>(n, h->bc_mask, h->f_w, h->f_dinv, h->f_res, dcur, dnext, h->f_y,
                                                   cc.c1[k], cc.c2[k], h->scal);
            } else if (kind == INNER_SELL16S) {
                if (V.dcols)
                    PLATO_CUDA(h, launch_pdl_smem(k_sell16s_st<0>, CBst, kThreads, size_t(kStSmem), s, V,
                                                  static_cast<const __half*>(h->sell16s), (const float*)dcur, h->f_res,
                                                  dnext, h->f_y, cc.c1[k], cc.c2[k], (const PcgScalars*)h->scal));
                else
                    PLATO_CUDA(h, launch_pdl(k_sell16s<0, false>, CB, kThreads, s, V,
                                             static_cast<const __half*>(h->sell16s), (const float*)dcur, h->f_res, dnext,
                                             h->f_y, cc.c1[k], cc.c2[k], (const PcgScalars*)h->scal));
            } else if (kind == INNER_SELL16) {
                k_cheb_sell<INNER_SELL16><<<SB, kThreads, 0, s>>>(V, h->sell16, h->f_dinv, h->f_res, dcur, dnext,
                                                                  h->f_y, cc.c1[k], cc.c2[k], h->scal);
            } else if (kind == INNER_SELL32) {
                k_cheb_sell<INNER_SELL32><<<SB, kThreads, 0, s>>>(V, h->sell32, h->f_dinv, h->f_res, dcur, dnext,
                                                                  h->f_y, cc.c1[k], cc.c2[k], h->scal);
            } else {
                k_cheb_sell<INNER_SELL64><<<SB, kThreads, 0, s>>>(V, h->sell64, h->f_dinv, h->f_res, dcur, dnext,
                                                                  h->f_y, cc.c1[k], cc.c2[k], h->scal);
            }
            PLATO_LAUNCH_CHECK(h);
            if (t1 && k == degree - 1) PLATO_CUDA(h, cudaEventRecord(t1, s));
            std::swap(dcur, dnext);
        }
        dlast = dcur;
        return PLATO_OK;
    };
    // M(r) with r in f_res (FP32) and, from the update kernel, d0 = c0 Dinv r, y = d0 already
    // written.  Without a coarse space M = the Chebyshev sweep S.  With it, the two-level form
    // A-DEF2 (Tang, Nabben, Vuik, Erlangga, J. Sci. Comput. 39, 2009), M = (I - CA) S + C with
    // C = Z E^-1 Z^T: s = S r; res = r - A s; y = s + C res - one coarse solve and one extra
    // inner operator apply per call (the balancing form C + (I - CA) S (I - AC) needs two of each).
    auto precondition = [&](float) -> int {
        int r2 = chebyshev_steps();
        if (r2 || !coarse) return r2;
        if (wave_S == 0) {
            r2 = inner_apply_sub(dlast);  // the sweep left res = r - A (s - d_last)
            if (r2) return r2;
        }
        if (!coarse_waited) {
            r2 = coarse_wait(h);
            if (r2) return r2;
            coarse_waited = true;
        }
        return coarse_apply(h, h->f_res, h->f_y, 1, h->scal, scaled ? h->f_sq : nullptr);
    };

    PcgScalars init{};
    PLATO_CUDA(h, cudaMemcpyAsync(h->scal, &init, sizeof(PcgScalars), cudaMemcpyHostToDevice, s));
    int32_t restarts = 0, iter_base = 0;
    bool keep_bb = false;
    int64_t precond_applies = 0;
    for (;;) {
        // r = b - A x; z = M r; p = z; p.r
        rc = outer_apply(x, h->v_r);
        if (rc) return rc;
        k_fcg_start<<<VB, kThreads, 0, s>>>(n, b, h->v_r, h->f_dinv, res_scale, h->f_res, h->f_d0, h->f_y, cc.c0, h->scal,
                                             h->partials, tol, keep_bb ? 1 : 0);
        PLATO_LAUNCH_CHECK(h);
        rc = precondition(cc.c0);
        if (rc) return rc;
        k_fcg_zq<<<VB, kThreads, 0, s>>>(n, h->f_y, res_scale, h->v_z, h->v_q, h->scal, h->partials, 1);
        k_fcg_direction<<<VB, kThreads, 0, s>>>(n, h->v_z, h->v_p, h->v_r, h->scal, h->partials, 1);
        h->launches += 1;
        PLATO_LAUNCH_CHECK(h);
        rc = deflate_direction(h, h->v_p, h->v_r, 1);
        if (rc) return rc;

        PcgScalars* slots = h->scal_host;
        int64_t enqueued = 0;
        timed_iters.clear();
        h->ev_used = 0;
        int cur = 0;
        bool have_prev = false;
        cudaEvent_t* ev = h->poll_ev;
        for (int e = 0; e < 2; ++e)
            if (!ev[e]) PLATO_CUDA(h, cudaEventCreateWithFlags(&ev[e], cudaEventDisableTiming));
        ChunkPlanner plan;
        plan.full = kChunk;
        int32_t chunk = kChunk;
        for (;;) {
            for (int k = 0; k < chunk; ++k, ++enqueued) {
                const bool timed = h->timing && (enqueued % kTimingStride) == 0;
                cudaEvent_t e0 = nullptr, e1 = nullptr;
                if (timed) {
                    rc = timing_events(h, &e0, &e1);
                    if (rc) return rc;
                    timed_iters.push_back(2 * enqueued);
                    PLATO_CUDA(h, cudaEventRecord(e0, s));
                }
                if (mf) {
                    rc = launch_ebe_apply64(h, h->v_p, h->v_q, h->scal);
                    if (rc) return rc;
                    k_fcg_mask_dot<<<VB, kThreads, 0, s>>>(n, h->bc_mask, h->v_p, h->v_q, h->scal, h->partials);
                } else {
                    PLATO_CUDA(h, launch_pdl(k_fcg_sell_apply, SB, kThreads, s, V, (const double*)h->sell64,
                                             (const double*)h->v_p, h->v_q, h->scal, h->partials));
                }
                if (timed) PLATO_CUDA(h, cudaEventRecord(e1, s));
                PLATO_CUDA(h, launch_pdl(k_fcg_update, VB, kThreads, s, n, x, h->v_r, (const double*)h->v_p,
                                         (const double*)h->v_q, (const float*)h->f_dinv, res_scale, h->f_res, h->f_d0,
                                         h->f_y, cc.c0, h->scal, h->partials, max_it));
                h->launches += 2;
                inner_record = timed ? 2 * enqueued + 1 : -1;
                rc = precondition(cc.c0);
                inner_record = -1;
                if (rc) return rc;
                PLATO_CUDA(h, launch_pdl(k_fcg_zq, VB, kThreads, s, n, (const float*)h->f_y, res_scale, h->v_z,
                                         (const double*)h->v_q, h->scal, h->partials, 0));
                PLATO_CUDA(h, launch_pdl(k_fcg_direction, VB, kThreads, s, n, (const double*)h->v_z, h->v_p,
                                         (const double*)h->v_r, h->scal, h->partials, 0));
                h->launches += 1;
                PLATO_LAUNCH_CHECK(h);
                rc = deflate_direction(h, h->v_p, h->v_r, 1);
                if (rc) return rc;
            }
            PLATO_CUDA(h, cudaMemcpyAsync(&slots[cur], h->scal, sizeof(PcgScalars), cudaMemcpyDeviceToHost, s));
            PLATO_CUDA(h, cudaEventRecord(ev[cur], s));
            const int32_t queued = chunk;  // behind the polled state: this chunk
            if (have_prev) {
                PLATO_CUDA(h, cudaEventSynchronize(ev[cur ^ 1]));
                if (slots[cur ^ 1].done) break;
                chunk = plan.next(slots[cur ^ 1], queued);
            }
            have_prev = true;
            cur ^= 1;
        }
        PLATO_CUDA(h, cudaStreamSynchronize(s));
        PcgScalars fin;
        PLATO_CUDA(h, cudaMemcpy(&fin, h->scal, sizeof(PcgScalars), cudaMemcpyDeviceToHost));
        if (wave_S > 0) {
            WaveCtl ctl{};
            PLATO_CUDA(h, cudaMemcpy(&ctl, h->wave_ctl, sizeof(WaveCtl), cudaMemcpyDeviceToHost));
            if (ctl.fail) {
                // a dependency wait ran out: no further multi-step launches on this handle; the
                // caller's fallback (plain FP64 Jacobi-PCG) redoes the solve
                PLATO_CUDA(h, cudaMemset(h->wave_ctl, 0, sizeof(WaveCtl)));
                h->wave_halo = -2;
                h->ev_used = 0;
                stats->converged = 0;
                stats->status = PLATO_NOT_CONVERGED;
                return plato_fail(h, PLATO_NOT_CONVERGED,
                                  "multi-step sweep: a bounded wait for a neighbouring tile ran out");
            }
        }
        h->inner_record_steps = wave_S > 0 ? wave_first_len : std::max(1, degree - 1);
        rc = collect_timing(h, timed_iters, fin.iter - iter_base);
        if (rc) return rc;
        precond_applies += int64_t(fin.iter - iter_base + 1) * (degree - 1);
        iter_base = fin.iter;
        stats->iterations = fin.iter;
        stats->refinements = int32_t(precond_applies);
        if (fin.nonfinite) {
            stats->relative_residual = NAN;
            stats->converged = 0;
            stats->status = PLATO_NONFINITE;
            return plato_fail(h, PLATO_NONFINITE, "non-finite value or loss of positivity in flexible CG");
        }
        // true residual r = b - A x
        rc = outer_apply(x, h->v_q);
        if (rc) return rc;
        rc = launch_axpby(h, n, 1.0, b, 0.0, h->v_r);
        if (rc) return rc;
        rc = launch_axpby(h, n, -1.0, h->v_q, 1.0, h->v_r);
        if (rc) return rc;
        double rr = 0.0;
        rc = launch_dot(h, h->v_r, h->v_r, n, &rr);
        if (rc) return rc;
        const double rel = fin.bb > 0.0 ? std::sqrt(rr / fin.bb) : 0.0;
        stats->relative_residual = rel;
        // same acceptance as the plain PCG: the recomputed FP64 residual meets the tolerance
        if (fin.bb == 0.0 || rel <= tol) {
            stats->converged = 1;
            stats->status = PLATO_OK;
            return PLATO_OK;
        }
        if (fin.iter >= max_it || restarts >= kMaxRestarts) {
            stats->converged = 0;
            stats->status = PLATO_NOT_CONVERGED;
            return plato_fail(h, PLATO_NOT_CONVERGED, "flexible CG stopped before ||b - A x|| <= tol ||b||");
        }
        ++restarts;
        keep_bb = true;
        PcgScalars cont = fin;
        cont.done = 0;
        PLATO_CUDA(h, cudaMemcpyAsync(h->scal, &cont, sizeof(PcgScalars), cudaMemcpyHostToDevice, s));
    }
}

// ---- batched flexible CG ------------------------------------------------------------------
//
// A batch is the disjoint union of independent problems, so its operator is block diagonal
// and every member's Krylov recurrence only needs member-wise dot products.  The segmented
// kernels below run one CTA per tile of at most kThreads rows of one member; each reduction
// publishes per-tile partials and the last tile of a member to finish (per-member ticket)
// sums that member's partials in tile order (deterministic) and updates its scalars.  Tiles
// of converged members return at once.  The Chebyshev preconditioner kernels are row-local
// and run over the whole union; the batch-wide PcgScalars::done is set when every member is
// done and stops them.

namespace {

struct BatchView {
    int32_t        nseg;
    int32_t        ntiles;
    const int32_t* cta_seg;   // member of each tile
    const int32_t* cta_row0;  // first row of each tile
    const int32_t* cta_row1;  // one past its last row
    const int32_t* seg_cta0;  // first tile of each member
    SegScalars*    S;
    PcgScalars*    G;
    int32_t*       ndone;
    double*        partials;  // NV per tile
};

// Block sums of tile t's values into its partials; true in the CTA that finishes the
// member's last tile (its view of the member's partials is then complete).
template <int NV>
__device__ __forceinline__ bool seg_publish(const BatchView& B, int s, int t, double (&v)[NV], double (*sh)[32],
                                            bool* sh_last) {
    block_sum_n<NV>(v, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) B.partials[NV * t + q] = v[q];
        __threadfence();
        const unsigned tiles = unsigned(B.seg_cta0[s + 1] - B.seg_cta0[s]);
        *sh_last = atomicAdd(&B.S[s].ticket, 1u) == tiles - 1u;
    }
    __syncthreads();
    return *sh_last;
}

template <int NV>
__device__ __forceinline__ void seg_final(const BatchView& B, int s, double (&t)[NV], double (*sh)[32]) {
    __threadfence();
#pragma unroll
    for (int q = 0; q < NV; ++q) t[q] = 0.0;
    for (int c = B.seg_cta0[s] + threadIdx.x; c < B.seg_cta0[s + 1]; c += blockDim.x)
#pragma unroll
        for (int q = 0; q < NV; ++q) t[q] += B.partials[NV * c + q];
    block_sum_n<NV>(t, sh);
}

// thread 0 of a member's last tile, when the member turns done
__device__ __forceinline__ void seg_mark_done(const BatchView& B) {
    if (atomicAdd(B.ndone, 1) + 1 == B.nseg) B.G->done = 1;
}

// Every batched kernel is persistent: a grid of (CTAs per SM) x SMs walks the member tiles
// (tile t, then t + gridDim.x, ...), one row of the tile per thread (blockDim.x = the tile
// rows the autotuner chose), skipping the tiles of members that are done.
constexpr int kMaxTileRows = 512;

// r = b - A x (A x in r on entry), r.r and b.b per member; starts the preconditioner.
// accept scales the stop test (1: the FP64 true residual must meet the tolerance).
__global__ void __launch_bounds__(kMaxTileRows)
k_bfcg_start(BatchView B, const double* __restrict__ b, double* __restrict__ r, const float* __restrict__ dinv32,
             float* __restrict__ res, float* __restrict__ d, float* __restrict__ y, float c0, double tol,
             int keep_bb, double accept) {
    __shared__ double sh[2][32];
    __shared__ bool last;
    for (int t = blockIdx.x; t < B.ntiles; t += gridDim.x) {
        const int s = B.cta_seg[t];
        const int64_t row = B.cta_row0[t] + threadIdx.x;
        double v[2] = {0.0, 0.0};
        if (row < B.cta_row1[t]) {
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const int64_t k = 3 * row + i;
                const double ri = b[k] - r[k];
                r[k] = ri;
                v[0] += ri * ri;
                v[1] += b[k] * b[k];
                const float rf = float(ri);
                const float di = c0 * dinv32[k] * rf;
                res[k] = rf;
                d[k] = di;
                y[k] = di;
            }
        }
        if (seg_publish<2>(B, s, t, v, sh, &last)) {
            double tt[2];
            seg_final<2>(B, s, tt, sh);
            if (threadIdx.x == 0) {
                SegScalars& S = B.S[s];
                S.rr = tt[0];
                if (!keep_bb) {
                    S.bb = tt[1];
                    S.tol2 = tol * tol * tt[1];
                    S.iter = 0;
                }
                S.nonfinite = (!isfinite(tt[0]) || !isfinite(tt[1])) ? 1 : 0;
                S.done = (tt[0] <= accept * accept * S.tol2 || S.nonfinite) ? 1 : 0;
                if (S.done) seg_mark_done(B);
                S.ticket = 0u;
            }
        }
    }
}

// q = A p (FP64 SELL rows of the tile), p.q per member -> alpha = (p.r)/(p.q)
__global__ void __launch_bounds__(kMaxTileRows)
k_bfcg_apply(BatchView B, SellView A, const double* __restrict__ vals, const double* __restrict__ p,
             double* __restrict__ q) {
    __shared__ double sh[1][32];
    __shared__ bool last;
    for (int t = blockIdx.x; t < B.ntiles; t += gridDim.x) {
        const int s = B.cta_seg[t];
        if (B.S[s].done) continue;
        const int64_t row = B.cta_row0[t] + threadIdx.x;
        double v[1] = {0.0};
        if (row < B.cta_row1[t]) {
            double a0, a1, a2;
            sell_row<double>(A, vals, p, row, a0, a1, a2);
            q[3 * row] = a0;
            q[3 * row + 1] = a1;
            q[3 * row + 2] = a2;
            v[0] = p[3 * row] * a0 + p[3 * row + 1] * a1 + p[3 * row + 2] * a2;
        }
        if (seg_publish<1>(B, s, t, v, sh, &last)) {
            double tt[1];
            seg_final<1>(B, s, tt, sh);
            if (threadIdx.x == 0) {
                SegScalars& S = B.S[s];
                S.pq = tt[0];
                S.alpha = S.pr / tt[0];
                if (!isfinite(S.alpha) || tt[0] <= 0.0) {
                    S.nonfinite = 1;
                    S.done = 1;
                    seg_mark_done(B);
                }
                S.ticket = 0u;
            }
        }
    }
}

// x += alpha p; r -= alpha q; r.r and the member's stop test; starts the preconditioner.
// Tiles of converged members clear their preconditioner vectors instead.
__global__ void __launch_bounds__(kMaxTileRows)
k_bfcg_update(BatchView B, double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
              const double* __restrict__ q, const float* __restrict__ dinv32, float* __restrict__ res,
              float* __restrict__ d, float* __restrict__ y, float c0, int32_t max_it) {
    __shared__ double sh[1][32];
    __shared__ bool last;
    for (int t = blockIdx.x; t < B.ntiles; t += gridDim.x) {
        const int s = B.cta_seg[t];
        const int64_t row = B.cta_row0[t] + threadIdx.x;
        const bool in = row < B.cta_row1[t];
        if (B.S[s].done) {
            if (in)
#pragma unroll
                for (int i = 0; i < 3; ++i) res[3 * row + i] = d[3 * row + i] = y[3 * row + i] = 0.f;
            continue;
        }
        const double alpha = B.S[s].alpha;
        double v[1] = {0.0};
        if (in) {
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const int64_t k = 3 * row + i;
                x[k] += alpha * p[k];
                const double ri = r[k] - alpha * q[k];
                r[k] = ri;
                v[0] += ri * ri;
                const float rf = float(ri);
                const float di = c0 * dinv32[k] * rf;
                res[k] = rf;
                d[k] = di;
                y[k] = di;
            }
        }
        if (seg_publish<1>(B, s, t, v, sh, &last)) {
            double tt[1];
            seg_final<1>(B, s, tt, sh);
            if (threadIdx.x == 0) {
                SegScalars& S = B.S[s];
                S.rr = tt[0];
                S.iter += 1;
                if (!isfinite(tt[0])) S.nonfinite = 1;
                if (S.nonfinite || tt[0] <= S.tol2 || S.iter >= max_it) {
                    S.done = 1;
                    seg_mark_done(B);
                }
                S.ticket = 0u;
            }
        }
    }
}

// z = y (widened); z.q per member -> beta = -(z.q)/(p.q).  first: only z = y.
__global__ void __launch_bounds__(kMaxTileRows)
k_bfcg_zq(BatchView B, const float* __restrict__ y, double* __restrict__ z, const double* __restrict__ q, int first) {
    __shared__ double sh[1][32];
    __shared__ bool last;
    for (int t = blockIdx.x; t < B.ntiles; t += gridDim.x) {
        const int s = B.cta_seg[t];
        if (B.S[s].done) continue;
        const int64_t row = B.cta_row0[t] + threadIdx.x;
        const bool in = row < B.cta_row1[t];
        double v[1] = {0.0};
        if (in)
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const int64_t k = 3 * row + i;
                const double zi = double(y[k]);
                z[k] = zi;
                if (!first) v[0] += zi * q[k];
            }
        if (first) continue;
        if (seg_publish<1>(B, s, t, v, sh, &last)) {
            double tt[1];
            seg_final<1>(B, s, tt, sh);
            if (threadIdx.x == 0) {
                SegScalars& S = B.S[s];
                S.zq = tt[0];
                S.beta = -tt[0] / S.pq;
                if (!isfinite(S.beta)) {
                    S.nonfinite = 1;
                    S.done = 1;
                    seg_mark_done(B);
                }
                S.ticket = 0u;
            }
        }
    }
}

// p = z + beta p; p.r per member.
__global__ void __launch_bounds__(kMaxTileRows)
k_bfcg_direction(BatchView B, const double* __restrict__ z, double* __restrict__ p, const double* __restrict__ r,
                 int first) {
    __shared__ double sh[1][32];
    __shared__ bool last;
    for (int t = blockIdx.x; t < B.ntiles; t += gridDim.x) {
        const int s = B.cta_seg[t];
        if (B.S[s].done) continue;
        const double beta = first ? 0.0 : B.S[s].beta;
        const int64_t row = B.cta_row0[t] + threadIdx.x;
        double v[1] = {0.0};
        if (row < B.cta_row1[t])
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const int64_t k = 3 * row + i;
                const double pi = z[k] + (first ? 0.0 : beta * p[k]);
                p[k] = pi;
                v[0] += pi * r[k];
            }
        if (seg_publish<1>(B, s, t, v, sh, &last)) {
            double tt[1];
            seg_final<1>(B, s, tt, sh);
            if (threadIdx.x == 0) {
                SegScalars& S = B.S[s];
                S.pr = tt[0];
                if (!isfinite(tt[0])) {
                    S.nonfinite = 1;
                    S.done = 1;
                    seg_mark_done(B);
                }
                S.ticket = 0u;
            }
        }
    }
}

// One Chebyshev step over the tiles of members still iterating (converged members' rows
// are skipped): w = A d_cur, res -= w, d_next = c1 d_cur + c2 Dinv res, y += d_next.
template <int KIND>
__global__ void __launch_bounds__(kMaxTileRows)
k_bcheb_sell(BatchView B, SellView A, const void* __restrict__ vals, const float* __restrict__ dinv32,
             float* __restrict__ res, const float* __restrict__ dcur, float* __restrict__ dnext, float* __restrict__ y,
             float c1, float c2) {
    for (int t = blockIdx.x; t < B.ntiles; t += gridDim.x) {
        if (B.S[B.cta_seg[t]].done) continue;
        const int64_t r = B.cta_row0[t] + threadIdx.x;
        if (r >= B.cta_row1[t]) continue;
        float w0, w1, w2;
        if (KIND == INNER_SELL16)
            sell_row_bf16(A, static_cast<const __nv_bfloat16*>(vals), dcur, r, w0, w1, w2);
        else if (KIND == INNER_SELL32)
            sell_row<float>(A, static_cast<const float*>(vals), dcur, r, w0, w1, w2);
        else {
            double a0, a1, a2;
            sell_row<double>(A, static_cast<const double*>(vals), dcur, r, a0, a1, a2);
            w0 = float(a0); w1 = float(a1); w2 = float(a2);
        }
        const float w[3] = {w0, w1, w2};
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const int64_t k = 3 * r + i;
            const float rs = res[k] - w[i];
            res[k] = rs;
            const float dn = c1 * dcur[k] + c2 * dinv32[k] * rs;
            dnext[k] = dn;
            y[k] += dn;
        }
    }
}

}  // namespace

// Batched flexible CG with the Chebyshev-Jacobi preconditioner on the assembled union
// operator (SELL copies prepared by prepare_mixed); x holds the initial guess.  Every member
// stops on its own residual test ||r_s|| <= tol ||b_s||, confirmed with its recomputed true
// residual; per-member statistics go to h->batch.last, the aggregate to *stats.
int fcg_batch(plato_problem* h, const double* b, double* x, plato_solve_stats* stats) {
    BatchState& bt = h->batch;
    const int64_t n = 3 * (int64_t)h->N;
    cudaStream_t s = h->stream;
    const double tol = h->opts.tolerance;
    const int32_t max_it = h->opts.max_iterations;
    const int degree = h->opts.chebyshev_degree < 1 ? 1 : (h->opts.chebyshev_degree > 64 ? 64 : h->opts.chebyshev_degree);
    const int kind = inner_kind(h);
    if (kind == INNER_SELL16S)
        return plato_fail(h, PLATO_NOT_SUPPORTED, "the FP16 scaled inner precision is built for single problems");
    const SellView V = sell_view(h);
    // persistent grid: the autotuned CTAs per SM x SMs (never more CTAs than tiles), one row of
    // a tile per thread
    const int TR = bt.tile_rows;
    int sms = 0;
    PLATO_CUDA(h, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
    const int T = std::max(1, std::min(bt.ncta, bt.ctas_per_sm * sms));
    const BatchView BV{bt.nseg, bt.ncta, bt.cta_seg, bt.cta_row0, bt.cta_row1, bt.seg_cta0, bt.S, h->scal, bt.ndone,
                       bt.partials};

    double lmax = 0.0;
    int rc = estimate_lambda_max(h, kind, kLanczosSteps, &lmax);
    if (rc) return rc;
    const double safety = kind == INNER_SELL16 ? 1.15 : 1.10;
    const ChebCoef cc = chebyshev(lmax * safety, h->opts.chebyshev_ratio > 1.0 ? h->opts.chebyshev_ratio : 30.0, degree,
                                   h->opts.chebyshev_kind);

    auto chebyshev_steps = [&]() -> int {
        float* dcur = h->f_d0;
        float* dnext = h->f_d1;
        for (int k = 1; k < degree; ++k) {
            if (kind == INNER_SELL16)
                k_bcheb_sell<INNER_SELL16><<<T, TR, 0, s>>>(BV, V, h->sell16, h->f_dinv, h->f_res, dcur, dnext,
                                                                  h->f_y, cc.c1[k], cc.c2[k]);
            else if (kind == INNER_SELL32)
                k_bcheb_sell<INNER_SELL32><<<T, TR, 0, s>>>(BV, V, h->sell32, h->f_dinv, h->f_res, dcur, dnext,
                                                                  h->f_y, cc.c1[k], cc.c2[k]);
            else
                k_bcheb_sell<INNER_SELL64><<<T, TR, 0, s>>>(BV, V, h->sell64, h->f_dinv, h->f_res, dcur, dnext,
                                                                  h->f_y, cc.c1[k], cc.c2[k]);
            PLATO_LAUNCH_CHECK(h);
            std::swap(dcur, dnext);
        }
        return PLATO_OK;
    };

    int64_t precond_applies = 0;
    // One chunk of kChunk iterations: every parameter of its launches (pointers, Chebyshev
    // coefficients, grid) is fixed for the solve and every scalar lives on the device, so on a
    // capturable stream the chunk is captured into a CUDA graph once and replayed.
    auto enqueue_chunk = [&]() -> int {
        for (int k = 0; k < kChunk; ++k) {
            k_bfcg_apply<<<T, TR, 0, s>>>(BV, V, h->sell64, h->v_p, h->v_q);
            k_bfcg_update<<<T, TR, 0, s>>>(BV, x, h->v_r, h->v_p, h->v_q, h->f_dinv, h->f_res, h->f_d0,
                                           h->f_y, cc.c0, max_it);
            h->launches += 2;
            int r2 = chebyshev_steps();
            if (r2) return r2;
            k_bfcg_zq<<<T, TR, 0, s>>>(BV, h->f_y, h->v_z, h->v_q, 0);
            k_bfcg_direction<<<T, TR, 0, s>>>(BV, h->v_z, h->v_p, h->v_r, 0);
            h->launches += 2;
            PLATO_LAUNCH_CHECK(h);
            precond_applies += degree - 1;
        }
        return PLATO_OK;
    };
    struct ChunkGraph {
        cudaGraphExec_t exec = nullptr;
        int64_t launches = 0;
        ~ChunkGraph() { if (exec) cudaGraphExecDestroy(exec); }
    } chunk;
    const bool graphs = s != nullptr && s != cudaStreamLegacy && s != cudaStreamPerThread;

    PcgScalars init{};
    PLATO_CUDA(h, cudaMemcpyAsync(h->scal, &init, sizeof(PcgScalars), cudaMemcpyHostToDevice, s));
    PLATO_CUDA(h, cudaMemsetAsync(bt.S, 0, sizeof(SegScalars) * bt.nseg, s));
    constexpr int kMaxPasses = 1 + kMaxRestarts;  // first pass + restarts from the true residual
    cudaEvent_t* ev = h->poll_ev;
    for (int e = 0; e < 2; ++e)
        if (!ev[e]) PLATO_CUDA(h, cudaEventCreateWithFlags(&ev[e], cudaEventDisableTiming));
    int pass = 0;
    for (;; ++pass) {
        // r = b - A x; members whose (true) residual passes are done
        PLATO_CUDA(h, cudaMemsetAsync(bt.ndone, 0, sizeof(int32_t), s));
        PLATO_CUDA(h, cudaMemsetAsync(&h->scal->done, 0, sizeof(int32_t), s));
        rc = launch_sell_spmv(h, h->sell64, x, h->v_r);
        if (rc) return rc;
        k_bfcg_start<<<T, TR, 0, s>>>(BV, b, h->v_r, h->f_dinv, h->f_res, h->f_d0, h->f_y, cc.c0, tol,
                                             pass > 0 ? 1 : 0, 1.0);
        PLATO_LAUNCH_CHECK(h);
        PcgScalars* slots = h->scal_host;
        PLATO_CUDA(h, cudaMemcpyAsync(&slots[0], h->scal, sizeof(PcgScalars), cudaMemcpyDeviceToHost, s));
        PLATO_CUDA(h, cudaStreamSynchronize(s));
        if (slots[0].done || pass == kMaxPasses - 1) break;
        // z = M r, p = z, p.r
        rc = chebyshev_steps();
        if (rc) return rc;
        k_bfcg_zq<<<T, TR, 0, s>>>(BV, h->f_y, h->v_z, h->v_q, 1);
        k_bfcg_direction<<<T, TR, 0, s>>>(BV, h->v_z, h->v_p, h->v_r, 1);
        h->launches += 2;
        PLATO_LAUNCH_CHECK(h);
        int cur = 0;
        bool have_prev = false;
        for (;;) {
            if (!graphs) {
                rc = enqueue_chunk();
                if (rc) return rc;
            } else {
                if (!chunk.exec) {  // capture the chunk once per solve, replay it afterwards
                    const int64_t l0 = h->launches;
                    cudaGraph_t g = nullptr;
                    PLATO_CUDA(h, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
                    rc = enqueue_chunk();
                    const cudaError_t ce = cudaStreamEndCapture(s, &g);
                    if (rc || ce != cudaSuccess) {
                        if (g) cudaGraphDestroy(g);
                        cudaGetLastError();
                        return rc ? rc : plato_cuda_fail(h, ce, "cudaStreamEndCapture", __FILE__, __LINE__);
                    }
                    const cudaError_t ie = cudaGraphInstantiate(&chunk.exec, g, 0);
                    cudaGraphDestroy(g);
                    PLATO_CUDA(h, ie);
                    chunk.launches = h->launches - l0;
                    h->launches = l0;
                    precond_applies -= int64_t(kChunk) * (degree - 1);
                }
                PLATO_CUDA(h, cudaGraphLaunch(chunk.exec, s));
                h->launches += chunk.launches;
                precond_applies += int64_t(kChunk) * (degree - 1);
            }
            PLATO_CUDA(h, cudaMemcpyAsync(&slots[cur], h->scal, sizeof(PcgScalars), cudaMemcpyDeviceToHost, s));
            PLATO_CUDA(h, cudaEventRecord(ev[cur], s));
            if (have_prev) {
                PLATO_CUDA(h, cudaEventSynchronize(ev[cur ^ 1]));
                if (slots[cur ^ 1].done) break;
            }
            have_prev = true;
            cur ^= 1;
        }
        PLATO_CUDA(h, cudaStreamSynchronize(s));
    }
    PLATO_CUDA(h, cudaMemcpyAsync(bt.S_host, bt.S, sizeof(SegScalars) * bt.nseg, cudaMemcpyDeviceToHost, s));
    PLATO_CUDA(h, cudaStreamSynchronize(s));
    bt.last.assign(bt.nseg, plato_solve_stats{});
    plato_solve_stats agg{};
    agg.converged = 1;
    agg.status = PLATO_OK;
    for (int m = 0; m < bt.nseg; ++m) {
        const SegScalars& S = bt.S_host[m];
        plato_solve_stats& st = bt.last[m];
        st.iterations = S.iter;
        st.refinements = int32_t(precond_applies);
        st.relative_residual = S.bb > 0.0 ? std::sqrt(S.rr / S.bb) : 0.0;
        const bool ok = !S.nonfinite && S.done && (S.bb == 0.0 || st.relative_residual <= tol);
        st.converged = ok ? 1 : 0;
        st.status = S.nonfinite ? PLATO_NONFINITE : (ok ? PLATO_OK : PLATO_NOT_CONVERGED);
        agg.iterations = std::max(agg.iterations, st.iterations);
        agg.relative_residual = std::max(agg.relative_residual, S.nonfinite ? NAN : st.relative_residual);
        if (!ok) agg.converged = 0;
        if (st.status != PLATO_OK && agg.status != PLATO_NONFINITE) agg.status = st.status;
    }
    agg.refinements = int32_t(precond_applies);
    *stats = agg;
    if (agg.status == PLATO_NONFINITE)
        return plato_fail(h, PLATO_NONFINITE, "non-finite value or loss of positivity in a batch member's solve");
    if (agg.status != PLATO_OK)
        return plato_fail(h, PLATO_NOT_CONVERGED, "a batch member stopped before ||b - A x|| <= tol ||b||");
    return PLATO_OK;
}

}  // namespace plato
