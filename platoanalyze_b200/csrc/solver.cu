// Jacobi-preconditioned conjugate gradients on the device.
//
// The reference hands the solve to Trilinos AztecOO / Belos or NVIDIA AmgX
// (src/alg/PlatoAbstractSolver.hpp:38-106, src/alg/EpetraLinearSolver.cpp:253-286); none of
// those is part of the reference tree.  This is Hestenes-Stiefel CG with M = diag(A), all
// vectors, dot products and step lengths in FP64, stopping on ||r||/||b|| <= tol and then
// confirming with the recomputed residual b - A x.
//
// Per iteration three kernels run back to back on the handle's stream with no host
// round-trip: (1) block-CRS SpMV fused with the p.Ap reduction, (2) the x/r update fused
// with the Jacobi apply and the r.z and r.r reductions, (3) the search-direction update.
// The global scalars (alpha, beta, convergence) live in device memory; each reduction is
// finished by the last block to arrive (ticket counter), so there is no extra launch and no
// spin-wait.  The host polls a pinned copy of the scalars every kChunk iterations while the
// next chunk is already queued, and every kernel returns at once after convergence.
#include "plato_internal.cuh"

namespace plato {

MeshView mesh_view(const plato_problem* h);
GraphView graph_view(const plato_problem* h);
int launch_axpby(plato_problem* h, int64_t n, double a, const double* x, double b, double* y);

namespace {

constexpr int kThreads = 256;
constexpr int kChunk = 32;
constexpr int kTimingStride = 8;

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sums NV per-thread values over the block; thread 0 gets the result.
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

// Last-block-done: returns true in the block that finishes last; partials[NV*block + q]
// hold every block's sums.
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

__device__ __forceinline__ bool finite(double v) { return isfinite(v); }

// y = A x on the 3x3 block CRS, one warp per node row: lanes stream the row's 9*nb values
// contiguously (coalesced), gather x through L2, and reduce the three row sums with
// shuffles.  With S != nullptr the kernel also forms p.Ap (x = p, y = Ap) and alpha.
__global__ void __launch_bounds__(kThreads)
k_bsr_spmv(int32_t N, const int32_t* __restrict__ row_map, const int32_t* __restrict__ cols,
           const double* __restrict__ A, const double* __restrict__ x, double* __restrict__ y,
           PcgScalars* S, double* partials) {
    __shared__ double sh[1][32];
    __shared__ bool last;
    if (S && S->done) return;
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    double dot = 0.0;
    for (int64_t r = warp; r < N; r += nwarps) {
        const int32_t rs = row_map[r], re = row_map[r + 1];
        const int64_t base = 9 * (int64_t)rs, end = 9 * (int64_t)re;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        int blk = lane / 9, ij = lane - 9 * (lane / 9);
        for (int64_t t = base + lane; t < end; t += 32) {
            const int i = (ij * 11) >> 5, j = ij - 3 * i;
            const double prod = __ldg(A + t) * __ldg(x + 3 * (int64_t)__ldg(cols + rs + blk) + j);
            a0 += (i == 0) ? prod : 0.0;
            a1 += (i == 1) ? prod : 0.0;
            a2 += (i == 2) ? prod : 0.0;
            blk += 3;
            ij += 5;
            if (ij >= 9) { ij -= 9; ++blk; }
        }
        a0 = warp_sum(a0);
        a1 = warp_sum(a1);
        a2 = warp_sum(a2);
        if (lane < 3) y[3 * r + lane] = lane == 0 ? a0 : (lane == 1 ? a1 : a2);
        if (S && lane == 0) dot += x[3 * r] * a0 + x[3 * r + 1] * a1 + x[3 * r + 2] * a2;
    }
    if (!S) return;
    double v[1] = {dot};
    block_sum_n<1>(v, sh);
    if (publish_partials<1>(v, partials, &S->ticket, &last)) {
        double t[1];
        final_sums<1>(t, partials, sh);
        if (threadIdx.x == 0) {
            S->pAp = t[0];
            S->alpha = S->rz / t[0];
            if (!finite(S->alpha) || t[0] <= 0.0) { S->nonfinite = 1; S->done = 1; }
            S->ticket = 0u;
        }
    }
}

// x += alpha p; r -= alpha Ap; z = Dinv r; then r.z, r.r -> beta and the stop test.
__global__ void __launch_bounds__(kThreads)
k_pcg_update(int64_t n, double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
             const double* __restrict__ Ap, const double* __restrict__ dinv, double* __restrict__ z,
             PcgScalars* S, double* partials, int32_t max_it) {
    __shared__ double sh[2][32];
    __shared__ bool last;
    if (S->done) return;
    const double alpha = S->alpha;
    double v[2] = {0.0, 0.0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        x[i] += alpha * p[i];
        const double ri = r[i] - alpha * Ap[i];
        r[i] = ri;
        const double zi = dinv[i] * ri;
        z[i] = zi;
        v[0] += ri * zi;
        v[1] += ri * ri;
    }
    block_sum_n<2>(v, sh);
    if (publish_partials<2>(v, partials, &S->ticket, &last)) {
        double t[2];
        final_sums<2>(t, partials, sh);
        if (threadIdx.x == 0) {
            S->beta = t[0] / S->rz;
            S->rz_new = t[0];
            S->rz = t[0];
            S->rr = t[1];
            S->iter += 1;
            if (!finite(t[0]) || !finite(t[1])) { S->nonfinite = 1; S->done = 1; }
            if (t[1] <= S->tol2 || S->iter >= max_it) S->done = 1;
            S->ticket = 0u;
        }
    }
}

__global__ void __launch_bounds__(kThreads)
k_pcg_direction(int64_t n, const double* __restrict__ z, double* __restrict__ p, const PcgScalars* S) {
    if (S->done) return;
    const double beta = S->beta;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        p[i] = z[i] + beta * p[i];
}

// r = b - Ax (Ax already in r_in_Ax); z = Dinv r; p = z; sums r.z, r.r, b.b -> init scalars.
__global__ void __launch_bounds__(kThreads)
k_pcg_start(int64_t n, const double* __restrict__ b, double* __restrict__ r, const double* __restrict__ dinv,
            double* __restrict__ z, double* __restrict__ p, PcgScalars* S, double* partials, double tol,
            int keep_bb) {
    __shared__ double sh[3][32];
    __shared__ bool last;
    double v[3] = {0.0, 0.0, 0.0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double ri = b[i] - r[i];
        r[i] = ri;
        const double zi = dinv[i] * ri;
        z[i] = zi;
        p[i] = zi;
        v[0] += ri * zi;
        v[1] += ri * ri;
        v[2] += b[i] * b[i];
    }
    block_sum_n<3>(v, sh);
    if (publish_partials<3>(v, partials, &S->ticket, &last)) {
        double t[3];
        final_sums<3>(t, partials, sh);
        if (threadIdx.x == 0) {
            S->rz = t[0];
            S->rr = t[1];
            if (!keep_bb) {
                S->bb = t[2];
                S->tol2 = tol * tol * t[2];
                S->iter = 0;
            }
            S->nonfinite = (!finite(t[0]) || !finite(t[1]) || !finite(t[2])) ? 1 : 0;
            S->done = (t[1] <= S->tol2 || S->nonfinite) ? 1 : 0;
            S->ticket = 0u;
        }
    }
}

__global__ void k_jacobi_from_blocks(int32_t N, const int32_t* __restrict__ diag, const double* __restrict__ A,
                                     double* __restrict__ dinv) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < 3 * (int64_t)N;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t a = t / 3;
        const int d = int(t - 3 * a);
        dinv[t] = 1.0 / A[9 * (int64_t)diag[a] + 4 * d];
    }
}

__global__ void __launch_bounds__(kThreads)
k_dot(int64_t n, const double* __restrict__ a, const double* __restrict__ b, double* partials,
      unsigned int* ticket, double* result) {
    __shared__ double sh[1][32];
    __shared__ bool last;
    double v[1] = {0.0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        v[0] += a[i] * b[i];
    block_sum_n<1>(v, sh);
    if (publish_partials<1>(v, partials, ticket, &last)) {
        double t[1];
        final_sums<1>(t, partials, sh);
        if (threadIdx.x == 0) {
            *result = t[0];
            *ticket = 0u;
        }
    }
}

}  // namespace

// a.b into *host_result (synchronises the stream).
int launch_dot(plato_problem* h, const double* a, const double* b, int64_t n, double* host_result) {
    const int blocks = grid_for(n, kThreads, h->partials_len);
    k_dot<<<blocks, kThreads, 0, h->stream>>>(n, a, b, h->partials, h->red_ticket, h->red_out);
    PLATO_LAUNCH_CHECK(h);
    PLATO_CUDA(h, cudaMemcpyAsync(host_result, h->red_out, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    PLATO_CUDA(h, cudaStreamSynchronize(h->stream));
    return PLATO_OK;
}


#define RC_(expr)              \
    do {                       \
        int _rc = (expr);      \
        if (_rc) return _rc;   \
    } while (0)

// Event pairs for the sampled operator timings (reused across solves).
int timing_events(plato_problem* h, cudaEvent_t* e0, cudaEvent_t* e1) {
    while ((int)h->ev_pool.size() < h->ev_used + 2) {
        cudaEvent_t e;
        PLATO_CUDA(h, cudaEventCreate(&e));
        h->ev_pool.push_back(e);
    }
    *e0 = h->ev_pool[h->ev_used];
    *e1 = h->ev_pool[h->ev_used + 1];
    h->ev_used += 2;
    return PLATO_OK;
}

// Adds the durations of the timed applies that belonged to executed iterations.
int collect_timing(plato_problem* h, const std::vector<int64_t>& iters, int64_t executed) {
    for (size_t k = 0; k < iters.size(); ++k) {
        if (iters[k] >= executed) break;
        float ms = 0.f;
        PLATO_CUDA(h, cudaEventElapsedTime(&ms, h->ev_pool[2 * k], h->ev_pool[2 * k + 1]));
        h->op_ms_total += ms;
        h->op_timed += 1;
    }
    h->ev_used = 0;
    return PLATO_OK;
}

int launch_spmv(plato_problem* h, const double* A, const double* x, double* y) {
    const int blocks = grid_for((int64_t)h->N * 32, kThreads, 148 * 16);
    k_bsr_spmv<<<blocks, kThreads, 0, h->stream>>>(h->N, h->row_map, h->cols, A, x, y, nullptr, nullptr);
    PLATO_LAUNCH_CHECK(h);
    return PLATO_OK;
}

int launch_jacobi(plato_problem* h, const double* A, double* dinv) {
    k_jacobi_from_blocks<<<grid_for(3 * (int64_t)h->N, kThreads), kThreads, 0, h->stream>>>(h->N, h->diag, A, dinv);
    PLATO_LAUNCH_CHECK(h);
    return PLATO_OK;
}

// Solves A x = b (A assembled, constrained).  x holds the initial guess.
int pcg_fp64_assembled(plato_problem* h, const double* A, const double* b, double* x,
                       plato_solve_stats* stats) {
    const int64_t n = 3 * (int64_t)h->N;
    cudaStream_t s = h->stream;
    const double tol = h->opts.tolerance;
    const int32_t max_it = h->opts.max_iterations;
    const int vec_blocks = grid_for(n, kThreads, 148 * 16);
    const int spmv_blocks = grid_for((int64_t)h->N * 32, kThreads, 148 * 16);
    if (vec_blocks * 3 > h->partials_len || spmv_blocks > h->partials_len)
        return plato_fail(h, PLATO_BAD_INPUT, "reduction scratch too small");
    int rc = launch_jacobi(h, A, h->v_dinv);
    if (rc) return rc;

    PcgScalars init{};
    init.tol2 = 0.0;
    PLATO_CUDA(h, cudaMemcpyAsync(h->scal, &init, sizeof(PcgScalars), cudaMemcpyHostToDevice, s));

    int32_t restarts = 0;
    int32_t iter_base = 0;
    bool keep_bb = false;
    for (;;) {
        // r = b - A x ; z = Dinv r ; p = z
        rc = launch_spmv(h, A, x, h->v_r);
        if (rc) return rc;
        k_pcg_start<<<vec_blocks, kThreads, 0, s>>>(n, b, h->v_r, h->v_dinv, h->v_z, h->v_p, h->scal,
                                                     h->partials, tol, keep_bb ? 1 : 0);
        PLATO_LAUNCH_CHECK(h);
        // iterate in chunks; poll the scalars of the previous chunk while the next one runs
        PcgScalars* slots = h->scal_host;
        int64_t enqueued = 0;
        std::vector<int64_t> timed_iters;
        h->ev_used = 0;
        int cur = 0;
        bool have_prev = false;
        cudaEvent_t ev[2];
        PLATO_CUDA(h, cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
        PLATO_CUDA(h, cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
        for (;;) {
            for (int k = 0; k < kChunk; ++k, ++enqueued) {
                const bool timed = h->timing && (enqueued % kTimingStride) == 0;
                cudaEvent_t e0 = nullptr, e1 = nullptr;
                if (timed) {
                    RC_(timing_events(h, &e0, &e1));
                    timed_iters.push_back(enqueued);
                    PLATO_CUDA(h, cudaEventRecord(e0, s));
                }
                k_bsr_spmv<<<spmv_blocks, kThreads, 0, s>>>(h->N, h->row_map, h->cols, A, h->v_p, h->v_Ap,
                                                            h->scal, h->partials);
                if (timed) PLATO_CUDA(h, cudaEventRecord(e1, s));
                k_pcg_update<<<vec_blocks, kThreads, 0, s>>>(n, x, h->v_r, h->v_p, h->v_Ap, h->v_dinv, h->v_z,
                                                             h->scal, h->partials, max_it);
                k_pcg_direction<<<vec_blocks, kThreads, 0, s>>>(n, h->v_z, h->v_p, h->scal);
            }
            h->launches += 3 * kChunk - 1;
            PLATO_LAUNCH_CHECK(h);
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
        cudaEventDestroy(ev[0]);
        cudaEventDestroy(ev[1]);
        PcgScalars fin;
        PLATO_CUDA(h, cudaMemcpy(&fin, h->scal, sizeof(PcgScalars), cudaMemcpyDeviceToHost));
        RC_(collect_timing(h, timed_iters, fin.iter - iter_base));
        iter_base = fin.iter;
        if (fin.nonfinite) {
            stats->iterations = fin.iter;
            stats->refinements = 1;
            stats->relative_residual = NAN;
            stats->converged = 0;
            stats->status = PLATO_NONFINITE;
            return plato_fail(h, PLATO_NONFINITE, "non-finite value in the conjugate-gradient recurrences");
        }
        // true residual check: r = b - A x
        rc = launch_spmv(h, A, x, h->v_Ap);
        if (rc) return rc;
        rc = launch_axpby(h, n, 1.0, b, 0.0, h->v_r);
        if (rc) return rc;
        rc = launch_axpby(h, n, -1.0, h->v_Ap, 1.0, h->v_r);
        if (rc) return rc;
        double rr = 0.0;
        rc = launch_dot(h, h->v_r, h->v_r, n, &rr);
        if (rc) return rc;
        const double rel = fin.bb > 0.0 ? sqrt(rr / fin.bb) : 0.0;
        stats->iterations = fin.iter;
        stats->refinements = 1;
        stats->relative_residual = rel;
        if (rel <= tol || fin.bb == 0.0) {
            stats->converged = 1;
            stats->status = PLATO_OK;
            return PLATO_OK;
        }
        if (fin.iter >= max_it || restarts >= 3) {
            stats->converged = 0;
            stats->status = PLATO_NOT_CONVERGED;
            return plato_fail(h, PLATO_NOT_CONVERGED, "PCG reached max_iterations without meeting the tolerance");
        }
        // the recurrence drifted from the true residual: restart from the current x
        ++restarts;
        keep_bb = true;
        PcgScalars cont = fin;
        cont.done = 0;
        PLATO_CUDA(h, cudaMemcpyAsync(h->scal, &cont, sizeof(PcgScalars), cudaMemcpyHostToDevice, s));
    }
}

}  // namespace plato
