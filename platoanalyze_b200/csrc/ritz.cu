// Initial guess from a subspace (no reference counterpart; used by the learned warm start).
//
// Given k <= kMaxRitz columns W (3N each) and the constrained system A x = b with initial
// iterate x, the Galerkin (Ritz) correction on span(P W) - P zeroes the constrained dofs so
// the correction keeps their values - minimises the A-norm error over x + span(P W):
//   r = b - A x,  (W^T P A P W) c = W^T P r,  x <- x + P W c.
// All products and dots are FP64 on the solver's SELL copy of A; the k x k system is solved
// on the host (Cholesky).  The correction lowers the energy (1/2) x^T A x - b^T x by
// (1/2) c^T G c >= 0, so the A-norm error never grows; it is dropped - x stays the caller's
// initial guess - when G is not numerically positive definite or the new residual is not
// finite or grows past kResidualGuard times the old one (a guess with node-scale noise has a
// residual far above ||b|| and gains the solver nothing).
//
// Deflation (plato_problem_solution_deflated): after the Galerkin guess the residual is
// orthogonal to span(P W), and the Krylov solver keeps it so by making every new search
// direction A-orthogonal to P W (deflated CG: Saad, Yeung, Erhel, Guyomarc'h, SIAM J. Sci.
// Comput. 21, 2000): p <- p - P W mu with mu = G^-1 (A P W)^T p, G = W^T P A P W.  Two launches
// per iteration (the k dot products with mu in the last block; the update with the new p.r
// for the flexible CG); W, A P W and G^-1 stay on the device for the solve.
#include <algorithm>
#include <cmath>
#include <vector>

#include "plato_internal.cuh"
#include "solver_common.cuh"

namespace plato {

int launch_sell_spmv(plato_problem* h, const double* vals, const double* x, double* y);
int launch_dot(plato_problem* h, const double* a, const double* b, int64_t n, double* host_result);

namespace {

constexpr int kMaxRitz = 8;
constexpr double kResidualGuard = 10.0;

// Wm[j] = (1 - mask) W[j]
__global__ void k_mask_columns(int64_t n, int k, const uint8_t* __restrict__ mask, const double* __restrict__ W,
                               double* __restrict__ Wm) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        for (int j = 0; j < k; ++j) Wm[j * n + i] = mask[i] ? 0.0 : W[j * n + i];
}

// Block partials of W_i . Q_j (i <= j) and W_i . r, in a fixed order per block.
__global__ void __launch_bounds__(kThreads)
k_ritz_dots(int64_t n, int k, const double* __restrict__ W, const double* __restrict__ Q, const double* __restrict__ r,
            double* __restrict__ partials) {
    __shared__ double sh[1][32];
    const int npair = k * (k + 1) / 2 + k;
    for (int q = 0; q < npair; ++q) {
        int i = 0, j = 0;
        if (q < k * (k + 1) / 2) {
            int t = q;
            while (t >= k - i) { t -= k - i; ++i; }
            j = i + t;
        } else {
            i = q - k * (k + 1) / 2;
        }
        const double* a = W + int64_t(i) * n;
        const double* b = q < k * (k + 1) / 2 ? Q + int64_t(j) * n : r;
        double v[1] = {0.0};
        for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n; e += int64_t(gridDim.x) * blockDim.x)
            v[0] += a[e] * b[e];
        block_sum_n<1>(v, sh);
        if (threadIdx.x == 0) partials[int64_t(q) * gridDim.x + blockIdx.x] = v[0];
    }
}

// x += sum_j c_j W_j; rnew = r - sum_j c_j Q_j; partial sums of rnew.rnew
__global__ void __launch_bounds__(kThreads)
k_ritz_update(int64_t n, int k, const double* __restrict__ W, const double* __restrict__ Q, double* __restrict__ x,
              const double* __restrict__ r, double* __restrict__ rnew, const double* __restrict__ c,
              double* __restrict__ partials) {
    __shared__ double sh[1][32];
    double v[1] = {0.0};
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n; e += int64_t(gridDim.x) * blockDim.x) {
        double dx = 0.0, dr = 0.0;
        for (int j = 0; j < k; ++j) {
            dx += c[j] * W[j * n + e];
            dr += c[j] * Q[j * n + e];
        }
        x[e] += dx;
        const double ri = r[e] - dr;
        rnew[e] = ri;
        v[0] += ri * ri;
    }
    block_sum_n<1>(v, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = v[0];
}

// mu = Ginv (Q^T p): block partials of the k dot products, finished by the last block.
__global__ void __launch_bounds__(kThreads)
k_deflate_mu(int64_t n, int k, const double* __restrict__ Q, const double* __restrict__ p,
             const double* __restrict__ Ginv, double* __restrict__ mu, PcgScalars* S, double* partials) {
    __shared__ double sh[kMaxRitz][32];
    __shared__ bool last;
    if (S->done) return;
    double v[kMaxRitz];
#pragma unroll
    for (int j = 0; j < kMaxRitz; ++j) v[j] = 0.0;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n; e += int64_t(gridDim.x) * blockDim.x) {
        const double pe = p[e];
#pragma unroll
        for (int j = 0; j < kMaxRitz; ++j)
            if (j < k) v[j] += Q[j * n + e] * pe;
    }
    block_sum_n<kMaxRitz>(v, sh);
    if (publish_partials<kMaxRitz>(v, partials, &S->ticket, &last)) {
        double t[kMaxRitz];
        final_sums<kMaxRitz>(t, partials, sh);
        if (threadIdx.x == 0) {
            for (int i = 0; i < k; ++i) {
                double m = 0.0;
                for (int j = 0; j < k; ++j) m += Ginv[i * k + j] * t[j];
                mu[i] = m;
            }
            S->ticket = 0u;
        }
    }
}

// p -= W mu; with update_pr also p.r into S->rz (the flexible CG's numerator of alpha).
__global__ void __launch_bounds__(kThreads)
k_deflate_apply(int64_t n, int k, const double* __restrict__ W, const double* __restrict__ mu, double* __restrict__ p,
                const double* __restrict__ r, PcgScalars* S, double* partials, int update_pr) {
    __shared__ double sh[1][32];
    __shared__ bool last;
    if (S->done) return;
    double m[kMaxRitz];
#pragma unroll
    for (int j = 0; j < kMaxRitz; ++j) m[j] = j < k ? mu[j] : 0.0;
    double v[1] = {0.0};
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n; e += int64_t(gridDim.x) * blockDim.x) {
        double pe = p[e];
#pragma unroll
        for (int j = 0; j < kMaxRitz; ++j)
            if (j < k) pe -= W[j * n + e] * m[j];
        p[e] = pe;
        if (update_pr) v[0] += pe * r[e];
    }
    if (!update_pr) return;
    block_sum_n<1>(v, sh);
    if (publish_partials<1>(v, partials, &S->ticket, &last)) {
        double t[1];
        final_sums<1>(t, partials, sh);
        if (threadIdx.x == 0) {
            S->rz = t[0];
            if (!isfinite(t[0])) { S->nonfinite = 1; S->done = 1; }
            S->ticket = 0u;
        }
    }
}

__global__ void k_residual(int64_t n, const double* __restrict__ b, const double* __restrict__ Ax,
                           double* __restrict__ r) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        r[i] = b[i] - Ax[i];
}

// dense SPD solve (Cholesky), false when the matrix is not numerically positive definite
bool cholesky_solve(std::vector<double> A, int k, std::vector<double>& x) {
    double scale = 0.0;
    for (int i = 0; i < k; ++i) scale = std::max(scale, A[i * k + i]);
    if (!(scale > 0.0)) return false;
    for (int j = 0; j < k; ++j) {
        double d = A[j * k + j];
        for (int p = 0; p < j; ++p) d -= A[j * k + p] * A[j * k + p];
        if (!(d > 1e-14 * scale)) return false;
        d = std::sqrt(d);
        A[j * k + j] = d;
        for (int i = j + 1; i < k; ++i) {
            double s = A[i * k + j];
            for (int p = 0; p < j; ++p) s -= A[i * k + p] * A[j * k + p];
            A[i * k + j] = s / d;
        }
    }
    for (int i = 0; i < k; ++i) {
        double s = x[i];
        for (int p = 0; p < i; ++p) s -= A[i * k + p] * x[p];
        x[i] = s / A[i * k + i];
    }
    for (int i = k - 1; i >= 0; --i) {
        double s = x[i];
        for (int p = i + 1; p < k; ++p) s -= A[p * k + i] * x[p];
        x[i] = s / A[i * k + i];
    }
    return true;
}

}  // namespace

// x <- x + P W c on the prepared SELL operator (h->sell64); W = h->ritz_W (k columns).
int ritz_guess(plato_problem* h, const double* b, double* x) {
    const int k = h->ritz_k;
    if (k <= 0 || !h->ritz_W) return PLATO_OK;
    if (k > kMaxRitz) return plato_fail(h, PLATO_BAD_INPUT, "at most 8 subspace columns");
    const int64_t n = 3 * int64_t(h->N);
    cudaStream_t s = h->stream;
    const size_t need = size_t(2 * k + 2) * size_t(n);
    if (h->ritz_scratch_len < need) {
        if (h->ritz_scratch) cudaFree(h->ritz_scratch);
        h->ritz_scratch = nullptr;
        h->ritz_scratch_len = 0;
        PLATO_CUDA(h, cudaMalloc(&h->ritz_scratch, sizeof(double) * need));
        h->ritz_scratch_len = need;
    }
    double* Wm = h->ritz_scratch;             // k columns
    double* Q = Wm + int64_t(k) * n;          // k columns: A P W
    double* r = Q + int64_t(k) * n;           // b - A x
    double* rn = r + n;                       // residual after the correction
    const int npair = k * (k + 1) / 2 + k;
    const int64_t capacity = 4 * int64_t(h->partials_len) - kMaxRitz;  // the tail holds the coefficients
    const int VB = grid_for(n, kThreads, std::min<int64_t>(148 * 8, capacity / npair));
    k_mask_columns<<<VB, kThreads, 0, s>>>(n, k, h->bc_mask, h->ritz_W, Wm);
    PLATO_LAUNCH_CHECK(h);
    int rc = launch_sell_spmv(h, h->sell64, x, rn);
    if (rc) return rc;
    k_residual<<<VB, kThreads, 0, s>>>(n, b, rn, r);
    PLATO_LAUNCH_CHECK(h);
    for (int j = 0; j < k; ++j) {
        rc = launch_sell_spmv(h, h->sell64, Wm + int64_t(j) * n, Q + int64_t(j) * n);
        if (rc) return rc;
    }
    std::vector<double> part(size_t(npair) * VB), host_rr(VB);
    k_ritz_dots<<<VB, kThreads, 0, s>>>(n, k, Wm, Q, r, h->partials);
    PLATO_LAUNCH_CHECK(h);
    PLATO_CUDA(h, cudaMemcpyAsync(part.data(), h->partials, sizeof(double) * npair * VB, cudaMemcpyDeviceToHost, s));
    PLATO_CUDA(h, cudaStreamSynchronize(s));
    std::vector<double> G(size_t(k) * k), c(k);
    int q = 0;
    for (int i = 0; i < k; ++i)
        for (int j = i; j < k; ++j, ++q) {
            double t = 0.0;
            for (int bk = 0; bk < VB; ++bk) t += part[size_t(q) * VB + bk];
            G[i * k + j] = G[j * k + i] = t;
        }
    for (int i = 0; i < k; ++i, ++q) {
        double t = 0.0;
        for (int bk = 0; bk < VB; ++bk) t += part[size_t(q) * VB + bk];
        c[i] = t;
    }
    std::vector<double> Gram = G;
    if (!cholesky_solve(G, k, c)) return PLATO_OK;  // degenerate subspace: keep x
    double rr0 = 0.0;
    rc = launch_dot(h, r, r, n, &rr0);
    if (rc) return rc;
    // the update on a copy of x, kept only if the residual stays within the guard
    double* cd = h->partials + capacity;  // the k coefficients
    PLATO_CUDA(h, cudaMemcpyAsync(cd, c.data(), sizeof(double) * k, cudaMemcpyHostToDevice, s));
    PLATO_CUDA(h, cudaMemcpyAsync(h->v_tmp, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    k_ritz_update<<<VB, kThreads, 0, s>>>(n, k, Wm, Q, h->v_tmp, r, rn, cd, h->partials);
    PLATO_LAUNCH_CHECK(h);
    PLATO_CUDA(h, cudaMemcpyAsync(host_rr.data(), h->partials, sizeof(double) * VB, cudaMemcpyDeviceToHost, s));
    PLATO_CUDA(h, cudaStreamSynchronize(s));
    double rr1 = 0.0;
    for (int bk = 0; bk < VB; ++bk) rr1 += host_rr[bk];
    h->ritz_rel_gain = rr0 > 0.0 ? std::sqrt(rr1 / rr0) : 1.0;
    // the residual guard protects a plain guess; deflated CG needs the Galerkin guess (it lowers
    // the energy error whatever the residual does), so with deflation only finiteness counts
    const bool keep = std::isfinite(rr1) && (h->ritz_deflate || rr1 <= kResidualGuard * kResidualGuard * rr0);
    if (keep)
        PLATO_CUDA(h, cudaMemcpyAsync(x, h->v_tmp, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    else
        h->ritz_rel_gain = 1.0;
    // deflation needs the Galerkin guess (residual orthogonal to P W): G^-1 column by column
    if (h->ritz_deflate && keep) {
        std::vector<double> Ginv(size_t(k) * k);
        for (int j = 0; j < k; ++j) {
            std::vector<double> e(k, 0.0);
            e[j] = 1.0;
            if (!cholesky_solve(Gram, k, e)) return PLATO_OK;
            for (int i = 0; i < k; ++i) Ginv[i * k + j] = e[i];
        }
        if (!h->ritz_small) PLATO_CUDA(h, cudaMalloc(&h->ritz_small, sizeof(double) * (kMaxRitz * kMaxRitz + kMaxRitz)));
        PLATO_CUDA(h, cudaMemcpyAsync(h->ritz_small, Ginv.data(), sizeof(double) * k * k, cudaMemcpyHostToDevice, s));
        PLATO_CUDA(h, cudaStreamSynchronize(s));
        h->ritz_deflating = 1;
    }
    return PLATO_OK;
}

// One deflation of the search direction p (see the file comment); update_pr recomputes p.r.
int deflate_direction(plato_problem* h, double* p, const double* r, int update_pr) {
    if (!h->ritz_deflating) return PLATO_OK;
    const int k = h->ritz_k;
    const int64_t n = 3 * int64_t(h->N);
    double* Wm = h->ritz_scratch;
    double* Q = Wm + int64_t(k) * n;
    const int VB = grid_for(n, kThreads, 148 * 8);
    double* Ginv = h->ritz_small;
    double* mu = h->ritz_small + kMaxRitz * kMaxRitz;
    k_deflate_mu<<<VB, kThreads, 0, h->stream>>>(n, k, Q, p, Ginv, mu, h->scal, h->partials);
    PLATO_LAUNCH_CHECK(h);
    k_deflate_apply<<<VB, kThreads, 0, h->stream>>>(n, k, Wm, mu, p, r, h->scal, h->partials, update_pr);
    PLATO_LAUNCH_CHECK(h);
    return PLATO_OK;
}

}  // namespace plato
