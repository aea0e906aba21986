// Two-level preconditioner: trilinear coarse space on a box grid and its Galerkin operator.
//
// Coarse space Z (3N x 3Nc): a box grid of nc[0] x nc[1] x nc[2] cells over the mesh
// bounding box; fine dof (p, d) = sum over the 8 corners J of p's cell of phi_J(x_p) U_(J,d),
// phi_J trilinear; constrained fine dofs are masked out (P Z), so the coarse space never
// moves a clamped dof.  The coarse operator is exactly Galerkin, E = (PZ)^T K (PZ), assembled
// element by element: with every element inside one coarse cell, the coarse basis restricted
// to an element is the linear interpolant of its nodal values, whose gradient is
// G_J^(d) = sum_a m_(a,d) phi_J(x_a) grad N_a, so E gets
// vol s(rho) (lambda G_J^(i)_i G_L^(j)_j + mu G_J^(i)_j G_L^(j)_i + mu delta_ij G_J^(i).G_L^(i))
// from each element (the isotropic block formula with coarse gradients).
//
// Per solve: the elements of each coarse cell are split over about eight CTAs per SM; each
// CTA stages batches of elements' coarse gradients in shared memory and accumulates its
// share of the cell's symmetric 24x24 block in registers (as a rank-k update of the
// gradients for the elements whose nodes are free or fully clamped, entry by entry for the
// rest), then adds it to E.  E is factored (blocked Cholesky, 64x64 tiles; each diagonal
// tile's inverse is formed as it is factored, so the panels are tile products) and L is
// inverted by doubling (batched 64x64 tile products), so a coarse solve in the iteration is
// two triangular matrix-vector products with X = L^-1 and its transpose.
// Per preconditioner call: restriction in two deterministic passes (per-cell partial sums by
// split CTAs, then a fixed-order sum per coarse dof), y_c = X^T (X r_c) with X = L^-1 (two
// triangular matrix-vector products, warp per row), prolongation (thread per fine node).
#include <algorithm>
#include <mutex>

#include <cub/cub.cuh>

#include "plato_internal.cuh"

namespace plato {

GraphView graph_view(const plato_problem* h);

namespace {

constexpr int kBatch = 32;     // elements staged per Galerkin batch (8 threads each)
constexpr int kThreadsPerCta = 256;

struct CoarseView {
    int nc0, nc1, nc2;
    double x0, y0, z0, hx, hy, hz;
    double ihx, ihy, ihz;  // 1 / h: local coordinates of the hot kernels are (x - lo) * ih
};

__host__ __device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

__device__ __forceinline__ void cell_of(const CoarseView& cv, double x, double y, double z, int& cx, int& cy,
                                        int& cz) {
    cx = clampi(int(floor((x - cv.x0) / cv.hx)), 0, cv.nc0 - 1);
    cy = clampi(int(floor((y - cv.y0) / cv.hy)), 0, cv.nc1 - 1);
    cz = clampi(int(floor((z - cv.z0) / cv.hz)), 0, cv.nc2 - 1);
}

__device__ __forceinline__ int cell_id(const CoarseView& cv, int cx, int cy, int cz) {
    return (cx * cv.nc1 + cy) * cv.nc2 + cz;
}

__device__ __forceinline__ int coarse_node(const CoarseView& cv, int ix, int iy, int iz) {
    return (ix * (cv.nc1 + 1) + iy) * (cv.nc2 + 1) + iz;
}

// trilinear weight of corner (bx,by,bz) at local coordinates (u,v,w)
__device__ __forceinline__ double corner_weight(int b, double u, double v, double w) {
    return ((b & 4) ? u : 1.0 - u) * ((b & 2) ? v : 1.0 - v) * ((b & 1) ? w : 1.0 - w);
}

__global__ void k_node_keys(int32_t N, const double* __restrict__ coords, CoarseView cv, uint32_t* __restrict__ key,
                            int32_t* __restrict__ val, int32_t* __restrict__ count) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        int cx, cy, cz;
        cell_of(cv, coords[3 * p], coords[3 * p + 1], coords[3 * p + 2], cx, cy, cz);
        const int c = cell_id(cv, cx, cy, cz);
        key[p] = uint32_t(c);
        val[p] = int32_t(p);
        atomicAdd(&count[c], 1);
    }
}

// cell of an element = cell of its centroid; flags elements with a node outside that cell.
// key = 2 cell + 1 when some node of the element has its three dofs constrained unalike
// (those take the general Galerkin kernel), 2 cell otherwise.
__global__ void k_elem_keys(int32_t C, const int4* __restrict__ conn, const double* __restrict__ coords, CoarseView cv,
                            const uint8_t* __restrict__ mask, uint32_t* __restrict__ key, int32_t* __restrict__ val,
                            int32_t* __restrict__ count, int32_t* __restrict__ bad) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < C; e += (int64_t)gridDim.x * blockDim.x) {
        const int4 n = conn[e];
        double x[4][3];
        load_cell_coords(coords, n, x);
        double c[3] = {0, 0, 0};
        for (int a = 0; a < 4; ++a)
            for (int d = 0; d < 3; ++d) c[d] += 0.25 * x[a][d];
        int cx, cy, cz;
        cell_of(cv, c[0], c[1], c[2], cx, cy, cz);
        const double lo[3] = {cv.x0 + cx * cv.hx, cv.y0 + cy * cv.hy, cv.z0 + cz * cv.hz};
        const double hh[3] = {cv.hx, cv.hy, cv.hz};
        for (int a = 0; a < 4; ++a)
            for (int d = 0; d < 3; ++d) {
                const double t = (x[a][d] - lo[d]) / hh[d];
                if (t < -1e-9 || t > 1.0 + 1e-9) atomicExch(bad, 1);
            }
        const int ids[4] = {n.x, n.y, n.z, n.w};
        int mixed = 0;
        for (int a = 0; a < 4; ++a) {
            const uint8_t* m = mask + 3 * (int64_t)ids[a];
            mixed |= (m[0] != m[1]) || (m[0] != m[2]);
        }
        const int k = 2 * cell_id(cv, cx, cy, cz) + mixed;
        key[e] = uint32_t(k);
        val[e] = int32_t(e);
        atomicAdd(&count[k], 1);
    }
}

// Upper-triangle entry t (row-major) of a 24x24 matrix -> (r, c), r <= c.
__device__ __forceinline__ void upper_entry(int t, int& r, int& c) {
    r = 0;
    while (t >= 24 - r) { t -= 24 - r; ++r; }
    c = r + t;
}

// Common path: for an element whose nodes are each either free or fully clamped, the coarse
// gradient is one vector per corner, g_J = sum over free nodes a of phi_J(x_a) grad N_a, and
// every entry of the cell's 24 x 24 block of E is a fixed combination of
//   M = sum_e w_e g g^T   (g = (g_0, ..., g_7), 24 values; w_e = vol s(rho))
// E_(J,i),(L,j) = lam M_(Ji),(Lj) + mu M_(Jj),(Li) + mu delta_ij sum_k M_(Jk),(Lk).
// M is a symmetric rank-k update: CTA (cell, split) stages kFastBatch elements' (w, g) in
// shared memory (one thread per element), then 250 threads accumulate the ten upper 6 x 6
// tiles of M in registers, each over a fixed slice of the batch (25 slices); the slices are
// summed in shared memory, the block formula applied, and the upper triangle added to E
// (mirrored) once per CTA.
constexpr int kFastBatch = 256;
constexpr int kSlices = 25;

__global__ void __launch_bounds__(kThreadsPerCta, 2)
k_galerkin_fast(CoarseView cv, int split, const int32_t* __restrict__ elem_ptr, const int32_t* __restrict__ elem_list,
                const int4* __restrict__ conn, const double* __restrict__ coords, const double* __restrict__ z,
                Material mat, const uint8_t* __restrict__ mask, int n, double* __restrict__ E) {
    extern __shared__ double smem[];
    double* Gs = smem;                       // [kFastBatch][25]: w, then g (24)
    double* Red = smem;                      // [kSlices][10][36] after the last batch
    double* Ms = smem + kSlices * 10 * 36;   // [24][24]
    const double lam = mat.c01, mu = mat.c33;
    const int cell = blockIdx.x / split, part = blockIdx.x - cell * split;
    const int cz = cell % cv.nc2, cy = (cell / cv.nc2) % cv.nc1, cx = cell / (cv.nc1 * cv.nc2);
    const double lo[3] = {cv.x0 + cx * cv.hx, cv.y0 + cy * cv.hy, cv.z0 + cz * cv.hz};
    const int q0 = elem_ptr[2 * cell], q1 = elem_ptr[2 * cell + 1];
    const int chunk = (q1 - q0 + split - 1) / split;
    const int e0 = q0 + part * chunk, e1 = min(q1, e0 + chunk);
    const int tid = threadIdx.x;
    // tile t of the upper 4 x 4 grid of 6 x 6 tiles: (ti, tj), ti <= tj
    const int tile = tid % 10, slice = tid / 10;
    int ti = 0, tj = tile;
    while (tj >= 4 - ti) { tj -= 4 - ti; ++ti; }
    tj += ti;
    double acc[36];
#pragma unroll
    for (int q = 0; q < 36; ++q) acc[q] = 0.0;
    for (int base = e0; base < e1; base += kFastBatch) {
        const int nb = min(kFastBatch, e1 - base);
        if (tid < nb) {
            const int32_t cell = elem_list[base + tid];
            const int4 nd = conn[cell];
            double x[4][3];
            load_cell_coords(coords, nd, x);
            TetGeom<double> G;
            tet_geometry(x, G);
            const double rho = cell_rho(mat, z, cell, nd);
            double* row = Gs + tid * 25;
            row[0] = G.vol * simp(mat, rho);
            const int ids[4] = {nd.x, nd.y, nd.z, nd.w};
            double uvw[4][3];
            bool freeN[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                uvw[a][0] = (x[a][0] - lo[0]) * cv.ihx;
                uvw[a][1] = (x[a][1] - lo[1]) * cv.ihy;
                uvw[a][2] = (x[a][2] - lo[2]) * cv.ihz;
                freeN[a] = mask[3 * (int64_t)ids[a]] == 0;
            }
#pragma unroll
            for (int J = 0; J < 8; ++J) {
                double gj[3] = {0.0, 0.0, 0.0};
#pragma unroll
                for (int a = 0; a < 4; ++a) {
                    if (!freeN[a]) continue;
                    const double wa = corner_weight(J, uvw[a][0], uvw[a][1], uvw[a][2]);
                    gj[0] += wa * G.g[a][0];
                    gj[1] += wa * G.g[a][1];
                    gj[2] += wa * G.g[a][2];
                }
                row[1 + 3 * J] = gj[0];
                row[2 + 3 * J] = gj[1];
                row[3 + 3 * J] = gj[2];
            }
        }
        __syncthreads();
        if (slice < kSlices) {
            for (int e = slice; e < nb; e += kSlices) {
                const double* row = Gs + e * 25;
                const double w = row[0];
                double a[6], b[6];
#pragma unroll
                for (int q = 0; q < 6; ++q) {
                    a[q] = w * row[1 + 6 * ti + q];
                    b[q] = row[1 + 6 * tj + q];
                }
#pragma unroll
                for (int r = 0; r < 6; ++r)
#pragma unroll
                    for (int c = 0; c < 6; ++c) acc[6 * r + c] += a[r] * b[c];
            }
        }
        __syncthreads();
    }
    if (e0 >= e1) return;  // uniform across the CTA: nothing staged, nothing to add
    if (slice < kSlices)
#pragma unroll
        for (int q = 0; q < 36; ++q) Red[(slice * 10 + tile) * 36 + q] = acc[q];
    __syncthreads();
    // M (full 24 x 24) from the slice sums of the upper tiles
    for (int t = tid; t < 360; t += blockDim.x) {
        const int tl = t / 36, q = t - 36 * tl;
        double sum = 0.0;
        for (int sl = 0; sl < kSlices; ++sl) sum += Red[(sl * 10 + tl) * 36 + q];
        int a0 = 0, b0 = tl;
        while (b0 >= 4 - a0) { b0 -= 4 - a0; ++a0; }
        b0 += a0;
        if (a0 == b0 && q / 6 > q % 6) continue;  // a diagonal tile's lower half mirrors its upper
        const int r = 6 * a0 + q / 6, c = 6 * b0 + q % 6;
        Ms[r * 24 + c] = sum;
        Ms[c * 24 + r] = sum;
    }
    __syncthreads();
    // upper triangle of the cell's E block
    for (int t = tid; t < 300; t += blockDim.x) {
        int R, Cc;
        upper_entry(t, R, Cc);
        const int Jr = R / 3, i = R - 3 * Jr, L = Cc / 3, j = Cc - 3 * L;
        double v = lam * Ms[(3 * Jr + i) * 24 + 3 * L + j] + mu * Ms[(3 * Jr + j) * 24 + 3 * L + i];
        if (i == j)
            v += mu * (Ms[(3 * Jr) * 24 + 3 * L] + Ms[(3 * Jr + 1) * 24 + 3 * L + 1] + Ms[(3 * Jr + 2) * 24 + 3 * L + 2]);
        if (v == 0.0) continue;
        const int gJ = coarse_node(cv, cx + ((Jr >> 2) & 1), cy + ((Jr >> 1) & 1), cz + (Jr & 1));
        const int gL = coarse_node(cv, cx + ((L >> 2) & 1), cy + ((L >> 1) & 1), cz + (L & 1));
        atomicAdd(&E[(int64_t)(3 * gJ + i) * n + 3 * gL + j], v);
        if (R != Cc) atomicAdd(&E[(int64_t)(3 * gL + j) * n + 3 * gJ + i], v);
    }
}

constexpr size_t kFastSmem = sizeof(double) * (kSlices * 10 * 36 + 24 * 24);
static_assert(kSlices * 10 * 36 >= kFastBatch * 25, "reduction area must cover the staging area");

// General path, for elements with a node whose dofs are constrained unalike (a roller): the
// coarse gradient then depends on the component, G_J^(d) = sum_a m_(a,d) phi_J(x_a) grad N_a.
// E (n x n, row-major) += their Galerkin contribution.  CTA (cell, split) takes a
// contiguous share of the coarse cell's such elements in batches of kBatch: eight threads per
// element (one corner J each) stage its coarse gradients G_J^(i) and Q_(J,i) = w G_J^(i) in
// shared memory, then each thread sums one or two of the 300 upper-triangle entries of the
// cell's symmetric 24x24 block over the batch in registers; the sums are added to E (and
// mirrored) once per CTA.
__global__ void __launch_bounds__(kThreadsPerCta)
k_galerkin(CoarseView cv, int split, const int32_t* __restrict__ elem_ptr, const int32_t* __restrict__ elem_list,
           const int4* __restrict__ conn, const double* __restrict__ coords, const double* __restrict__ z,
           Material mat, const uint8_t* __restrict__ mask, int n, double* __restrict__ E) {
    __shared__ double Gs[kBatch][3][8][3];
    __shared__ double Qs[kBatch][3][8][3];
    const double lam = mat.c01, mu = mat.c33;
    const int cell = blockIdx.x / split, part = blockIdx.x - cell * split;
    const int cz = cell % cv.nc2, cy = (cell / cv.nc2) % cv.nc1, cx = cell / (cv.nc1 * cv.nc2);
    const double lo[3] = {cv.x0 + cx * cv.hx, cv.y0 + cy * cv.hy, cv.z0 + cz * cv.hz};
    const int q0 = elem_ptr[2 * cell + 1], q1 = elem_ptr[2 * cell + 2];
    const int chunk = (q1 - q0 + split - 1) / split;
    const int e0 = q0 + part * chunk, e1 = min(q1, e0 + chunk);
    if (e0 >= e1) return;
    int R[2], Cc[2];
    const int nent = threadIdx.x + kThreadsPerCta < 300 ? 2 : 1;
    upper_entry(threadIdx.x, R[0], Cc[0]);
    R[1] = Cc[1] = 0;
    if (nent == 2) upper_entry(threadIdx.x + kThreadsPerCta, R[1], Cc[1]);
    double acc[2] = {0.0, 0.0};
    const int k = threadIdx.x >> 3, J = threadIdx.x & 7;  // staging: element k of the batch, corner J
    for (int base = e0; base < e1; base += kBatch) {
        if (base + k < e1) {
            const int32_t cell = elem_list[base + k];
            const int4 nd = conn[cell];
            double x[4][3];
            load_cell_coords(coords, nd, x);
            TetGeom<double> G;
            tet_geometry(x, G);
            const double rho = cell_rho(mat, z, cell, nd);
            const double w = G.vol * simp(mat, rho);
            const int ids[4] = {nd.x, nd.y, nd.z, nd.w};
            double wa[4];
#pragma unroll
            for (int a = 0; a < 4; ++a)
                wa[a] = corner_weight(J, (x[a][0] - lo[0]) * cv.ihx, (x[a][1] - lo[1]) * cv.ihy, (x[a][2] - lo[2]) * cv.ihz);
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                double gj[3] = {0.0, 0.0, 0.0};
#pragma unroll
                for (int a = 0; a < 4; ++a) {
                    if (mask[3 * (int64_t)ids[a] + d]) continue;
                    gj[0] += wa[a] * G.g[a][0];
                    gj[1] += wa[a] * G.g[a][1];
                    gj[2] += wa[a] * G.g[a][2];
                }
#pragma unroll
                for (int t = 0; t < 3; ++t) {
                    Gs[k][d][J][t] = gj[t];
                    Qs[k][d][J][t] = w * gj[t];
                }
            }
        }
        __syncthreads();
        const int nb = min(kBatch, e1 - base);
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            if (s >= nent) break;
            const int Jr = R[s] / 3, i = R[s] - 3 * Jr, L = Cc[s] / 3, j = Cc[s] - 3 * L;
            double a = 0.0;
            if (i == j) {
                for (int e = 0; e < nb; ++e) {
                    const double* Qi = Qs[e][i][Jr];
                    const double* Gj = Gs[e][j][L];
                    a += (lam + mu) * Qi[i] * Gj[i] + mu * (Qi[0] * Gj[0] + Qi[1] * Gj[1] + Qi[2] * Gj[2]);
                }
            } else {
                for (int e = 0; e < nb; ++e) {
                    const double* Qi = Qs[e][i][Jr];
                    const double* Gj = Gs[e][j][L];
                    a += lam * Qi[i] * Gj[j] + mu * Qi[j] * Gj[i];
                }
            }
            acc[s] += a;
        }
        __syncthreads();
    }
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        if (s >= nent || acc[s] == 0.0) continue;
        const int Jr = R[s] / 3, i = R[s] - 3 * Jr, L = Cc[s] / 3, j = Cc[s] - 3 * L;
        const int gJ = coarse_node(cv, cx + ((Jr >> 2) & 1), cy + ((Jr >> 1) & 1), cz + (Jr & 1));
        const int gL = coarse_node(cv, cx + ((L >> 2) & 1), cy + ((L >> 1) & 1), cz + (L & 1));
        atomicAdd(&E[(int64_t)(3 * gJ + i) * n + 3 * gL + j], acc[s]);
        if (R[s] != Cc[s]) atomicAdd(&E[(int64_t)(3 * gL + j) * n + 3 * gJ + i], acc[s]);
    }
}

// Zero rows/columns (coarse dofs whose basis vanishes after masking) get a unit diagonal.
__global__ void k_regularize(int n, double* __restrict__ E) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        if (!(E[(int64_t)k * n + k] > 0.0)) E[(int64_t)k * n + k] = 1.0;
}

// ---- dense SPD inverse: blocked Cholesky and L^-1 by doubling, 64 x 64 tiles -------------
// E (n x n, row-major, stride n) is factored in place (lower), each diagonal tile's inverse
// kept in D; then X = L^-1 by doubling and E^-1 = X^T X.  Every bulk step is a product of
// 64 x 64 tiles (`tile_gemm`: 8 warps of FP64 mma.sync m8n8k4, a 32 x 16 block per warp,
// operands staged 16 columns at a time through two shared-memory buffers), so the O(n^3)
// work runs at tile-GEMM speed and the number of launches grows with n/64.

constexpr int kNB = 64;   // tile edge
constexpr int kKB = 16;   // k columns staged per pass
constexpr int kRowPad = kKB + 4;  // [row][k] staging stride: 4 (mod 16) doubles, conflict-free fragments
constexpr int kColPad = kNB + 4;  // [k][row] staging stride: 4 (mod 16) doubles
constexpr int kStage = kNB * kRowPad;  // doubles per staged operand (>= kKB * kColPad)

__device__ __forceinline__ void mma_f64(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

// C(ti,tj) = beta C + alpha sum_{kt in [k0,k1)} opA(ti,kt) opB(kt,tj), tiles of kNB; opA(ti,kt)
// is A's tile (ti,kt), or the transpose of its tile (kt,ti) with TA; opB likewise with TB.
// Entries outside n read as 0 and are not stored.  Each operand is staged in the layout its
// global reads are contiguous in: [row][k] (stride kRowPad) for a row-major A or a transposed
// B, [k][row] (stride kColPad) otherwise; both strides keep the m8n8k4 fragment reads (lane
// l: row l/4, k l%4) on distinct banks.
template <int TA, int TB>
__device__ __forceinline__ void tile_gemm(int n, const double* __restrict__ A, const double* __restrict__ B,
                                          double* __restrict__ C, int ti, int tj, int k0, int k1, double alpha,
                                          double beta) {
    __shared__ double As[2][kStage];
    __shared__ double Bs[2][kStage];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = (warp & 1) * 32, wn = (warp >> 1) * 16;  // warp block: rows wm.., cols wn..
    const int g = lane >> 2, q = lane & 3;
    const int r0 = ti * kNB, c0 = tj * kNB;
    const int nstage = (k1 - k0) * (kNB / kKB);
    double acc[4][2][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    double ra[4], rb[4];
    // global -> registers for stage st (1024 values per operand, 4 per thread)
    auto fetch = [&](int st) {
        const int kbase = k0 * kNB + st * kKB;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int e = tid + 256 * u;
            if (TA == 0) {  // A[r0 + row][kbase + c]: c fastest
                const int c = e & 15, row = e >> 4, gr = r0 + row, gc = kbase + c;
                ra[u] = (gr < n && gc < n) ? A[(int64_t)gr * n + gc] : 0.0;
            } else {        // A[kbase + c][r0 + row]: row fastest
                const int row = e & 63, c = e >> 6, gr = kbase + c, gc = r0 + row;
                ra[u] = (gr < n && gc < n) ? A[(int64_t)gr * n + gc] : 0.0;
            }
            if (TB == 0) {  // B[kbase + c][c0 + col]: col fastest
                const int col = e & 63, c = e >> 6, gr = kbase + c, gc = c0 + col;
                rb[u] = (gr < n && gc < n) ? B[(int64_t)gr * n + gc] : 0.0;
            } else {        // B[c0 + col][kbase + c]: c fastest
                const int c = e & 15, col = e >> 4, gr = c0 + col, gc = kbase + c;
                rb[u] = (gr < n && gc < n) ? B[(int64_t)gr * n + gc] : 0.0;
            }
        }
    };
    auto store = [&](int buf) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int e = tid + 256 * u;
            if (TA == 0) As[buf][(e >> 4) * kRowPad + (e & 15)] = ra[u];
            else As[buf][(e >> 6) * kColPad + (e & 63)] = ra[u];
            if (TB == 0) Bs[buf][(e >> 6) * kColPad + (e & 63)] = rb[u];
            else Bs[buf][(e >> 4) * kRowPad + (e & 15)] = rb[u];
        }
    };
    // C's old values (beta != 0) are loaded all at once before the epilogue's stores: one
    // round trip per CTA instead of one per read-modify-write
    double cold[4][2][2];
    auto fetch_c = [&]() {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int gr = r0 + wm + 8 * i + g;
#pragma unroll
            for (int j = 0; j < 2; ++j)
#pragma unroll
                for (int t = 0; t < 2; ++t) {
                    const int gc = c0 + wn + 8 * j + 2 * q + t;
                    cold[i][j][t] = (beta != 0.0 && gr < n && gc < n) ? C[(int64_t)gr * n + gc] : 0.0;
                }
        }
    };
    fetch(0);
    store(0);
    __syncthreads();
    for (int st = 0; st < nstage; ++st) {
        const int buf = st & 1;
        if (st + 1 < nstage) fetch(st + 1);  // in flight during the products below
        const double* as = As[buf];
        const double* bs = Bs[buf];
#pragma unroll
        for (int k4 = 0; k4 < kKB; k4 += 4) {
            const int k = k4 + q;
            double a[4], b[2];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int row = wm + 8 * i + g;
                a[i] = TA == 0 ? as[row * kRowPad + k] : as[k * kColPad + row];
            }
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const int col = wn + 8 * j + g;
                b[j] = TB == 0 ? bs[k * kColPad + col] : bs[col * kRowPad + k];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j) mma_f64(acc[i][j], a[i], b[j]);
        }
        if (st + 1 < nstage) store(buf ^ 1);  // that buffer was last read before the previous barrier
        __syncthreads();
    }
    fetch_c();
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int gr = r0 + wm + 8 * i + g;
        if (gr >= n) continue;
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int t = 0; t < 2; ++t) {
                const int gc = c0 + wn + 8 * j + 2 * q + t;
                if (gc < n) C[(int64_t)gr * n + gc] = beta * cold[i][j][t] + alpha * acc[i][j][t];
            }
    }
}

// Factors diagonal tile kb in place (lower, zeros above) and writes its inverse to D[kb]
// (kNB x kNB, row-major).  One CTA of 256 threads, blocked by 8: for each 8-column block s,
//   A: warp 0 factors the 8 x 8 diagonal block (L_ss) and inverts it (Li = L_ss^-1);
//   B: the block column below, Lp = T[below, s] Li^T, and block row s of L^-1,
//      Wr = Li R_s (R = the rows of [L | I] still to be eliminated, kept in W);
//   C: the rank-8 trailing update T -= Lp Lp^T, the row elimination W[below] -= Lp Wr, and
//      Lp, Wr copied into place.
// B and C are FP64 mma.sync tile products; 24 barriers in all; rows and columns past m are an
// identity block that factors to itself.
constexpr int kDiagThreads = 256;
constexpr int kDiagPad = kNB + 1;
constexpr size_t kDiagSmem = sizeof(double) * (2 * kNB * kDiagPad + kNB * 9 + 8 * kDiagPad + 8 * 9 + 8 * 9);
constexpr size_t kTwoTiles = kDiagSmem;

__global__ void __launch_bounds__(kDiagThreads) k_chol_diag(int n, double* __restrict__ A, int kb,
                                                           double* __restrict__ D, int32_t* __restrict__ bad) {
    extern __shared__ double dyn[];
    double (*T)[kDiagPad] = reinterpret_cast<double (*)[kDiagPad]>(dyn);                  // L (lower)
    double (*W)[kDiagPad] = reinterpret_cast<double (*)[kDiagPad]>(dyn + kNB * kDiagPad);  // L^-1
    double (*Lp)[9] = reinterpret_cast<double (*)[9]>(dyn + 2 * kNB * kDiagPad);           // block column
    double (*Wr)[kDiagPad] = reinterpret_cast<double (*)[kDiagPad]>(dyn + 2 * kNB * kDiagPad + kNB * 9);
    double (*Li)[9] = reinterpret_cast<double (*)[9]>(dyn + 2 * kNB * kDiagPad + kNB * 9 + 8 * kDiagPad);
    double (*W8)[9] = Li + 8;
    const int r0 = kb * kNB, m = min(kNB, n - r0);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int tx = tid & 15, ty = tid >> 4;  // phase C: rows ty + 16a, columns tx + 16b
    {
        double v[kNB * kNB / kDiagThreads];
#pragma unroll
        for (int u = 0; u < kNB * kNB / kDiagThreads; ++u) {
            const int e = tid + kDiagThreads * u, i = e >> 6, j = e & 63;
            v[u] = (i < m && j < m) ? A[(int64_t)(r0 + i) * n + r0 + j] : (i == j ? 1.0 : 0.0);
        }
#pragma unroll
        for (int u = 0; u < kNB * kNB / kDiagThreads; ++u) {
            const int e = tid + kDiagThreads * u, i = e >> 6, j = e & 63;
            T[i][j] = v[u];
            W[i][j] = (i == j) ? 1.0 : 0.0;
        }
    }
    __syncthreads();
    for (int s = 0; s < kNB / 8; ++s) {
        const int o = 8 * s, nb = kNB - o - 8;  // block offset, rows below the block
        // A: unscaled elimination of the 8 x 8 block (lane: row lane/4, columns lane%4 and +4),
        // W8 = the unit factor's inverse; then L_ss = T D^1/2 and Li = D^-1/2 W8
        if (warp == 0) {
            const int r = lane >> 2, c0 = lane & 3;
            W8[r][c0] = (r == c0) ? 1.0 : 0.0;
            W8[r][c0 + 4] = (r == c0 + 4) ? 1.0 : 0.0;
            __syncwarp();
            for (int k = 0; k < 8; ++k) {
                double d = T[o + k][o + k];
                if (!(d > 0.0)) d = 1.0;
                const double inv = 1.0 / d;
                if (r > k) {
                    const double cr = T[o + r][o + k] * inv;
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int c = c0 + 4 * h;
                        if (c > k && c <= r) T[o + r][o + c] -= cr * T[o + c][o + k];
                        else if (c <= k) W8[r][c] -= cr * W8[k][c];
                    }
                }
                __syncwarp();
            }
            const double dr = T[o + r][o + r], dc0 = T[o + c0][o + c0], dc1 = T[o + c0 + 4][o + c0 + 4];
            if (!(dr > 0.0) && c0 == 0) atomicExch(bad, 1);
            const double sr = sqrt(dr > 0.0 ? dr : 1.0);
            const double sc[2] = {sqrt(dc0 > 0.0 ? dc0 : 1.0), sqrt(dc1 > 0.0 ? dc1 : 1.0)};
            __syncwarp();  // every lane has read the pivots before the block is overwritten
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int c = c0 + 4 * h;
                Li[r][c] = (c <= r) ? W8[r][c] / sr : 0.0;
                if (c < r) T[o + r][o + c] /= sc[h];
                else if (c == r) T[o + r][o + r] = sr;
            }
        }
        __syncthreads();
        // B and C on 8 x 8 tiles, one warp per tile, two FP64 m8n8k4 products per tile (lane l
        // holds A[l/4][l%4], B[l%4][l/4] and C[l/4][2(l%4) + t]).  Li is zero above its
        // diagonal, and a diagonal tile's upper half takes the trailing update too (never read).
        const int nI = 7 - s;  // block rows below block s
        const int g = lane >> 2, q = lane & 3;
        // B: Lp = T[below, s] Li^T (tiles I < nI);  Wr = Li W[s, :] (tiles J <= s)
        for (int tile = warp; tile < nI + s + 1; tile += kDiagThreads / 32) {
            double acc[2] = {0.0, 0.0};
            if (tile < nI) {
#pragma unroll
                for (int kh = 0; kh < 2; ++kh)
                    mma_f64(acc, T[o + 8 + 8 * tile + g][o + 4 * kh + q], Li[g][4 * kh + q]);
                Lp[8 * tile + g][2 * q] = acc[0];
                Lp[8 * tile + g][2 * q + 1] = acc[1];
            } else {
                const int J = tile - nI;
#pragma unroll
                for (int kh = 0; kh < 2; ++kh) mma_f64(acc, Li[g][4 * kh + q], W[o + 4 * kh + q][8 * J + g]);
                Wr[g][8 * J + 2 * q] = acc[0];
                Wr[g][8 * J + 2 * q + 1] = acc[1];
            }
        }
        __syncthreads();
        const int nB1 = nb * 8, nB2 = 8 * (o + 8);
        // C: T[I, J] -= Lp_I Lp_J^T (s < J <= I);  W[I, J] -= Lp_I Wr_J (J <= s < I)
        const int t1 = nI * (nI + 1) / 2, t2 = nI * (s + 1);
        for (int tile = warp; tile < t1 + t2; tile += kDiagThreads / 32) {
            double acc[2] = {0.0, 0.0};
            if (tile < t1) {
                int I = 0, J = tile;
                while (J >= I + 1) { J -= I + 1; ++I; }
#pragma unroll
                for (int kh = 0; kh < 2; ++kh) mma_f64(acc, Lp[8 * I + g][4 * kh + q], Lp[8 * J + g][4 * kh + q]);
                const int i = o + 8 + 8 * I + g, j = o + 8 + 8 * J + 2 * q;
                T[i][j] -= acc[0];
                T[i][j + 1] -= acc[1];
            } else {
                const int f = tile - t1, I = f / (s + 1), J = f - I * (s + 1);
#pragma unroll
                for (int kh = 0; kh < 2; ++kh) mma_f64(acc, Lp[8 * I + g][4 * kh + q], Wr[4 * kh + q][8 * J + g]);
                const int i = o + 8 + 8 * I + g, j = 8 * J + 2 * q;
                W[i][j] -= acc[0];
                W[i][j + 1] -= acc[1];
            }
        }
        for (int e = tid; e < nB1 + nB2; e += kDiagThreads) {
            if (e < nB1) {
                const int i = e >> 3, c = e & 7;
                T[o + 8 + i][o + c] = Lp[i][c];
            } else {
                const int f = e - nB1, rr = f / (o + 8), j = f - rr * (o + 8);
                W[o + rr][j] = Wr[rr][j];
            }
        }
        __syncthreads();
    }
    for (int e = tid; e < kNB * kNB; e += kDiagThreads) {
        const int i = e >> 6, j = e & 63;
        if (i < m && j < m) A[(int64_t)(r0 + i) * n + r0 + j] = (j <= i) ? T[i][j] : 0.0;
        D[(int64_t)kb * kNB * kNB + e] = (i < m && j < m && j <= i) ? W[i][j] : 0.0;
    }
}

// Panel: A[ib,kb] <- A[ib,kb] L_kk^-T for every tile row ib > kb (one CTA per tile row): both
// 64 x 64 operands staged whole ([row][k], stride kColPad), then the FP64 mma.sync product
// (P L^-T)[i][j] = sum_k P[i][k] Linv[j][k] with the warp blocks of `tile_gemm`.
constexpr size_t kPanelSmem = sizeof(double) * 2 * kNB * kColPad;

__global__ void __launch_bounds__(256) k_chol_panel(int n, double* __restrict__ A, int kb,
                                                   const double* __restrict__ D) {
    extern __shared__ double dyn[];
    double* Ps = dyn;
    double* Ds = dyn + kNB * kColPad;
    const int ib = kb + 1 + blockIdx.x;
    const int r0 = ib * kNB, c0 = kb * kNB;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = (warp & 1) * 32, wn = (warp >> 1) * 16;
    const int g = lane >> 2, q = lane & 3;
    {   // all 32 loads of a thread in flight at once, then the shared-memory stores
        double dv[16], pv[16];
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            const int e = tid + 256 * u, i = e >> 6, j = e & 63;
            dv[u] = D[(int64_t)kb * kNB * kNB + e];
            pv[u] = (r0 + i < n && c0 + j < n) ? A[(int64_t)(r0 + i) * n + c0 + j] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            const int e = tid + 256 * u, i = e >> 6, j = e & 63;
            Ds[i * kColPad + j] = dv[u];
            Ps[i * kColPad + j] = pv[u];
        }
    }
    __syncthreads();
    double acc[4][2][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
#pragma unroll 4
    for (int k4 = 0; k4 < kNB; k4 += 4) {
        const int k = k4 + q;
        double a[4], b[2];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = Ps[(wm + 8 * i + g) * kColPad + k];
#pragma unroll
        for (int j = 0; j < 2; ++j) b[j] = Ds[(wn + 8 * j + g) * kColPad + k];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j) mma_f64(acc[i][j], a[i], b[j]);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int gr = r0 + wm + 8 * i + g;
        if (gr >= n) continue;
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int t = 0; t < 2; ++t) {
                const int gc = c0 + wn + 8 * j + 2 * q + t;
                if (gc < n) A[(int64_t)gr * n + gc] = acc[i][j][t];
            }
    }
}

// Trailing update A[ib,jb] -= A[ib,kb] A[jb,kb]^T.  COL: the next tile column jb = kb + 1
// (one CTA per tile, ib > kb); otherwise the tiles kb + 2 <= jb <= ib (blockIdx enumerates
// that lower triangle).
template <bool COL>
__global__ void __launch_bounds__(256) k_chol_update(int n, double* __restrict__ A, int kb, int nblk) {
    int gi, gj;
    if (COL) {
        gi = kb + 1 + blockIdx.x;
        gj = kb + 1;
    } else {
        int idx = blockIdx.x, ib = 0;
        while (idx >= ib + 1) { idx -= ib + 1; ++ib; }
        gi = kb + 2 + ib;
        gj = kb + 2 + idx;
    }
    if (gi >= nblk) return;
    tile_gemm<0, 1>(n, A, A, A, gi, gj, kb, kb + 1, -1.0, 1.0);
}

// X = L^-1 by doubling: X starts as its diagonal tiles D[i] and zeros; level s joins blocks
// of s tiles into blocks of 2s: X[B2,B1] = -X[B2,B2] L[B2,B1] X[B1,B1], in two batched passes:
// mode 0: T[i,j] = sum_{k in B1, k >= j} L[i,k] X[k,j];  mode 1: X[i,j] = -sum_{k in B2, k <= i} X[i,k] T[k,j].
// L is banded (tile (i,k) zero for i - k > tb), so T's rows i >= b2 + tb are zero: mode 0
// forms only rows [b2, b2 + tb) over k >= i - tb, and mode 1 sums over k < b2 + tb.
__global__ void k_tri_init(int n, const double* __restrict__ D, double* __restrict__ X) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)n * n;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int r = int(e / n), c = int(e - (int64_t)r * n);
        const int ib = r / kNB, jb = c / kNB;
        X[e] = (ib == jb) ? D[(int64_t)ib * kNB * kNB + (r - ib * kNB) * kNB + (c - jb * kNB)] : 0.0;
    }
}

__device__ __forceinline__ int tri_rows(int mode, int s, int tb) { return mode == 0 ? min(s, tb) : s; }

__global__ void __launch_bounds__(256) k_tri_level(int n, int nblk, int s, int mode, int tb,
                                                  const double* __restrict__ L, double* __restrict__ X,
                                                  double* __restrict__ T) {
    const int per_pair = tri_rows(mode, s, tb) * s;
    const int pair = blockIdx.x / per_pair, rem = blockIdx.x - pair * per_pair;
    const int b1 = pair * 2 * s, b2 = b1 + s;
    const int e1 = min(b2, nblk), e2 = min(b2 + s, nblk);
    const int i = b2 + rem / s, j = b1 + rem % s;
    if (b2 >= nblk || i >= e2 || j >= e1) return;
    if (mode == 0) tile_gemm<0, 0>(n, L, X, T, i, j, min(max(j, i - tb), e1), e1, 1.0, 0.0);
    else tile_gemm<0, 0>(n, X, T, X, i, j, b2, min(i + 1, b2 + tb), -1.0, 0.0);
}

// Einv = X^T X for X = L^-1 (lower): Einv[i,j] = sum_{k >= max(i,j)} X[k,i]^T X[k,j]
__global__ void __launch_bounds__(256) k_gram(int n, int nblk, const double* __restrict__ X,
                                             double* __restrict__ Einv) {
    const int i = blockIdx.y, j = blockIdx.x;
    tile_gemm<1, 0>(n, X, X, Einv, i, j, max(i, j), nblk, 1.0, 0.0);
}

// ---- per-iteration kernels ----------------------------------------------------------------

// Restriction rc[(J,d)] = sum_p phi_J(x_p) m_(p,d) v[(p,d)], deterministic, in two passes.
// Pass 1: CTA (cell, split) sums over its share of the coarse cell's fine nodes the 24 values
// phi_b(x_p) m_(p,d) v[(p,d)] (corner b of the cell, component d) into part[CTA][24].
__global__ void __launch_bounds__(kThreadsPerCta)
k_restrict_cells(CoarseView cv, int split, const int32_t* __restrict__ node_ptr,
                 const int32_t* __restrict__ node_list, const double* __restrict__ coords,
                 const uint8_t* __restrict__ mask, const float* __restrict__ v, const float* __restrict__ vscale,
                 double* __restrict__ part, const PcgScalars* S) {
    __shared__ double sh[kThreadsPerCta / 32][24];
    pdl_wait();
    pdl_trigger();
    if (S && S->done) return;
    const int cell = blockIdx.x / split, piece = blockIdx.x - cell * split;
    const int cz = cell % cv.nc2, cy = (cell / cv.nc2) % cv.nc1, cx = cell / (cv.nc1 * cv.nc2);
    const double lo[3] = {cv.x0 + cx * cv.hx, cv.y0 + cy * cv.hy, cv.z0 + cz * cv.hz};
    const int q0 = node_ptr[cell], q1 = node_ptr[cell + 1];
    const int chunk = (q1 - q0 + split - 1) / split;
    const int a0 = q0 + piece * chunk, a1 = min(q1, a0 + chunk);
    double s[24];
#pragma unroll
    for (int t = 0; t < 24; ++t) s[t] = 0.0;
    for (int q = a0 + threadIdx.x; q < a1; q += kThreadsPerCta) {
        const int64_t p = node_list[q];
        const double u = (coords[3 * p] - lo[0]) * cv.ihx, vv = (coords[3 * p + 1] - lo[1]) * cv.ihy,
                     w = (coords[3 * p + 2] - lo[2]) * cv.ihz;
        double val[3];
#pragma unroll
        for (int d = 0; d < 3; ++d)
            val[d] = mask[3 * p + d] ? 0.0 : double(vscale ? vscale[3 * p + d] * v[3 * p + d] : v[3 * p + d]);
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            const double wgt = corner_weight(b, u, vv, w);
#pragma unroll
            for (int d = 0; d < 3; ++d) s[3 * b + d] += wgt * val[d];
        }
    }
    // warp sums of the 24 values by halving: each exchange hands half of a lane's values to its
    // partner, so after offsets 16, 8, 4 a lane holds 3 of the 24 sums (which 3 set by lane bits
    // 4..2) and offsets 2, 1 finish them -- 27 shuffles instead of 24 x 5
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double t12[12], t6[6], t3[3];
    {
        const bool hi = (lane & 16) != 0;
#pragma unroll
        for (int i = 0; i < 12; ++i) {
            const double send = hi ? s[i] : s[12 + i];
            t12[i] = (hi ? s[12 + i] : s[i]) + __shfl_xor_sync(0xffffffffu, send, 16);
        }
    }
    {
        const bool hi = (lane & 8) != 0;
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            const double send = hi ? t12[i] : t12[6 + i];
            t6[i] = (hi ? t12[6 + i] : t12[i]) + __shfl_xor_sync(0xffffffffu, send, 8);
        }
    }
    {
        const bool hi = (lane & 4) != 0;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const double send = hi ? t6[i] : t6[3 + i];
            t3[i] = (hi ? t6[3 + i] : t6[i]) + __shfl_xor_sync(0xffffffffu, send, 4);
        }
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        t3[i] += __shfl_xor_sync(0xffffffffu, t3[i], 2);
        t3[i] += __shfl_xor_sync(0xffffffffu, t3[i], 1);
    }
    if ((lane & 3) == 0) {
        const int base = ((lane & 16) ? 12 : 0) + ((lane & 8) ? 6 : 0) + ((lane & 4) ? 3 : 0);
#pragma unroll
        for (int i = 0; i < 3; ++i) sh[wid][base + i] = t3[i];
    }
    __syncthreads();
    if (threadIdx.x < 24) {
        double t = 0.0;
        for (int k = 0; k < kThreadsPerCta / 32; ++k) t += sh[k][threadIdx.x];
        part[(int64_t)blockIdx.x * 24 + threadIdx.x] = t;
    }
}

// Pass 2: rc[(J,d)] = sum over the <= 8 cells around coarse node J (J is corner b of the cell)
// and over their splits, in a fixed order.
__global__ void k_restrict_sum(CoarseView cv, int split, const double* __restrict__ part, double* __restrict__ rc,
                               const PcgScalars* S) {
    pdl_wait();
    pdl_trigger();
    if (S && S->done) return;
    const int ncn = (cv.nc0 + 1) * (cv.nc1 + 1) * (cv.nc2 + 1);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 3 * ncn; t += gridDim.x * blockDim.x) {
        const int J = t / 3, d = t - 3 * J;
        const int iz = J % (cv.nc2 + 1), iy = (J / (cv.nc2 + 1)) % (cv.nc1 + 1), ix = J / ((cv.nc1 + 1) * (cv.nc2 + 1));
        double sum = 0.0;
        for (int b = 0; b < 8; ++b) {
            const int cx = ix - ((b >> 2) & 1), cy = iy - ((b >> 1) & 1), cz = iz - (b & 1);
            if (cx < 0 || cy < 0 || cz < 0 || cx >= cv.nc0 || cy >= cv.nc1 || cz >= cv.nc2) continue;
            const double* pc = part + (int64_t)cell_id(cv, cx, cy, cz) * split * 24 + 3 * b + d;
            for (int k = 0; k < split; ++k) sum += pc[24 * k];
        }
        rc[t] = sum;
    }
}

// The coarse solve is y = U (X r) with X = L^-1 and U = X^T (E^-1 = X^T X); the factorization
// and inversion run in FP64, the two products per preconditioner apply read FP32 copies.
// out = M in for a triangular FP32 matrix (row stride ld, zeros outside the triangle and in
// the padding columns), FP64 vectors and sums.  A CTA of 4 warps per row (the longest rows hold
// n/4 16-byte groups, so one warp per row left the product waiting on their load latency);
// 16-byte loads from the row's first 4-aligned column, the in[] reads past n skipped; the four
// warp sums are added in a fixed order.
template <bool LOWER>
__global__ void __launch_bounds__(128) k_coarse_trmv(int n, int ld, const float* __restrict__ M,
                                                     const double* __restrict__ in, double* __restrict__ out,
                                                     const PcgScalars* S) {
    pdl_wait();
    pdl_trigger();
    if (S && S->done) return;
    __shared__ double part[4];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int row = blockIdx.x; row < n; row += gridDim.x) {
        const int q0 = LOWER ? 0 : (row >> 2), q1 = LOWER ? (row >> 2) + 1 : (n + 3) >> 2;
        const float4* mp = reinterpret_cast<const float4*>(M + (int64_t)row * ld);
        double s = 0.0;
#pragma unroll 4
        for (int q = q0 + threadIdx.x; q < q1; q += 128) {
            const float4 v = __ldg(mp + q);
            const int c = 4 * q;
            s += double(v.x) * in[c];
            if (c + 1 < n) s += double(v.y) * in[c + 1];
            if (c + 2 < n) s += double(v.z) * in[c + 2];
            if (c + 3 < n) s += double(v.w) * in[c + 3];
        }
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) part[warp] = s;
        __syncthreads();
        if (threadIdx.x == 0) out[row] = (part[0] + part[1]) + (part[2] + part[3]);
        __syncthreads();
    }
}

// Xf = L^-1 (lower) and Uf = its transpose (upper) in FP32, row stride ld, from X = L^-1 (FP64,
// stride n); every entry of a row up to ld is written (zeros off the triangle and past n).
// Block (bj, bi) of 32 x 32: Xf tile (bi, bj) when bj <= bi, Uf tile (bi, bj) when bj >= bi.
__global__ void k_coarse_pack(int n, int ld, const double* __restrict__ X, float* __restrict__ Xf,
                              float* __restrict__ Uf) {
    __shared__ double t[32][33];
    const int bi = blockIdx.y, bj = blockIdx.x;
    const int tx = threadIdx.x, ty = threadIdx.y;
    if (bj <= bi) {
        for (int r = ty; r < 32; r += 8) {
            const int gr = bi * 32 + r, gc = bj * 32 + tx;
            if (gr < n && gc < ld) Xf[(int64_t)gr * ld + gc] = (gc <= gr && gc < n) ? float(X[(int64_t)gr * n + gc]) : 0.f;
        }
    }
    if (bj < bi) return;
    for (int r = ty; r < 32; r += 8) {
        const int gr = bj * 32 + r, gc = bi * 32 + tx;  // X row block bj, column block bi
        t[r][tx] = (gr < n && gc < n) ? X[(int64_t)gr * n + gc] : 0.0;
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const int gr = bi * 32 + r, gc = bj * 32 + tx;
        if (gr < n && gc < ld) Uf[(int64_t)gr * ld + gc] = (gc >= gr && gc < n) ? float(t[tx][r]) : 0.f;
    }
}


// y[(p,d)] (+)= yscale[(p,d)] m_(p,d) sum_J phi_J(x_p) yc[(J,d)]  (yscale may be NULL: 1)
__global__ void k_prolong(int32_t N, CoarseView cv, const double* __restrict__ coords, const uint8_t* __restrict__ mask,
                          const double* __restrict__ yc, const float* __restrict__ yscale, float* __restrict__ y,
                          int accumulate, const PcgScalars* S) {
    pdl_wait();
    pdl_trigger();
    if (S && S->done) return;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        const double x = coords[3 * p], yy = coords[3 * p + 1], zz = coords[3 * p + 2];
        int cx, cy, cz;
        cell_of(cv, x, yy, zz, cx, cy, cz);
        const double u = (x - (cv.x0 + cx * cv.hx)) * cv.ihx, v = (yy - (cv.y0 + cy * cv.hy)) * cv.ihy,
                     w = (zz - (cv.z0 + cz * cv.hz)) * cv.ihz;
        double s[3] = {0.0, 0.0, 0.0};
        for (int b = 0; b < 8; ++b) {
            const double wgt = corner_weight(b, u, v, w);
            const int J = coarse_node(cv, cx + ((b >> 2) & 1), cy + ((b >> 1) & 1), cz + (b & 1));
            s[0] += wgt * yc[3 * J];
            s[1] += wgt * yc[3 * J + 1];
            s[2] += wgt * yc[3 * J + 2];
        }
        for (int d = 0; d < 3; ++d) {
            const float val = mask[3 * p + d] ? 0.f : (yscale ? yscale[3 * p + d] * float(s[d]) : float(s[d]));
            y[3 * p + d] = accumulate ? y[3 * p + d] + val : val;
        }
    }
}

}  // namespace

static CoarseView coarse_view(const plato_problem* h) {
    const CoarseSpace& c = h->coarse;
    return CoarseView{c.nc[0], c.nc[1], c.nc[2], c.x0[0], c.x0[1], c.x0[2], c.h[0], c.h[1], c.h[2],
                      1.0 / c.h[0], 1.0 / c.h[1], 1.0 / c.h[2]};
}

static int csr_by_key(plato_problem* h, int64_t count, uint32_t* keys, int32_t* vals, int32_t* hist, int nkeys,
                      int32_t** ptr_out, int32_t** list_out) {
    cudaStream_t s = h->stream;
    uint32_t* k2 = nullptr;
    int32_t* v2 = nullptr;
    PLATO_CUDA(h, cudaMallocAsync(&k2, sizeof(uint32_t) * count, s));
    PLATO_CUDA(h, cudaMalloc(&v2, sizeof(int32_t) * count));
    PLATO_CUDA(h, cudaMalloc(ptr_out, sizeof(int32_t) * (nkeys + 1)));
    size_t tb = 0, tb2 = 0;
    PLATO_CUDA(h, cub::DeviceRadixSort::SortPairs(nullptr, tb, keys, k2, vals, v2, count, 0, 32, s));
    PLATO_CUDA(h, cub::DeviceScan::ExclusiveSum(nullptr, tb2, hist, *ptr_out, nkeys + 1, s));
    void* tmp = nullptr;
    PLATO_CUDA(h, cudaMallocAsync(&tmp, tb > tb2 ? tb : tb2, s));
    PLATO_CUDA(h, cub::DeviceRadixSort::SortPairs(tmp, tb, keys, k2, vals, v2, count, 0, 32, s));
    PLATO_CUDA(h, cub::DeviceScan::ExclusiveSum(tmp, tb2, hist, *ptr_out, nkeys + 1, s));
    PLATO_CUDA(h, cudaFreeAsync(tmp, s));
    PLATO_CUDA(h, cudaFreeAsync(k2, s));
    *list_out = v2;
    return PLATO_OK;
}

// Mesh-level setup for the requested coarse grid (once per grid size).
int coarse_setup_mesh(plato_problem* h) {
    CoarseSpace& c = h->coarse;
    const int* want = h->opts.coarse_cells;
    if (c.ready && c.nc[0] == want[0] && c.nc[1] == want[1] && c.nc[2] == want[2]) return PLATO_OK;
    coarse_release(h);
    for (int d = 0; d < 3; ++d) {
        if (want[d] < 1 || want[d] > 64) return plato_fail(h, PLATO_BAD_INPUT, "coarse_cells must be in [1, 64]");
        c.nc[d] = want[d];
        c.x0[d] = h->bbox_min[d];
        c.h[d] = (h->bbox_max[d] - h->bbox_min[d]) / want[d];
        if (!(c.h[d] > 0.0)) return plato_fail(h, PLATO_BAD_INPUT, "degenerate mesh bounding box");
    }
    c.ncells = c.nc[0] * c.nc[1] * c.nc[2];
    c.nnodes = (c.nc[0] + 1) * (c.nc[1] + 1) * (c.nc[2] + 1);
    c.ndof = 3 * c.nnodes;
    if (c.ndof > 6144) return plato_fail(h, PLATO_BAD_INPUT, "coarse grid too large for the dense coarse solve");
    cudaStream_t s = h->stream;
    const CoarseView cv = coarse_view(h);
    const int T = 256;
    uint32_t* keys = nullptr;
    int32_t *vals = nullptr, *hist = nullptr, *bad = nullptr;
    const int64_t mx = h->C > h->N ? h->C : h->N;
    PLATO_CUDA(h, cudaMallocAsync(&keys, sizeof(uint32_t) * mx, s));
    PLATO_CUDA(h, cudaMallocAsync(&vals, sizeof(int32_t) * mx, s));
    PLATO_CUDA(h, cudaMallocAsync(&hist, sizeof(int32_t) * (2 * c.ncells + 1), s));
    PLATO_CUDA(h, cudaMallocAsync(&bad, sizeof(int32_t), s));
    // nodes by cell
    PLATO_CUDA(h, cudaMemsetAsync(hist, 0, sizeof(int32_t) * (c.ncells + 1), s));
    k_node_keys<<<grid_for(h->N, T), T, 0, s>>>(h->N, h->coords, cv, keys, vals, hist);
    PLATO_LAUNCH_CHECK(h);
    int rc = csr_by_key(h, h->N, keys, vals, hist, c.ncells, &c.node_ptr, &c.node_list);
    if (rc) return rc;
    // elements by cell and kind (+ the every-element-in-one-cell check)
    PLATO_CUDA(h, cudaMemsetAsync(hist, 0, sizeof(int32_t) * (2 * c.ncells + 1), s));
    PLATO_CUDA(h, cudaMemsetAsync(bad, 0, sizeof(int32_t), s));
    k_elem_keys<<<grid_for(h->C, T), T, 0, s>>>(h->C, h->conn, h->coords, cv, h->bc_mask, keys, vals, hist, bad);
    PLATO_LAUNCH_CHECK(h);
    rc = csr_by_key(h, h->C, keys, vals, hist, 2 * c.ncells, &c.elem_ptr, &c.elem_list);
    if (rc) return rc;
    int32_t bad_h = 0;
    PLATO_CUDA(h, cudaMemcpyAsync(&bad_h, bad, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    PLATO_CUDA(h, cudaStreamSynchronize(s));
    PLATO_CUDA(h, cudaFreeAsync(keys, s));
    PLATO_CUDA(h, cudaFreeAsync(vals, s));
    PLATO_CUDA(h, cudaFreeAsync(hist, s));
    PLATO_CUDA(h, cudaFreeAsync(bad, s));
    if (bad_h)
        return plato_fail(h, PLATO_BAD_INPUT,
                          "coarse grid does not align with the mesh: an element straddles two coarse cells");
    // Every element lies in one coarse cell, so E couples only corners of a common cell: nodes
    // at most (nc1+1)(nc2+1) + (nc2+1) + 1 apart in the x-major numbering, 3 dofs each.
    c.band = 3 * ((c.nc[1] + 1) * (c.nc[2] + 1) + (c.nc[2] + 1) + 1) + 2;
    c.tband = (c.band + kNB - 1) / kNB;
    const size_t nn = size_t(c.ndof) * c.ndof;
    PLATO_CUDA(h, cudaMalloc(&c.E, sizeof(double) * nn));
    c.ldf = (c.ndof + 3) & ~3;
    PLATO_CUDA(h, cudaMalloc(&c.Xf, sizeof(float) * 2 * size_t(c.ndof) * c.ldf));
    c.Uf = c.Xf + size_t(c.ndof) * c.ldf;
    PLATO_CUDA(h, cudaMalloc(&c.X, sizeof(double) * nn));
    PLATO_CUDA(h, cudaMalloc(&c.T, sizeof(double) * nn));
    const int nblk = (c.ndof + kNB - 1) / kNB;
    PLATO_CUDA(h, cudaMalloc(&c.Dt, sizeof(double) * size_t(nblk) * kNB * kNB));
    // splits of each coarse cell's node / element lists so that the restriction and the
    // Galerkin sum run about 8 CTAs per SM
    c.rsplit = clampi((148 * 8 + c.ncells - 1) / c.ncells, 1, 64);
    c.gsplit = clampi((148 * 8 + c.ncells - 1) / c.ncells, 1, 64);
    PLATO_CUDA(h, cudaMalloc(&c.rpart, sizeof(double) * 24 * c.ncells * c.rsplit));
    PLATO_CUDA(h, cudaMalloc(&c.rc, sizeof(double) * c.ndof));
    PLATO_CUDA(h, cudaMalloc(&c.yc, sizeof(double) * c.ndof));
    PLATO_CUDA(h, cudaMalloc(&c.tc, sizeof(double) * c.ndof));
    PLATO_CUDA(h, cudaMalloc(&c.flag, sizeof(int32_t)));
    c.ready = 1;
    return PLATO_OK;
}

void coarse_release(plato_problem* h) {
    CoarseSpace& c = h->coarse;
    for (int32_t** p : {&c.node_ptr, &c.node_list, &c.elem_ptr, &c.elem_list, &c.flag})
        if (*p) { cudaFree(*p); *p = nullptr; }
    for (double** p : {&c.E, &c.X, &c.T, &c.Dt, &c.rc, &c.yc, &c.tc, &c.rpart})
        if (*p) { cudaFree(*p); *p = nullptr; }
    if (c.Xf) { cudaFree(c.Xf); c.Xf = c.Uf = nullptr; }
    if (c.pending && c.ev_ready) cudaEventSynchronize(c.ev_ready);
    c.pending = 0;
    c.start_marked = 0;
    for (cudaEvent_t* e : {&c.ev_panel, &c.ev_trail, &c.ev_start, &c.ev_ready})
        if (*e) { cudaEventDestroy(*e); *e = nullptr; }
    if (c.chain) { cudaGraphExecDestroy(c.chain); c.chain = nullptr; }
    if (c.side) { cudaStreamDestroy(c.side); c.side = nullptr; }
    if (c.cs) { cudaStreamDestroy(c.cs); c.cs = nullptr; }
    if (c.flag_host) { cudaFreeHost(c.flag_host); c.flag_host = nullptr; }
    c.ready = 0;
}

// The coarse set-up is a chain of small dependent kernels running beside the fine-level
// work: its streams take the highest priority, so each of its CTAs is scheduled as soon as an
// SM has room rather than behind the queued fine-level CTAs.
static int coarse_stream(plato_problem* h, cudaStream_t* st) {
    int least = 0, greatest = 0;
    PLATO_CUDA(h, cudaDeviceGetStreamPriorityRange(&least, &greatest));
    PLATO_CUDA(h, cudaStreamCreateWithPriority(st, cudaStreamNonBlocking, greatest));
    return PLATO_OK;
}

// Enqueues on the coarse stream (being captured) the banded blocked Cholesky of E, the
// doubling inverse X = L^-1 and the FP32 packing of X and X^T.
static int enqueue_factorization(plato_problem* h, int* launches) {
    CoarseSpace& c = h->coarse;
    cudaStream_t s = c.cs;
    const int n = c.ndof;
    const int nblk = (n + kNB - 1) / kNB;
    double *X = c.X, *D = c.Dt, *Tmp = c.T;  // scratch allocated with the coarse grid
    int nl = 0;
    PLATO_CUDA(h, cudaMemsetAsync(c.flag, 0, sizeof(int32_t), s));
    // Right-looking blocked Cholesky with a look-ahead of one tile column.  Step kb on the
    // coarse stream: diagonal tile, panel, then the update of column kb + 1 alone, which the
    // next step's diagonal tile needs; the rest of the trailing update (columns >= kb + 2)
    // runs on the side stream meanwhile.  The two write disjoint tile columns; the coarse
    // stream waits for the side stream's step kb - 1 before it updates column kb + 1 (which
    // that step also writes), and the side stream starts step kb after panel kb.  E is banded
    // and the factor keeps its band (no fill outside it), so a step touches only the tband
    // tile rows below kb.
    bool trail_pending = false;
    for (int kb = 0; kb < nblk; ++kb) {
        k_chol_diag<<<1, kDiagThreads, kTwoTiles, s>>>(n, c.E, kb, D, c.flag);
        ++nl;
        const int rem = std::min(nblk - kb - 1, c.tband);
        if (rem == 0) break;
        k_chol_panel<<<rem, 256, kPanelSmem, s>>>(n, c.E, kb, D);
        ++nl;
        if (trail_pending) PLATO_CUDA(h, cudaStreamWaitEvent(s, c.ev_trail, 0));
        trail_pending = false;
        if (rem > 1) {
            PLATO_CUDA(h, cudaEventRecord(c.ev_panel, s));
            PLATO_CUDA(h, cudaStreamWaitEvent(c.side, c.ev_panel, 0));
            k_chol_update<false><<<(rem - 1) * rem / 2, 256, 0, c.side>>>(n, c.E, kb, nblk);
            PLATO_CUDA(h, cudaEventRecord(c.ev_trail, c.side));
            trail_pending = true;
            ++nl;
        }
        k_chol_update<true><<<rem, 256, 0, s>>>(n, c.E, kb, nblk);
        ++nl;
    }
    if (trail_pending) PLATO_CUDA(h, cudaStreamWaitEvent(s, c.ev_trail, 0));
    PLATO_LAUNCH_CHECK(h);
    k_tri_init<<<grid_for(int64_t(n) * n, 256, 148 * 16), 256, 0, s>>>(n, D, X);
    ++nl;
    PLATO_LAUNCH_CHECK(h);
    for (int lv = 1; lv < nblk; lv *= 2) {
        const int pairs = (nblk + 2 * lv - 1) / (2 * lv);
        k_tri_level<<<pairs * std::min(lv, c.tband) * lv, 256, 0, s>>>(n, nblk, lv, 0, c.tband, c.E, X, Tmp);
        k_tri_level<<<pairs * lv * lv, 256, 0, s>>>(n, nblk, lv, 1, c.tband, c.E, X, Tmp);
        nl += 2;
        PLATO_LAUNCH_CHECK(h);
    }
    // the coarse solve applies X then U = X^T: FP32 copies with 16-byte rows
    const int nt = (n + 31) / 32;
    k_coarse_pack<<<dim3(nt, nt), dim3(32, 8), 0, s>>>(n, c.ldf, X, c.Xf, c.Uf);
    ++nl;
    PLATO_LAUNCH_CHECK(h);
    *launches = nl;
    return PLATO_OK;
}

// Captures enqueue_factorization into c.chain (once per coarse grid).
static int capture_factorization(plato_problem* h) {
    CoarseSpace& c = h->coarse;
    PLATO_RC(ensure_smem_attribute(h, reinterpret_cast<const void*>(k_chol_diag), int(kTwoTiles)));
    PLATO_RC(ensure_smem_attribute(h, reinterpret_cast<const void*>(k_chol_panel), int(kPanelSmem)));
    if (!c.side) PLATO_RC(coarse_stream(h, &c.side));
    for (cudaEvent_t* e : {&c.ev_panel, &c.ev_trail})
        if (!*e) PLATO_CUDA(h, cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    PLATO_CUDA(h, cudaStreamBeginCapture(c.cs, cudaStreamCaptureModeThreadLocal));
    int launches = 0;
    const int rc = enqueue_factorization(h, &launches);
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(c.cs, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (ce != cudaSuccess) return plato_fail(h, PLATO_CUDA_ERROR, cudaGetErrorString(ce));
    const cudaError_t ie = cudaGraphInstantiate(&c.chain, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
        c.chain = nullptr;
        return plato_fail(h, PLATO_CUDA_ERROR, cudaGetErrorString(ie));
    }
    c.chain_launches = launches;
    return PLATO_OK;
}

// Per-solve setup: Galerkin operator of control z, Cholesky, explicit inverse, on the coarse
// stream after the work already queued on the handle's stream.  E_copy (device, may be NULL)
// receives E before it is factored.  deferred: return at once (coarse_wait before the first
// use, coarse_finish after the solve); otherwise wait here.
int coarse_setup_operator(plato_problem* h, const double* z, double* E_copy, int deferred) {
    CoarseSpace& c = h->coarse;
    if (!c.cs) PLATO_RC(coarse_stream(h, &c.cs));
    for (cudaEvent_t* e : {&c.ev_start, &c.ev_ready})
        if (!*e) PLATO_CUDA(h, cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    if (!c.flag_host) PLATO_CUDA(h, cudaMallocHost(reinterpret_cast<void**>(&c.flag_host), sizeof(int32_t)));
    if (!c.start_marked) PLATO_CUDA(h, cudaEventRecord(c.ev_start, h->stream));
    c.start_marked = 0;
    PLATO_CUDA(h, cudaStreamWaitEvent(c.cs, c.ev_start, 0));
    cudaStream_t s = c.cs;
    const int n = c.ndof;
    const size_t nn = size_t(n) * n;
    if (h->timing) {
        for (cudaEvent_t& e : h->coarse_ev)
            if (!e) PLATO_CUDA(h, cudaEventCreate(&e));
        PLATO_CUDA(h, cudaEventRecord(h->coarse_ev[0], s));
    }
    PLATO_CUDA(h, cudaMemsetAsync(c.E, 0, sizeof(double) * nn, s));
    PLATO_RC(ensure_smem_attribute(h, reinterpret_cast<const void*>(k_galerkin_fast), int(kFastSmem)));
    k_galerkin_fast<<<c.ncells * c.gsplit, kThreadsPerCta, kFastSmem, s>>>(
        coarse_view(h), c.gsplit, c.elem_ptr, c.elem_list, h->conn, h->coords, z, h->material, h->bc_mask, n, c.E);
    PLATO_LAUNCH_CHECK(h);
    k_galerkin<<<c.ncells * c.gsplit, kThreadsPerCta, 0, s>>>(coarse_view(h), c.gsplit, c.elem_ptr, c.elem_list,
                                                               h->conn, h->coords, z, h->material, h->bc_mask, n, c.E);
    PLATO_LAUNCH_CHECK(h);
    k_regularize<<<grid_for(n, 256), 256, 0, s>>>(n, c.E);
    PLATO_LAUNCH_CHECK(h);
    if (h->timing) PLATO_CUDA(h, cudaEventRecord(h->coarse_ev[1], s));
    if (E_copy) PLATO_CUDA(h, cudaMemcpyAsync(E_copy, c.E, sizeof(double) * nn, cudaMemcpyDeviceToDevice, s));
    // The factorization and inversion chain is the same launch sequence every solve (its
    // kernels read only E and the coarse scratch): captured once into a CUDA graph and replayed,
    // so the host does not spend a launch per tile step while the fine-level set-up waits.
    if (!c.chain) PLATO_RC(capture_factorization(h));
    PLATO_CUDA(h, cudaGraphLaunch(c.chain, s));
    h->launches += c.chain_launches;
    if (h->timing) PLATO_CUDA(h, cudaEventRecord(h->coarse_ev[2], s));
    PLATO_CUDA(h, cudaMemcpyAsync(c.flag_host, c.flag, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    PLATO_CUDA(h, cudaEventRecord(c.ev_ready, s));
    c.pending = 1;
    if (deferred) return PLATO_OK;
    PLATO_RC(coarse_wait(h));
    return coarse_finish(h);
}

// Marks the point of the handle's stream after which the next coarse set-up may start (its
// control is final there), so that fine-level work queued in between does not delay it.
int coarse_mark_start(plato_problem* h) {
    CoarseSpace& c = h->coarse;
    if (!c.ev_start) PLATO_CUDA(h, cudaEventCreateWithFlags(&c.ev_start, cudaEventDisableTiming));
    PLATO_CUDA(h, cudaEventRecord(c.ev_start, h->stream));
    c.start_marked = 1;
    return PLATO_OK;
}

int coarse_wait(plato_problem* h) {
    CoarseSpace& c = h->coarse;
    if (c.pending) PLATO_CUDA(h, cudaStreamWaitEvent(h->stream, c.ev_ready, 0));
    return PLATO_OK;
}

int coarse_finish(plato_problem* h) {
    CoarseSpace& c = h->coarse;
    if (!c.pending) return PLATO_OK;
    PLATO_CUDA(h, cudaEventSynchronize(c.ev_ready));
    c.pending = 0;
    if (h->timing) {
        float ms[2] = {0.f, 0.f};
        PLATO_CUDA(h, cudaEventElapsedTime(&ms[0], h->coarse_ev[0], h->coarse_ev[1]));
        PLATO_CUDA(h, cudaEventElapsedTime(&ms[1], h->coarse_ev[1], h->coarse_ev[2]));
        h->coarse_gal_ms += ms[0];
        h->coarse_inv_ms += ms[1];
        h->coarse_timed += 1;
    }
    if (*c.flag_host) return plato_fail(h, PLATO_NONFINITE, "coarse operator is not positive definite");
    return PLATO_OK;
}

// y (FP32) = / += Z E^-1 Z^T v (v FP32); kernels return at once after convergence.  With sq
// (the scaled mixed precision, v and y in D^1/2-scaled variables): y += sq Z E^-1 Z^T (sq v).
int coarse_apply(plato_problem* h, const float* v, float* y, int accumulate, const PcgScalars* S, const float* sq) {
    CoarseSpace& c = h->coarse;
    cudaStream_t s = h->stream;
    const CoarseView cv = coarse_view(h);
    // programmatic dependent launches (see launch_pdl): each kernel waits for its predecessor
    PLATO_CUDA(h, launch_pdl(k_restrict_cells, c.ncells * c.rsplit, kThreadsPerCta, s, cv, c.rsplit,
                             (const int32_t*)c.node_ptr, (const int32_t*)c.node_list, (const double*)h->coords,
                             (const uint8_t*)h->bc_mask, v, sq, c.rpart, S));
    PLATO_CUDA(h, launch_pdl(k_restrict_sum, grid_for(c.ndof, 256), 256, s, cv, c.rsplit, (const double*)c.rpart,
                             c.rc, S));
    const int GB = std::min(c.ndof, 148 * 16);  // a CTA per row
    PLATO_CUDA(h, launch_pdl(k_coarse_trmv<true>, GB, 128, s, c.ndof, c.ldf, (const float*)c.Xf, (const double*)c.rc,
                             c.tc, S));
    PLATO_CUDA(h, launch_pdl(k_coarse_trmv<false>, GB, 128, s, c.ndof, c.ldf, (const float*)c.Uf, (const double*)c.tc,
                             c.yc, S));
    PLATO_CUDA(h, launch_pdl(k_prolong, grid_for(h->N, 256), 256, s, h->N, cv, (const double*)h->coords,
                             (const uint8_t*)h->bc_mask, (const double*)c.yc, sq, y, accumulate, S));
    h->launches += 4;
    PLATO_LAUNCH_CHECK(h);
    return PLATO_OK;
}

}  // namespace plato

extern "C" int plato_coarse_operator(plato_problem* h, const double* z, int32_t* ndof, double* E, double* Einv) {
    using namespace plato;
    if (!h || !ndof) return PLATO_BAD_INPUT;
    if (h->opts.coarse_cells[0] <= 0) return plato_fail(h, PLATO_BAD_INPUT, "no coarse grid in the solver options");
    int rc = coarse_setup_mesh(h);
    if (rc) return rc;
    *ndof = h->coarse.ndof;
    if (!E && !Einv) return PLATO_OK;
    if (!z) return plato_fail(h, PLATO_BAD_INPUT, "null control");
    const size_t nn = size_t(h->coarse.ndof) * h->coarse.ndof;
    h->coarse.start_marked = 0;  // z is final at this point of the stream
    double* Ed = nullptr;
    PLATO_CUDA(h, cudaMalloc(&Ed, sizeof(double) * nn));
    rc = coarse_setup_operator(h, z, Ed);
    if (!rc && E) rc = cudaMemcpy(E, Ed, sizeof(double) * nn, cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : PLATO_CUDA_ERROR;
    if (!rc && Einv) {  // E^-1 = X^T X, formed here only (the solver applies X and X^T)
        const int nblk = (h->coarse.ndof + kNB - 1) / kNB;
        k_gram<<<dim3(nblk, nblk), 256, 0, h->stream>>>(h->coarse.ndof, nblk, h->coarse.X, h->coarse.T);
        rc = cudaGetLastError() == cudaSuccess ? 0 : PLATO_CUDA_ERROR;
        if (!rc) rc = cudaMemcpy(Einv, h->coarse.T, sizeof(double) * nn, cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : PLATO_CUDA_ERROR;
    }
    cudaFree(Ed);
    return rc;
}
