// Block-CRS assembly of (dR/dz)^T (1x3 blocks), the warp-per-row Jacobian path for
// high-valence rows (the thread-per-row kernel of assembly_rows.cu assembles the others), and
// the symmetric Dirichlet elimination.
//
// The reference assembles cell by cell with one FP64 atomic per entry and finds each entry
// by a linear search of its row (assemble_jacobian_fad, src/Assembly.hpp:1374-1438;
// BlockMatrixEntryOrdinal, src/ImplicitFunctors.hpp:730-766).  Here the assembly is
// node-centric: one warp owns one block row and writes it exactly once, coalesced, with no
// global atomics.
//
// K(z) (k_assemble_jacobian): the lanes take the row node's incident cells, one cell each,
// and compute its gradients and weight w = vol s(rho) once.  The isotropic block of a cell is
//   K_ab = w (lambda g_a g_b^T + mu g_b g_a^T + mu (g_a . g_b) I),
// so each block of the row is K = lambda M + mu M^T + mu tr(M) I with M = sum_cells w g_a g_b^T.
// Lanes then switch roles: the contributions are bucketed by block slot with __match_any_sync
// (no atomics), each lane owns one off-diagonal block and sums its M in registers, and the
// diagonal block (every incident cell contributes) is a warp butterfly reduction.
#include "plato_internal.cuh"

namespace plato {
namespace {

constexpr int kWarpsPerBlock = 8;
constexpr int kMaxRowBlocks = 64;  // (dR/dz)^T rows with more blocks take the global-atomic path

__device__ __forceinline__ int find_slot(const int32_t* cols, int n, int32_t node) {
    // rows are sorted: binary search
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (cols[mid] < node) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// ---- K(z) -----------------------------------------------------------------------------------

constexpr int kJacWarps = 4;
constexpr int kFastCells = 32;   // rows with at most this many incident cells and blocks use the
constexpr int kFastBlocks = 32;  // register path; larger rows accumulate with global atomics

struct JacRowSmem {
    int32_t cols[kFastBlocks];
    int32_t count[kFastBlocks];                // contributions bucketed into each block slot
    uint8_t rec[kFastCells][kFastBlocks];      // [k][slot] = lane * 4 + local node of the k-th one
    double  wga[kFastCells][3];                // w g_a of each incident cell (a = the row node)
    double  g[kFastCells][12];                 // the 4 gradients of each cell; reused for the output
};
static_assert(9 * kFastBlocks <= 12 * kFastCells, "output staging must fit in the gradient area");

// The row kernel of assembly_rows.cu writes only the upper blocks of a narrow row and leaves
// its lower blocks to the rows that own them as upper blocks.  A wide row assembled here
// (`wide` given) therefore also writes the transpose of each of its upper blocks into the
// neighbour's row when that neighbour is narrow; a wide neighbour writes its own row.
__device__ __forceinline__ void transpose_upper_blocks(const GraphView& g, const uint8_t* __restrict__ wide,
                                                       double* __restrict__ entries, int64_t row, int lane) {
    const int32_t rs = g.row_map[row], nbk = g.row_map[row + 1] - rs;
    for (int k = g.diag[row] - rs + 1 + lane; k < nbk; k += 32) {
        const int32_t c = g.cols[rs + k];
        if (wide[c]) continue;
        const int32_t cs = g.row_map[c];
        const double* src = entries + 9 * ((int64_t)rs + k);
        double* dst = entries + 9 * ((int64_t)cs + find_slot(g.cols + cs, g.row_map[c + 1] - cs, int32_t(row)));
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) dst[3 * i + j] = src[3 * j + i];
    }
}

// Rows beyond the fast-path limits: every lane walks cells and adds its four blocks with
// global FP64 atomics into the zeroed row (general meshes with high-valence nodes).
__device__ __noinline__ void jacobian_row_atomic(const MeshView& m, const GraphView& g, const Material& mat,
                                                 const double* __restrict__ z, double* __restrict__ entries,
                                                 int64_t row, int lane, const uint8_t* __restrict__ wide) {
    const int32_t rs = g.row_map[row], nbk = g.row_map[row + 1] - rs;
    for (int64_t t = lane; t < (int64_t)nbk * 9; t += 32) entries[9 * (int64_t)rs + t] = 0.0;
    __syncwarp();
    for (int32_t k = g.n2c_ptr[row] + lane; k < g.n2c_ptr[row + 1]; k += 32) {
        const int32_t packed = g.n2c[k];
        const int32_t c = packed >> 2, la = packed & 3;
        const int4 n = m.conn[c];
        double x[4][3];
        load_cell_coords(m.coords, n, x);
        TetGeom<double> G;
        tet_geometry(x, G);
        const double rho = cell_rho(mat, z, c, n);
        const double w = G.vol * simp(mat, rho);
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            double Kb[9];
            stiffness_block(mat, G.g[la], G.g[b], w, Kb);
            const int slot = find_slot(g.cols + rs, nbk, node_of(n, b));
#pragma unroll
            for (int q = 0; q < 9; ++q) atomicAdd(&entries[9 * ((int64_t)rs + slot) + q], Kb[q]);
        }
    }
    __syncwarp();
    if (wide) transpose_upper_blocks(g, wide, entries, row, lane);
}

// Warp per block row over the rows in `rows` (count of them): the path for rows with more
// blocks than the thread-per-row kernel (assembly_rows.cu) holds.
__global__ void __launch_bounds__(kJacWarps * 32, 5)
k_assemble_jacobian(MeshView m, GraphView g, Material mat, const double* __restrict__ z,
                    double* __restrict__ entries, const int32_t* __restrict__ rows, int32_t count,
                    const uint8_t* __restrict__ wide) {
    __shared__ JacRowSmem sm[kJacWarps];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    JacRowSmem& S = sm[wib];
    const double c01 = mat.c01, c33 = mat.c33;
    const int64_t warps_total = (int64_t)gridDim.x * kJacWarps;
    for (int64_t it = blockIdx.x * (int64_t)kJacWarps + wib; it < count; it += warps_total) {
        const int64_t row = rows[it];
        const int32_t rs = g.row_map[row];
        const int nbk = g.row_map[row + 1] - rs;
        const int32_t ks = g.n2c_ptr[row];
        const int ncell = g.n2c_ptr[row + 1] - ks;
        if (nbk > kFastBlocks || ncell > kFastCells) {  // warp-uniform
            jacobian_row_atomic(m, g, mat, z, entries, row, lane, wide);
            continue;
        }
        if (lane < nbk) {
            S.cols[lane] = g.cols[rs + lane];
            S.count[lane] = 0;
        }
        __syncwarp();

        // 1. one incident cell per lane: gradients, weight, diagonal contribution w g_a g_a^T
        const bool active = lane < ncell;
        int4 n = make_int4(0, 0, 0, 0);
        int la = -1;
        double d[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // xx yy zz yz xz xy
        if (active) {
            const int32_t packed = g.n2c[ks + lane];
            la = packed & 3;
            n = m.conn[packed >> 2];
            double x[4][3];
            load_cell_coords(m.coords, n, x);
            TetGeom<double> G;
            tet_geometry(x, G);
            const double rho = cell_rho(mat, z, packed >> 2, n);
            const double w = G.vol * simp(mat, rho);
            double ga[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) ga[i] = la == 0 ? G.g[0][i] : la == 1 ? G.g[1][i] : la == 2 ? G.g[2][i] : G.g[3][i];
            const double a0 = w * ga[0], a1 = w * ga[1], a2 = w * ga[2];
            S.wga[lane][0] = a0;
            S.wga[lane][1] = a1;
            S.wga[lane][2] = a2;
#pragma unroll
            for (int b = 0; b < 4; ++b)
#pragma unroll
                for (int i = 0; i < 3; ++i) S.g[lane][3 * b + i] = G.g[b][i];
            d[0] = a0 * ga[0]; d[1] = a1 * ga[1]; d[2] = a2 * ga[2];
            d[3] = a1 * ga[2]; d[4] = a0 * ga[2]; d[5] = a0 * ga[1];
        }

        // 2. bucket the off-diagonal contributions (cell, local node b) by block slot
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int key = (active && b != la) ? find_slot(S.cols, nbk, node_of(n, b)) : -1;
            const unsigned peers = __match_any_sync(0xffffffffu, key);
            const int rank = __popc(peers & below);
            if (key >= 0) S.rec[S.count[key] + rank][key] = uint8_t(lane * 4 + b);
            __syncwarp();
            if (key >= 0 && rank == 0) S.count[key] += __popc(peers);
            __syncwarp();
        }

        // 3. diagonal block: butterfly sum of the incident cells' w g_a g_a^T
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
#pragma unroll
            for (int q = 0; q < 6; ++q) d[q] += __shfl_xor_sync(0xffffffffu, d[q], off);

        // 4. lane = block slot: M = sum w g_a g_b^T, K = lambda M + mu M^T + mu tr(M) I
        const int dslot = g.diag[row] - rs;
        double K[9];
        if (lane < nbk) {
            double M[9];
            if (lane == dslot) {
                M[0] = d[0]; M[4] = d[1]; M[8] = d[2];
                M[5] = M[7] = d[3];
                M[2] = M[6] = d[4];
                M[1] = M[3] = d[5];
            } else {
#pragma unroll
                for (int q = 0; q < 9; ++q) M[q] = 0.0;
                const int cnt = S.count[lane];
                for (int r = 0; r < cnt; ++r) {
                    const int code = S.rec[r][lane];
                    const int c = code >> 2, b = code & 3;
                    const double a[3] = {S.wga[c][0], S.wga[c][1], S.wga[c][2]};
                    const double gb[3] = {S.g[c][3 * b], S.g[c][3 * b + 1], S.g[c][3 * b + 2]};
#pragma unroll
                    for (int i = 0; i < 3; ++i)
#pragma unroll
                        for (int j = 0; j < 3; ++j) M[3 * i + j] = fma(a[i], gb[j], M[3 * i + j]);
                }
            }
            const double tr = c33 * (M[0] + M[4] + M[8]);
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) K[3 * i + j] = c01 * M[3 * i + j] + c33 * M[3 * j + i] + (i == j ? tr : 0.0);
        }
        __syncwarp();  // every read of S.g is done before it becomes the output stage
        double* out = &S.g[0][0];
        if (lane < nbk)
#pragma unroll
            for (int q = 0; q < 9; ++q) out[9 * lane + q] = K[q];
        __syncwarp();
        double* dst = entries + 9 * (int64_t)rs;
        for (int q = lane; q < 9 * nbk; q += 32) dst[q] = out[q];
        __syncwarp();
        if (wide) transpose_upper_blocks(g, wide, entries, row, lane);
    }
}

// ---- (dR/dz)^T --------------------------------------------------------------------------------

template <int BS>
struct RowSmem {
    int32_t cols[kMaxRowBlocks];
    double  acc[kMaxRowBlocks * BS];
};

// (dR/dz)^T with 1x3 blocks: entry (a, (b,d)) = sum over cells of dR_(b,d)/dz_a
// = vol s'(rho)/4 (B_b^T sigma0(u))_d.  Lanes take the row node's cells and accumulate the
// four 1x3 blocks of each in shared memory.
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
k_assemble_dRdz_rows(MeshView m, GraphView g, Material mat, const double* __restrict__ z,
                     const double* __restrict__ u, double* __restrict__ entries) {
    constexpr int BS = 3;
    __shared__ RowSmem<BS> sm[kWarpsPerBlock];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    RowSmem<BS>& S = sm[wib];
    const int64_t warps_total = (int64_t)gridDim.x * kWarpsPerBlock;
    for (int64_t row = blockIdx.x * (int64_t)kWarpsPerBlock + wib; row < g.num_nodes; row += warps_total) {
        const int32_t rs = g.row_map[row], re = g.row_map[row + 1];
        const int nbk = re - rs;
        const bool fast = nbk <= kMaxRowBlocks;
        if (fast) {
            for (int t = lane; t < nbk; t += 32) S.cols[t] = g.cols[rs + t];
            for (int t = lane; t < nbk * BS; t += 32) S.acc[t] = 0.0;
        } else {
            for (int64_t t = lane; t < (int64_t)nbk * BS; t += 32) entries[(int64_t)BS * rs + t] = 0.0;
        }
        __syncwarp();
        const int32_t ks = g.n2c_ptr[row], ke = g.n2c_ptr[row + 1];
        for (int32_t k = ks + lane; k < ke; k += 32) {
            const int32_t packed = g.n2c[k];
            const int32_t c = packed >> 2;
            const int4 n = m.conn[c];
            double x[4][3];
            load_cell_coords(m.coords, n, x);
            TetGeom<double> G;
            tet_geometry(x, G);
            const double rho = cell_rho(mat, z, c, n);
            double ue[4][3], e[6], s[6];
            const int ids[4] = {n.x, n.y, n.z, n.w};
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int d = 0; d < 3; ++d) ue[a][d] = __ldg(u + 3 * (int64_t)ids[a] + d);
            strain_voigt(G.g, ue, e);
            stress_voigt(mat, e, s);
            const double w = G.vol * simp_dx(mat, rho) * rho_dz(mat);
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                double f[3];
                divergence_node(G.g[b], s, w, f);
                const int32_t nb = ids[b];
                if (fast) {
                    const int slot = find_slot(S.cols, nbk, nb);
#pragma unroll
                    for (int q = 0; q < 3; ++q) atomicAdd(&S.acc[3 * slot + q], f[q]);
                } else {
                    const int slot = find_slot(g.cols + rs, nbk, nb);
#pragma unroll
                    for (int q = 0; q < 3; ++q) atomicAdd(&entries[3 * ((int64_t)rs + slot) + q], f[q]);
                }
            }
        }
        __syncwarp();
        if (fast)
            for (int t = lane; t < nbk * BS; t += 32) entries[(int64_t)BS * rs + t] = S.acc[t];
        __syncwarp();
    }
}

// applyBlockConstraints<3>, first loop (src/ApplyConstraints.hpp:68-104): for BC dof d,
// diag = 1, every other entry of row d is zeroed after lifting rhs_j -= A_dj * value, and the
// mirror entry (j, d) is zeroed too.
__global__ void k_dirichlet_rows(int32_t nbc, const int32_t* __restrict__ dofs,
                                 const double* __restrict__ vals, double scale,
                                 const int32_t* __restrict__ row_map, const int32_t* __restrict__ cols,
                                 double* __restrict__ A, double* __restrict__ rhs) {
    for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < nbc;
         b += (int64_t)gridDim.x * blockDim.x) {
        const int32_t rdof = dofs[b];
        const double value = scale * vals[b];
        const int32_t rnode = rdof / 3, lr = rdof % 3;
        for (int32_t off = row_map[rnode]; off < row_map[rnode + 1]; ++off) {
            const int32_t cnode = cols[off];
            for (int lc = 0; lc < 3; ++lc) {
                const int64_t e = 9 * (int64_t)off + 3 * lr + lc;
                const int32_t cdof = 3 * cnode + lc;
                if (cdof == rdof) {
                    A[e] = 1.0;
                } else {
                    if (rhs && value != 0.0) atomicAdd(&rhs[cdof], -A[e] * value);
                    A[e] = 0.0;
                    for (int32_t off2 = row_map[cnode]; off2 < row_map[cnode + 1]; ++off2)
                        if (cols[off2] == rnode) A[9 * (int64_t)off2 + 3 * lc + lr] = 0.0;
                }
            }
        }
    }
}

// Second loop (src/ApplyConstraints.hpp:106-110): rhs_d = value.
__global__ void k_dirichlet_rhs(int32_t nbc, const int32_t* __restrict__ dofs,
                                const double* __restrict__ vals, double scale, double* __restrict__ rhs) {
    for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < nbc;
         b += (int64_t)gridDim.x * blockDim.x)
        rhs[dofs[b]] = scale * vals[b];
}

// y += A x for a block CRS with RB x CB blocks: MatrixTimesVectorPlusVector
// (src/PlatoMathHelpers.hpp:78-159).  Thread per (node row, block row i).
template <int RB, int CB>
__global__ void k_matvec_plus(int32_t N, const int32_t* __restrict__ row_map,
                              const int32_t* __restrict__ cols, const double* __restrict__ A,
                              const double* __restrict__ x, double* __restrict__ y) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < (int64_t)N * RB;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int32_t r = int32_t(t / RB);
        const int i = int(t % RB);
        double sum = 0.0;
        for (int32_t k = row_map[r]; k < row_map[r + 1]; ++k) {
            const double* blk = A + (int64_t)RB * CB * k + CB * i;
            const double* xv = x + (int64_t)CB * cols[k];
#pragma unroll
            for (int j = 0; j < CB; ++j) sum += blk[j] * xv[j];
        }
        y[t] += sum;
    }
}

}  // namespace

MeshView mesh_view(const plato_problem* h);
GraphView graph_view(const plato_problem* h);

// The rows in `rows`, whole; with `wide` (the row kernel's wide-row flags) also the transposes
// of their upper blocks into narrow neighbours.
int launch_assemble_jacobian_list(plato_problem* h, const double* z, double* entries, const int32_t* rows,
                                  int32_t count, const uint8_t* wide) {
    if (count <= 0) return PLATO_OK;
    const int blocks = grid_for(count, kJacWarps, 148 * 5 * 8);
    k_assemble_jacobian<<<blocks, kJacWarps * 32, 0, h->stream>>>(mesh_view(h), graph_view(h), h->material, z,
                                                                  entries, rows, count, wide);
    PLATO_LAUNCH_CHECK(h);
    return PLATO_OK;
}

int launch_assemble_gradient_z(plato_problem* h, const double* u, const double* z, double* entries) {
    const int blocks = grid_for(h->N, kWarpsPerBlock, 148 * 64);
    k_assemble_dRdz_rows<<<blocks, kWarpsPerBlock * 32, 0, h->stream>>>(mesh_view(h), graph_view(h), h->material,
                                                                         z, u, entries);
    PLATO_LAUNCH_CHECK(h);
    return PLATO_OK;
}

int launch_dirichlet(plato_problem* h, double* A, double* rhs, double scale) {
    if (h->nbc == 0) return PLATO_OK;
    k_dirichlet_rows<<<grid_for(h->nbc, 128), 128, 0, h->stream>>>(h->nbc, h->bc_dofs, h->bc_values, scale,
                                                                    h->row_map, h->cols, A, rhs);
    PLATO_LAUNCH_CHECK(h);
    if (rhs) {
        k_dirichlet_rhs<<<grid_for(h->nbc, 128), 128, 0, h->stream>>>(h->nbc, h->bc_dofs, h->bc_values, scale, rhs);
        PLATO_LAUNCH_CHECK(h);
    }
    return PLATO_OK;
}

// rhs_d = scale * value_d on constrained dofs only (no matrix).
int launch_dirichlet_rhs(plato_problem* h, double* rhs, double scale) {
    if (h->nbc == 0) return PLATO_OK;
    k_dirichlet_rhs<<<grid_for(h->nbc, 128), 128, 0, h->stream>>>(h->nbc, h->bc_dofs, h->bc_values, scale, rhs);
    PLATO_LAUNCH_CHECK(h);
    return PLATO_OK;
}

int launch_matvec_plus(plato_problem* h, int rb, int cb, const double* A, const double* x, double* y) {
    const int64_t n = (int64_t)h->N * rb;
    if (rb == 3 && cb == 3)
        k_matvec_plus<3, 3><<<grid_for(n, 256), 256, 0, h->stream>>>(h->N, h->row_map, h->cols, A, x, y);
    else if (rb == 1 && cb == 3)
        k_matvec_plus<1, 3><<<grid_for(n, 256), 256, 0, h->stream>>>(h->N, h->row_map, h->cols, A, x, y);
    else
        return plato_fail(h, PLATO_BAD_INPUT, "matvec supports 3x3 and 1x3 blocks");
    PLATO_LAUNCH_CHECK(h);
    return PLATO_OK;
}

}  // namespace plato
