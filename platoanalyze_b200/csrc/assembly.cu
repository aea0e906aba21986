// Block-CRS assembly of the Jacobian K(z) (3x3 blocks) and of (dR/dz)^T (1x3 blocks), and
// the symmetric Dirichlet elimination.
//
// The reference assembles cell by cell with one FP64 atomic per entry and finds each entry
// by a linear search of its row (assemble_jacobian_fad, src/Assembly.hpp:1374-1438;
// BlockMatrixEntryOrdinal, src/ImplicitFunctors.hpp:730-766).  Here the assembly is
// node-centric: one warp owns one block row, its lanes walk the row node's incident cells,
// each lane computes the four 3x3 blocks K_ab of its cell in closed form
// (w B_a^T C B_b), and the row is accumulated in shared memory and written once, coalesced.
// No global atomics; every value is written exactly once.
#include "plato_internal.cuh"

namespace plato {
namespace {

constexpr int kWarpsPerBlock = 8;
constexpr int kMaxRowBlocks = 64;  // rows with more blocks take the global-atomic path

template <int BS>
struct RowSmem {
    int32_t cols[kMaxRowBlocks];
    double  acc[kMaxRowBlocks * BS];
};

__device__ __forceinline__ int find_slot(const int32_t* cols, int n, int32_t node) {
    // rows are sorted: binary search
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (cols[mid] < node) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// MODE 0: K(z) 3x3 blocks.  MODE 1: (dR/dz)^T 1x3 blocks: entry (a, (b,d)) =
// sum over cells of dR_(b,d)/dz_a = vol s'(rho)/4 (B_b^T sigma0(u))_d.
template <int MODE>
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
k_assemble_rows(MeshView m, GraphView g, Material mat, const double* __restrict__ z,
                const double* __restrict__ u, double* __restrict__ entries) {
    constexpr int BS = (MODE == 0) ? 9 : 3;
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
            const int32_t c = packed >> 2, la = packed & 3;
            const int4 n = m.conn[c];
            double x[4][3];
            load_cell_coords(m.coords, n, x);
            TetGeom<double> G;
            tet_geometry(x, G);
            const double rho = (__ldg(z + n.x) + __ldg(z + n.y) + __ldg(z + n.z) + __ldg(z + n.w)) * 0.25;
            const double* ga = G.g[la];
            if (MODE == 0) {
                const double w = G.vol * simp(mat, rho);
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    double Kb[9];
                    stiffness_block(mat, ga, G.g[b], w, Kb);
                    const int32_t nb = node_of(n, b);
                    if (fast) {
                        const int slot = find_slot(S.cols, nbk, nb);
#pragma unroll
                        for (int q = 0; q < 9; ++q) atomicAdd(&S.acc[9 * slot + q], Kb[q]);
                    } else {
                        const int slot = find_slot(g.cols + rs, nbk, nb);
#pragma unroll
                        for (int q = 0; q < 9; ++q) atomicAdd(&entries[9 * ((int64_t)rs + slot) + q], Kb[q]);
                    }
                }
            } else {
                double ue[4][3], e[6], s[6];
                const int ids[4] = {n.x, n.y, n.z, n.w};
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int d = 0; d < 3; ++d) ue[a][d] = __ldg(u + 3 * (int64_t)ids[a] + d);
                strain_voigt(G.g, ue, e);
                stress_voigt(mat, e, s);
                const double w = G.vol * simp_dx(mat, rho) * 0.25;
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

int launch_assemble_jacobian(plato_problem* h, const double* z, double* entries) {
    const int blocks = grid_for(h->N, kWarpsPerBlock, 148 * 64);
    k_assemble_rows<0><<<blocks, kWarpsPerBlock * 32, 0, h->stream>>>(mesh_view(h), graph_view(h),
                                                                       h->material, z, nullptr, entries);
    PLATO_LAUNCH_CHECK(h);
    return PLATO_OK;
}

int launch_assemble_gradient_z(plato_problem* h, const double* u, const double* z, double* entries) {
    const int blocks = grid_for(h->N, kWarpsPerBlock, 148 * 64);
    k_assemble_rows<1><<<blocks, kWarpsPerBlock * 32, 0, h->stream>>>(mesh_view(h), graph_view(h),
                                                                       h->material, z, u, entries);
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
