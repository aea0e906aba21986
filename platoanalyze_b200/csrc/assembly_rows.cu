// Jacobian assembly with one thread per block row.
//
// K(z) row a holds, for every node b sharing a cell with a, the block
//   K_ab = sum over cells e containing a and b of  w_e (lambda g_a g_b^T + mu g_b g_a^T + mu (g_a . g_b) I)
// (w_e = vol_e s(rho_e), g the basis gradients of the cell; StressDivergence of LinearStress
// of Strain, src/StressDivergence.hpp:70-90, src/LinearStress.hpp:102-120, assembled by
// assemble_jacobian_fad, src/Assembly.hpp:1374-1438).  With S_ab = sum_e w_e g_a g_b^T the
// block is lambda S + mu S^T + mu tr(S) I, so a row only needs S for each of its blocks.
//
// One thread owns one row and walks the row's incident cells (the node -> cell incidence
// of the graph, sorted by cell): per cell it gathers the three other nodes' coordinates and
// densities, forms the gradients with the row node as the reference vertex, adds w g_a g_a^T
// to the diagonal block (registers, 6 symmetric components) and w g_a g_b^T into the slot of
// each other node b with a larger index -- the upper blocks only.  K is symmetric, so the
// thread writes each upper block K_ab into its own row and its transpose K_ba into row b;
// every lower block is written exactly once, by the row that owns it as an upper block.
// That halves the shared-memory accumulator (9 values per upper block per thread) and the
// slot updates, and doubles the warps an SM holds.  The slot of each (row, cell, b) and the
// position of the row in each upper neighbour's row are looked up once per mesh (the
// assembly plan: three 4-bit upper-slot numbers per incidence entry, 15 for a lower node;
// one byte per upper block for the mirror slot), so the hot loop has no search and no
// inter-thread reduction.  A warp owns the 32 rows of one SELL slice and the layout of its
// accumulator is [slot][component][lane ^ component]: in the accumulation every lane
// touches the same component at a time, so the 64-bit accesses of a half warp hit 16
// distinct bank pairs; in the row-major write-out (CRS) 16 consecutive entries of one row
// span at most 9 components, two to a bank pair.
//
// Rows with more than kAsmMaxUp upper blocks or more than 255 blocks (high-valence nodes of
// general meshes) are "wide": skipped here and assembled whole, with the transposes of their
// upper blocks, by the warp-per-row kernel of assembly.cu; narrow rows write no transpose
// into a wide row.
//
// Outputs: the reference's block CRS (the API path), or -- for the solver -- the SELL-32
// component-major copy of the constrained matrix directly (applyBlockConstraints with zero
// values, src/ApplyConstraints.hpp:40-112: constrained rows and columns zero, unit
// diagonal), its inverse Jacobi diagonal, and optionally FP32 / BF16 copies, so the solve
// never materialises the 1.12 GB CRS copy of the bench mesh nor re-reads it.
#include <cuda_bf16.h>

#include "plato_internal.cuh"

namespace plato {

int ensure_smem_attribute(plato_problem* h, const void* kernel, int bytes);
MeshView mesh_view(const plato_problem* h);
GraphView graph_view(const plato_problem* h);

namespace {

constexpr int kAsmMaxWarps = 12;         // warps per CTA, one CTA per SM (170 registers each)
constexpr int kAsmMaxUp = 15;            // upper blocks per row held in shared memory (4-bit codes)
constexpr int kAsmMaxBlocks = 255;       // blocks per row with a one-byte mirror slot
constexpr int kAsmSmemMax = 227 * 1024;  // dynamic shared memory per CTA
constexpr uint8_t kNoMirror = 255;       // the upper neighbour is wide: it writes its own row

// Accumulator layout [upper slot][component][lane]: the SELL output reads a thread's own
// entries back, so the lanes of one access are 32 consecutive doubles (conflict free per half
// warp); the CRS output writes each row as one contiguous run, so there the lane index is
// swizzled by the component (16 consecutive entries of a row then span 9 bank pairs).
template <bool kSwizzle>
__device__ __forceinline__ int acc_lane_t(int lane, int q) { return kSwizzle ? (lane ^ q) : lane; }
template <bool kSell>
__device__ __forceinline__ int acc_index(int u, int q, int lane) { return (9 * u + q) * 32 + acc_lane_t<!kSell>(lane, q); }

__device__ __forceinline__ int warp_max(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ int row_slot(const int32_t* cols, int n, int32_t node) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (cols[mid] < node) lo = mid + 1; else hi = mid;
    }
    return lo;
}

struct SellOut {
    const int64_t* ptr;      // SELL slice offsets
    const int32_t* cols;     // SELL column node of each slot
    const uint8_t* bc_mask;  // [3N] constrained dofs
    double* v64;             // FP64 entries (component-major SELL)
    float* v32;              // optional FP32 copy
    __nv_bfloat16* v16;      // optional BF16 copy
    double* dinv;            // [3N] inverse diagonal of the constrained matrix
    float* dinv32;           // optional FP32 copy of it
};

// Per mesh, pass 1: the wide rows (list + flags) and the largest upper-block count of the others.
__global__ void k_asm_flags(GraphView g, uint8_t* __restrict__ wide, int32_t* __restrict__ list,
                            int32_t* __restrict__ nwide, int32_t* __restrict__ maxup) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < g.num_nodes;
         r += (int64_t)gridDim.x * blockDim.x) {
        const int32_t rs = g.row_map[r], nb = g.row_map[r + 1] - rs;
        const int32_t nup = nb - (g.diag[r] - rs) - 1;
        const bool w = nup > kAsmMaxUp || nb > kAsmMaxBlocks;
        wide[r] = w ? 1 : 0;
        if (w) list[atomicAdd(nwide, 1)] = int32_t(r);
        else atomicMax(maxup, nup);
    }
}

// Per mesh, pass 2 (narrow rows): for every (row, incident cell) entry of n2c, the upper slots
// of the cell's three other nodes (ascending local ordinal), 4 bits each, 15 for a node with a
// smaller index; for every upper block, the slot of the row in the neighbour's row
// (kNoMirror when the neighbour is wide).
__global__ void k_asm_plan(GraphView g, const int4* __restrict__ conn, const uint8_t* __restrict__ wide,
                           uint16_t* __restrict__ plan, uint8_t* __restrict__ mirror) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < g.num_nodes;
         r += (int64_t)gridDim.x * blockDim.x) {
        if (wide[r]) continue;
        const int32_t rs = g.row_map[r], nb = g.row_map[r + 1] - rs;
        const int dslot = g.diag[r] - rs;
        for (int32_t k = g.n2c_ptr[r]; k < g.n2c_ptr[r + 1]; ++k) {
            const int32_t packed = g.n2c[k];
            const int la = packed & 3;
            const int4 n = conn[packed >> 2];
            uint32_t code = 0;
            int t = 0;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                if (b == la) continue;
                const int slot = row_slot(g.cols + rs, nb, node_of(n, b));
                code |= uint32_t(slot > dslot ? slot - dslot - 1 : 15) << (4 * t);
                ++t;
            }
            plan[k] = uint16_t(code);
        }
        for (int k = dslot + 1; k < nb; ++k) {
            const int32_t c = g.cols[rs + k];
            const int32_t cs = g.row_map[c];
            mirror[rs + k] = wide[c] ? kNoMirror : uint8_t(row_slot(g.cols + cs, g.row_map[c + 1] - cs, int32_t(r)));
        }
    }
}

__device__ __forceinline__ void store_sell(const SellOut& so, int64_t o, double v) {
    if (so.v64) so.v64[o] = v;
    if (so.v32) so.v32[o] = float(v);
    if (so.v16) so.v16[o] = __float2bfloat16_rn(float(v));
}

// T = double, kSell = false: block CRS values (unconstrained) into crs[9 * nblocks].
// T = double, kSell = true:  constrained SELL copy + inverse diagonal (+ optional FP32 / BF16
//                            copies rounded from the FP64 values) into `so`.
// T = float,  kSell = true:  FP32 element assembly -- gradients, weights and sums in FP32 -- of
//                            the constrained SELL copy (so.v32) and its inverse diagonal
//                            (so.dinv32), the preconditioner matrix of the mixed-precision solve
//                            whose FP64 outer operator is the matrix-free element apply.
// `up` is the largest upper-block count of the narrow rows: each warp's accumulator holds
// 9 x 32 x up values and the CTA as many warps as the shared memory takes (at most 14).
template <bool kSell, typename T>
__global__ void __launch_bounds__(kAsmMaxWarps * 32, 1)
k_assemble_rows(MeshView m, GraphView g, Material mat, const double* __restrict__ z,
                const uint16_t* __restrict__ plan, const uint8_t* __restrict__ mirror,
                const uint8_t* __restrict__ wide, int up, double* __restrict__ crs, SellOut so) {
    const int nwarps = blockDim.x >> 5;
    extern __shared__ double smem_raw[];
    T* smem = reinterpret_cast<T*>(smem_raw);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    T* acc = smem + warp * (9 * 32 * up);
    const T lam = T(mat.c01), mu = T(mat.c33);
    const int32_t nslices = (g.num_nodes + 31) >> 5;
    for (int32_t s = blockIdx.x * nwarps + warp; s < nslices; s += gridDim.x * nwarps) {
        const int32_t r = 32 * s + lane;
        int32_t rs = 0, nb = 0, ks = 0, kc = 0, dslot = -1, nup = 0;
        T xr[3] = {T(0), T(0), T(0)}, zr = T(0);
        if (r < g.num_nodes) {
            rs = g.row_map[r];
            nb = g.row_map[r + 1] - rs;
            if (!wide[r]) {
                ks = g.n2c_ptr[r];
                kc = g.n2c_ptr[r + 1] - ks;
                dslot = g.diag[r] - rs;
                nup = nb - dslot - 1;
                xr[0] = T(__ldg(m.coords + 3 * (int64_t)r));
                xr[1] = T(__ldg(m.coords + 3 * (int64_t)r + 1));
                xr[2] = T(__ldg(m.coords + 3 * (int64_t)r + 2));
                zr = mat.cell_control ? T(0) : T(__ldg(z + r));
            }
        }
        const int nupw = warp_max(nup);
        for (int u = 0; u < nupw; ++u)
#pragma unroll
            for (int q = 0; q < 9; ++q) acc[acc_index<kSell>(u, q, lane)] = T(0);
        __syncwarp();
        T d0 = T(0), d1 = T(0), d2 = T(0), d3 = T(0), d4 = T(0), d5 = T(0);  // xx yy zz yz xz xy
        const int kmax = warp_max(kc);
        // Two-stage prefetch: the incidence entry, plan and connectivity two cells ahead, the
        // three other nodes' coordinates and controls one cell ahead, so each cell's gathers are
        // in flight during the previous cell's arithmetic.
        int32_t pA = 0, pB = 0;  // cells j + 1 (connectivity loaded) and j (geometry loaded)
        uint32_t plA = 0, plB = 0;
        int4 nA = make_int4(0, 0, 0, 0);
        double cx[9], cz[3];
        auto load_geometry = [&](int32_t pk, int4 nk) {
            const int la = pk & 3;  // the three other nodes in ascending local order
            const int32_t i0 = la == 0 ? nk.y : nk.x;
            const int32_t i1 = la <= 1 ? nk.z : nk.y;
            const int32_t i2 = la <= 2 ? nk.w : nk.z;
            const double* c0 = m.coords + 3 * (int64_t)i0;
            const double* c1 = m.coords + 3 * (int64_t)i1;
            const double* c2 = m.coords + 3 * (int64_t)i2;
            cx[0] = __ldg(c0); cx[1] = __ldg(c0 + 1); cx[2] = __ldg(c0 + 2);
            cx[3] = __ldg(c1); cx[4] = __ldg(c1 + 1); cx[5] = __ldg(c1 + 2);
            cx[6] = __ldg(c2); cx[7] = __ldg(c2 + 1); cx[8] = __ldg(c2 + 2);
            if (mat.cell_control) {
                cz[0] = __ldg(z + (pk >> 2));
                cz[1] = cz[2] = 0.0;
            } else {
                cz[0] = __ldg(z + i0);
                cz[1] = __ldg(z + i1);
                cz[2] = __ldg(z + i2);
            }
        };
        if (kc > 0) {
            pB = __ldg(g.n2c + ks);
            plB = __ldg(plan + ks);
            load_geometry(pB, __ldg(m.conn + (pB >> 2)));
        }
        if (kc > 1) {
            pA = __ldg(g.n2c + ks + 1);
            plA = __ldg(plan + ks + 1);
            nA = __ldg(m.conn + (pA >> 2));
        }
#pragma unroll 1
        for (int j = 0; j < kmax; ++j) {
            const uint32_t pl = plB;
            double x9[9], z3[3];
#pragma unroll
            for (int e = 0; e < 9; ++e) x9[e] = cx[e];
#pragma unroll
            for (int e = 0; e < 3; ++e) z3[e] = cz[e];
            if (j + 1 < kc) {
                pB = pA;
                plB = plA;
                load_geometry(pA, nA);
            }
            if (j + 2 < kc) {
                pA = __ldg(g.n2c + ks + j + 2);
                plA = __ldg(plan + ks + j + 2);
                nA = __ldg(m.conn + (pA >> 2));
            }
            if (j < kc) {
                const T j11 = T(x9[0]) - xr[0], j21 = T(x9[1]) - xr[1], j31 = T(x9[2]) - xr[2];
                const T j12 = T(x9[3]) - xr[0], j22 = T(x9[4]) - xr[1], j32 = T(x9[5]) - xr[2];
                const T j13 = T(x9[6]) - xr[0], j23 = T(x9[7]) - xr[1], j33 = T(x9[8]) - xr[2];
                const T rho = mat.cell_control ? T(z3[0]) : (T(z3[0]) + T(z3[1]) + T(z3[2]) + zr) * T(0.25);
                // ComputeGradientWorkset<3> (src/ImplicitFunctors.hpp:169-221) with x_3 = the row node
                const T c11 = j22 * j33 - j23 * j32, c12 = j13 * j32 - j12 * j33, c13 = j12 * j23 - j13 * j22;
                const T detj = j11 * c11 + j21 * c12 + j31 * c13;
                const T inv = T(1) / detj;
                T gb[3][3];
                gb[0][0] = c11 * inv;
                gb[0][1] = c12 * inv;
                gb[0][2] = c13 * inv;
                gb[1][0] = (j23 * j31 - j21 * j33) * inv;
                gb[1][1] = (j11 * j33 - j13 * j31) * inv;
                gb[1][2] = (j13 * j21 - j11 * j23) * inv;
                gb[2][0] = (j21 * j32 - j22 * j31) * inv;
                gb[2][1] = (j12 * j31 - j11 * j32) * inv;
                gb[2][2] = (j11 * j22 - j12 * j21) * inv;
                const T w = fabs(detj) * (T(1) / T(6)) * simp(mat, rho);
                const T ga0 = -(gb[0][0] + gb[1][0] + gb[2][0]);
                const T ga1 = -(gb[0][1] + gb[1][1] + gb[2][1]);
                const T ga2 = -(gb[0][2] + gb[1][2] + gb[2][2]);
                const T a0 = w * ga0, a1 = w * ga1, a2 = w * ga2;
                d0 = fma(a0, ga0, d0);
                d1 = fma(a1, ga1, d1);
                d2 = fma(a2, ga2, d2);
                d3 = fma(a1, ga2, d3);
                d4 = fma(a0, ga2, d4);
                d5 = fma(a0, ga1, d5);
#pragma unroll
                for (int t = 0; t < 3; ++t) {
                    const int u = (pl >> (4 * t)) & 15;
                    if (u == 15) continue;  // a lower node: its row writes the block
                    T* row = acc + 9 * 32 * u;
#pragma unroll
                    for (int q = 0; q < 9; ++q) {
                        const T ai = q < 3 ? a0 : (q < 6 ? a1 : a2);
                        T& v = row[q * 32 + acc_lane_t<!kSell>(lane, q)];
                        v = fma(ai, gb[t][q % 3], v);
                    }
                }
            }
        }
        __syncwarp();

        // K = lambda S + mu S^T + mu tr(S) I per block
        T Kd[9];  // the diagonal block
        {
            const T tr = mu * (d0 + d1 + d2);
            const T S[9] = {d0, d5, d4, d5, d1, d3, d4, d3, d2};
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int jj = 0; jj < 3; ++jj)
                    Kd[3 * i + jj] = lam * S[3 * i + jj] + mu * S[3 * jj + i] + (i == jj ? tr : T(0));
        }
        if (kSell) {
            // own row: slots k of the slice (width nbw); lower slots k < dslot are left to the
            // transposes, slots k >= nb of the slice are zero padding
            const int nbw = warp_max(nb);
            const int64_t pbase = __ldg(so.ptr + s);
            const int64_t sbase = 9 * pbase;
            // constrained components of the row, read once (a padding lane has nb = 0)
            bool mrow[3] = {false, false, false};
            if (nb > 0)
#pragma unroll
                for (int i = 0; i < 3; ++i) mrow[i] = __ldg(so.bc_mask + 3 * (int64_t)r + i) != 0;
            for (int k = 0; k < nbw; ++k) {
                const bool diag = k == dslot, upper = k > dslot && k < nb, pad = k >= nb;
                if (!(diag || upper || pad)) continue;
                T K[9];
                int32_t c = r;
                if (upper) {
                    const int u = k - dslot - 1;
                    T S[9];
#pragma unroll
                    for (int q = 0; q < 9; ++q) S[q] = acc[acc_index<kSell>(u, q, lane)];
                    const T tr = mu * (S[0] + S[4] + S[8]);
#pragma unroll
                    for (int i = 0; i < 3; ++i)
#pragma unroll
                        for (int jj = 0; jj < 3; ++jj)
                            K[3 * i + jj] = lam * S[3 * i + jj] + mu * S[3 * jj + i] + (i == jj ? tr : T(0));
                    c = __ldg(so.cols + pbase + 32 * k + lane);
                } else {
#pragma unroll
                    for (int q = 0; q < 9; ++q) K[q] = diag ? Kd[q] : T(0);
                }
                // constrained components of the column node, read once per block and reused
                // for the transpose
                bool mcol[3] = {false, false, false};
                if (!pad)
#pragma unroll
                    for (int jj = 0; jj < 3; ++jj) mcol[jj] = __ldg(so.bc_mask + 3 * (int64_t)c + jj) != 0;
#pragma unroll
                for (int q = 0; q < 9; ++q) {
                    const int i = q / 3, jj = q % 3;
                    double v = pad ? 0.0 : double(K[q]);
                    if (!pad && (mrow[i] || mcol[jj])) v = (diag && i == jj) ? 1.0 : 0.0;
                    store_sell(so, sbase + 32 * (9 * k + q) + lane, v);
                    if (diag && i == jj) {
                        if (so.dinv) so.dinv[3 * (int64_t)r + i] = 1.0 / v;
                        if (so.dinv32) so.dinv32[3 * (int64_t)r + i] = float(1.0 / v);
                    }
                }
                if (upper) {  // the transpose into row c: K_cr[i][j] = K_rc[j][i]
                    const uint8_t ms = __ldg(mirror + rs + k);
                    if (ms != kNoMirror) {
                        const int64_t cb = 9 * __ldg(so.ptr + (c >> 5)) + 32 * 9 * int64_t(ms) + (c & 31);
#pragma unroll
                        for (int q = 0; q < 9; ++q) {
                            const int i = q / 3, jj = q % 3;
                            store_sell(so, cb + 32 * q, (mcol[i] || mrow[jj]) ? 0.0 : double(K[3 * jj + i]));
                        }
                    }
                }
            }
        } else {
            // upper blocks: K back into the accumulator, the transposes straight to row c
            for (int u = 0; u < nup; ++u) {
                T S[9];
#pragma unroll
                for (int q = 0; q < 9; ++q) S[q] = acc[acc_index<kSell>(u, q, lane)];
                const T tr = mu * (S[0] + S[4] + S[8]);
                T K[9];
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int jj = 0; jj < 3; ++jj)
                        K[3 * i + jj] = lam * S[3 * i + jj] + mu * S[3 * jj + i] + (i == jj ? tr : T(0));
#pragma unroll
                for (int q = 0; q < 9; ++q) acc[acc_index<kSell>(u, q, lane)] = K[q];
                const int k = dslot + 1 + u;
                const uint8_t ms = __ldg(mirror + rs + k);
                if (ms != kNoMirror) {
                    const int32_t c = __ldg(g.cols + rs + k);
                    double* dst = crs + 9 * ((int64_t)__ldg(g.row_map + c) + ms);
#pragma unroll
                    for (int i = 0; i < 3; ++i)
#pragma unroll
                        for (int jj = 0; jj < 3; ++jj) dst[3 * i + jj] = double(K[3 * jj + i]);
                }
            }
            if (dslot >= 0) {
                double* dst = crs + 9 * ((int64_t)rs + dslot);
#pragma unroll
                for (int q = 0; q < 9; ++q) dst[q] = double(Kd[q]);
            }
            __syncwarp();
            // row-major write-out of the upper blocks: one contiguous run per row
            for (int l = 0; l < 32; ++l) {
                const int nv = 9 * __shfl_sync(0xffffffffu, nup, l);
                if (nv == 0) continue;
                const int32_t st = __shfl_sync(0xffffffffu, rs + dslot + 1, l);
                double* dst = crs + 9 * (int64_t)st;
                for (int e = lane; e < nv; e += 32) {
                    const int q = e % 9;
                    dst[e] = double(acc[e * 32 + (l ^ q)]);
                }
            }
        }
        __syncwarp();
    }
}

}  // namespace

int launch_assemble_jacobian_list(plato_problem* h, const double* z, double* entries, const int32_t* rows,
                                  int32_t count, const uint8_t* wide);

// Builds the assembly plan, the mirror slots and the wide-row list once per mesh.
int assembly_plan(plato_problem* h) {
    if (h->asm_plan) return PLATO_OK;
    cudaStream_t s = h->stream;
    const int64_t ninc = 4 * (int64_t)h->C;
    PLATO_CUDA(h, cudaMalloc(&h->asm_plan, sizeof(uint16_t) * (ninc > 0 ? ninc : 1)));
    PLATO_CUDA(h, cudaMalloc(&h->asm_mirror, sizeof(uint8_t) * (h->nblocks > 0 ? h->nblocks : 1)));
    PLATO_CUDA(h, cudaMalloc(&h->asm_wideflag, sizeof(uint8_t) * (h->N > 0 ? h->N : 1)));
    PLATO_CUDA(h, cudaMalloc(&h->asm_wide, sizeof(int32_t) * (h->N + 2)));
    PLATO_CUDA(h, cudaMemsetAsync(h->asm_wide + h->N, 0, 2 * sizeof(int32_t), s));
    k_asm_flags<<<grid_for(h->N, 128), 128, 0, s>>>(graph_view(h), h->asm_wideflag, h->asm_wide, h->asm_wide + h->N,
                                                    h->asm_wide + h->N + 1);
    PLATO_LAUNCH_CHECK(h);
    k_asm_plan<<<grid_for(h->N, 128), 128, 0, s>>>(graph_view(h), h->conn, h->asm_wideflag, h->asm_plan,
                                                   h->asm_mirror);
    PLATO_LAUNCH_CHECK(h);
    int32_t counts[2] = {0, 0};
    PLATO_CUDA(h, cudaMemcpyAsync(counts, h->asm_wide + h->N, sizeof(counts), cudaMemcpyDeviceToHost, s));
    PLATO_CUDA(h, cudaStreamSynchronize(s));
    h->asm_nwide = counts[0];
    h->asm_maxup = counts[1] > 0 ? counts[1] : 1;
    return PLATO_OK;
}

// One CTA per SM with as many warps as the accumulators of `up` upper blocks let fit.
static int asm_launch(plato_problem* h, const void* kernel, size_t elem, int* grid, int* threads, int* smem) {
    const int per_warp = int(9 * 32 * h->asm_maxup * elem);
    const int warps = std::min(kAsmMaxWarps, kAsmSmemMax / per_warp);
    *threads = 32 * warps;
    *smem = warps * per_warp;
    PLATO_RC(ensure_smem_attribute(h, kernel, *smem));
    int sms = 0;
    PLATO_CUDA(h, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
    const int64_t nslices = (int64_t(h->N) + 31) / 32;
    *grid = int(std::min<int64_t>(sms, (nslices + warps - 1) / warps));
    if (*grid < 1) *grid = 1;
    return PLATO_OK;
}

// K(z) into the block CRS `entries` (unconstrained): narrow rows here, wide rows (and the
// transposes of their upper blocks) by the warp-per-row kernel.
int launch_assemble_jacobian(plato_problem* h, const double* z, double* entries) {
    PLATO_RC(assembly_plan(h));
    int grid = 0, threads = 0, smem = 0;
    PLATO_RC(asm_launch(h, reinterpret_cast<const void*>(k_assemble_rows<false, double>), sizeof(double), &grid,
                        &threads, &smem));
    k_assemble_rows<false, double><<<grid, threads, smem, h->stream>>>(mesh_view(h), graph_view(h), h->material, z,
                                                                      h->asm_plan, h->asm_mirror, h->asm_wideflag,
                                                                      h->asm_maxup, entries, SellOut{});
    PLATO_LAUNCH_CHECK(h);
    if (h->asm_nwide > 0)
        PLATO_RC(launch_assemble_jacobian_list(h, z, entries, h->asm_wide, h->asm_nwide, h->asm_wideflag));
    return PLATO_OK;
}

// Whether the solver's constrained SELL copy can be assembled directly: every row narrow and
// homogeneous essential BCs (inhomogeneous values need the unconstrained columns to lift the
// right-hand side, which the CRS path does).
int assembly_direct_sell_ok(plato_problem* h, int* ok) {
    PLATO_RC(assembly_plan(h));
    *ok = (h->asm_nwide == 0 && !h->bc_nonzero) ? 1 : 0;
    return PLATO_OK;
}

// Constrained SELL copy of K(z) + inverse diagonal (+ FP32 / BF16 copies when given).
int launch_assemble_sell(plato_problem* h, const double* z, double* v64, float* v32, void* v16, double* dinv,
                         float* dinv32) {
    PLATO_RC(assembly_plan(h));
    if (h->asm_nwide > 0) return plato_fail(h, PLATO_NOT_SUPPORTED, "direct SELL assembly needs every row narrow");
    int grid = 0, threads = 0, smem = 0;
    PLATO_RC(asm_launch(h, reinterpret_cast<const void*>(k_assemble_rows<true, double>), sizeof(double), &grid,
                        &threads, &smem));
    SellOut so{h->sell.ptr, h->sell.cols, h->bc_mask, v64, v32, static_cast<__nv_bfloat16*>(v16), dinv, dinv32};
    // the solver's assembly timing (instrumentation) brackets this one kernel
    if (h->timing && h->asm_ev[0]) PLATO_CUDA(h, cudaEventRecord(h->asm_ev[0], h->stream));
    k_assemble_rows<true, double><<<grid, threads, smem, h->stream>>>(mesh_view(h), graph_view(h), h->material, z,
                                                                     h->asm_plan, h->asm_mirror, h->asm_wideflag,
                                                                     h->asm_maxup, nullptr, so);
    PLATO_LAUNCH_CHECK(h);
    if (h->timing && h->asm_ev[1]) PLATO_CUDA(h, cudaEventRecord(h->asm_ev[1], h->stream));
    return PLATO_OK;
}

// FP32 element assembly of the constrained SELL copy (values and inverse diagonal in FP32),
// the preconditioner matrix when the FP64 outer operator is the matrix-free element apply.
int launch_assemble_sell32(plato_problem* h, const double* z, float* v32, float* dinv32) {
    PLATO_RC(assembly_plan(h));
    if (h->asm_nwide > 0) return plato_fail(h, PLATO_NOT_SUPPORTED, "FP32 element assembly needs every row narrow");
    if (h->bc_nonzero) return plato_fail(h, PLATO_NOT_SUPPORTED, "FP32 element assembly needs homogeneous essential BCs");
    int grid = 0, threads = 0, smem = 0;
    PLATO_RC(asm_launch(h, reinterpret_cast<const void*>(k_assemble_rows<true, float>), sizeof(float), &grid,
                        &threads, &smem));
    SellOut so{h->sell.ptr, h->sell.cols, h->bc_mask, nullptr, v32, nullptr, nullptr, dinv32};
    k_assemble_rows<true, float><<<grid, threads, smem, h->stream>>>(mesh_view(h), graph_view(h), h->material, z,
                                                                    h->asm_plan, h->asm_mirror, h->asm_wideflag,
                                                                    h->asm_maxup, nullptr, so);
    PLATO_LAUNCH_CHECK(h);
    return PLATO_OK;
}

}  // namespace plato
