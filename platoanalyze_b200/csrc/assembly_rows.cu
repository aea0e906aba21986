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
// densities, forms the gradients with the row node as the reference vertex, and adds
// w g_a g_b^T into the slot of each other node b.  The slot of each (row, cell, b) is looked
// up once per mesh (the assembly plan: three 4-bit slot numbers per incidence entry), so the
// hot loop has no search and no inter-thread reduction.  The diagonal block, which every
// incident cell feeds, is accumulated in registers (6 symmetric components); the other
// slots accumulate in shared memory, 9 doubles per slot per thread.  A warp owns the 32 rows
// of one SELL slice and the layout of its accumulator is [slot][component][lane ^ component]:
// in the accumulation every lane touches the same component at a time, so the 64-bit
// accesses of a half warp hit 16 distinct bank pairs; in the row-major write-out (CRS) 16
// consecutive entries of one row span at most 9 components, two to a bank pair.
//
// Rows with more than kAsmSlots blocks (high-valence nodes of general meshes) are skipped
// here and assembled by the warp-per-row kernel of assembly.cu.
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

constexpr int kAsmWarps = 6;                        // warps per CTA, one CTA per SM
constexpr int kAsmSlots = 15;                       // blocks per row held in shared memory
constexpr int kAccPerWarp = 9 * kAsmSlots * 32;     // doubles
constexpr size_t kAsmSmem = size_t(kAsmWarps) * kAccPerWarp * sizeof(double);  // 207,360 B

__device__ __forceinline__ int acc_index(int k, int q, int lane) { return (9 * k + q) * 32 + (lane ^ q); }

__device__ __forceinline__ int warp_max(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
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

// Per mesh: for every (row, incident cell) entry of n2c, the slots of the cell's three other
// nodes (ascending local ordinal) in the row, 4 bits each.  Rows with more than kAsmSlots
// blocks get no plan and are appended to the wide-row list.
__global__ void k_asm_plan(GraphView g, const int4* __restrict__ conn, uint16_t* __restrict__ plan,
                           int32_t* __restrict__ wide, int32_t* __restrict__ nwide) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < g.num_nodes;
         r += (int64_t)gridDim.x * blockDim.x) {
        const int32_t rs = g.row_map[r], nb = g.row_map[r + 1] - rs;
        if (nb > kAsmSlots) {
            wide[atomicAdd(nwide, 1)] = int32_t(r);
            continue;
        }
        for (int32_t k = g.n2c_ptr[r]; k < g.n2c_ptr[r + 1]; ++k) {
            const int32_t packed = g.n2c[k];
            const int la = packed & 3;
            const int4 n = conn[packed >> 2];
            uint32_t code = 0;
            int t = 0;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                if (b == la) continue;
                const int32_t node = node_of(n, b);
                int lo = 0, hi = nb - 1;
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (g.cols[rs + mid] < node) lo = mid + 1; else hi = mid;
                }
                code |= uint32_t(lo) << (4 * t);
                ++t;
            }
            plan[k] = uint16_t(code);
        }
    }
}

// T = double, kSell = false: block CRS values (unconstrained) into crs[9 * nblocks].
// T = double, kSell = true:  constrained SELL copy + inverse diagonal (+ optional FP32 / BF16
//                            copies rounded from the FP64 values) into `so`.
// T = float,  kSell = true:  FP32 element assembly -- gradients, weights and sums in FP32 -- of
//                            the constrained SELL copy (so.v32) and its inverse diagonal
//                            (so.dinv32), the preconditioner matrix of the mixed-precision solve
//                            whose FP64 outer operator is the matrix-free element apply.
// Shared memory is the same 207,360 bytes per CTA: 6 warps of FP64 or 12 warps of FP32 sums.
template <bool kSell, typename T>
__global__ void __launch_bounds__(kAsmWarps * 32 * (sizeof(T) == 8 ? 1 : 2), 1)
k_assemble_rows(MeshView m, GraphView g, Material mat, const double* __restrict__ z,
                const uint16_t* __restrict__ plan, double* __restrict__ crs, SellOut so) {
    constexpr int kWarps = kAsmWarps * (sizeof(T) == 8 ? 1 : 2);
    extern __shared__ double smem_raw[];
    T* smem = reinterpret_cast<T*>(smem_raw);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    T* acc = smem + warp * kAccPerWarp;
    const T lam = T(mat.c01), mu = T(mat.c33);
    const int32_t nslices = (g.num_nodes + 31) >> 5;
    for (int32_t s = blockIdx.x * kWarps + warp; s < nslices; s += gridDim.x * kWarps) {
        const int32_t r = 32 * s + lane;
        int32_t rs = 0, nb = 0, ks = 0, kc = 0, dslot = -1;
        T xr[3] = {T(0), T(0), T(0)}, zr = T(0);
        if (r < g.num_nodes) {
            rs = g.row_map[r];
            nb = g.row_map[r + 1] - rs;
            if (nb <= kAsmSlots) {
                ks = g.n2c_ptr[r];
                kc = g.n2c_ptr[r + 1] - ks;
                dslot = g.diag[r] - rs;
                xr[0] = T(__ldg(m.coords + 3 * (int64_t)r));
                xr[1] = T(__ldg(m.coords + 3 * (int64_t)r + 1));
                xr[2] = T(__ldg(m.coords + 3 * (int64_t)r + 2));
                zr = mat.cell_control ? T(0) : T(__ldg(z + r));
            } else {
                nb = 0;  // wide row: assembled by the warp-per-row kernel
            }
        }
        const int nbw = warp_max(nb);
        for (int k = 0; k < nbw; ++k)
#pragma unroll
            for (int q = 0; q < 9; ++q) acc[acc_index(k, q, lane)] = T(0);
        __syncwarp();

        T d0 = T(0), d1 = T(0), d2 = T(0), d3 = T(0), d4 = T(0), d5 = T(0);  // xx yy zz yz xz xy
        const int kmax = warp_max(kc);
        // one cell ahead: incidence entry, plan and connectivity of the next cell
        int32_t p_next = 0;
        uint32_t pl_next = 0;
        int4 n_next = make_int4(0, 0, 0, 0);
        if (kc > 0) {
            p_next = __ldg(g.n2c + ks);
            pl_next = __ldg(plan + ks);
            n_next = __ldg(m.conn + (p_next >> 2));
        }
#pragma unroll 1
        for (int j = 0; j < kmax; ++j) {
            const int32_t p = p_next;
            const uint32_t pl = pl_next;
            const int4 n = n_next;
            if (j + 1 < kc) {
                p_next = __ldg(g.n2c + ks + j + 1);
                pl_next = __ldg(plan + ks + j + 1);
                n_next = __ldg(m.conn + (p_next >> 2));
            }
            if (j < kc) {
                // the three other nodes in ascending local order; the row node is vertex 3
                const int la = p & 3;
                const int32_t i0 = la == 0 ? n.y : n.x;
                const int32_t i1 = la <= 1 ? n.z : n.y;
                const int32_t i2 = la <= 2 ? n.w : n.z;
                const double* c0 = m.coords + 3 * (int64_t)i0;
                const double* c1 = m.coords + 3 * (int64_t)i1;
                const double* c2 = m.coords + 3 * (int64_t)i2;
                const T j11 = T(__ldg(c0)) - xr[0], j21 = T(__ldg(c0 + 1)) - xr[1], j31 = T(__ldg(c0 + 2)) - xr[2];
                const T j12 = T(__ldg(c1)) - xr[0], j22 = T(__ldg(c1 + 1)) - xr[1], j32 = T(__ldg(c1 + 2)) - xr[2];
                const T j13 = T(__ldg(c2)) - xr[0], j23 = T(__ldg(c2 + 1)) - xr[1], j33 = T(__ldg(c2 + 2)) - xr[2];
                const T rho = mat.cell_control ? T(__ldg(z + (p >> 2)))
                                               : (T(__ldg(z + i0)) + T(__ldg(z + i1)) + T(__ldg(z + i2)) + zr) * T(0.25);
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
                    const int k = (pl >> (4 * t)) & 15;
                    T* row = acc + 9 * 32 * k;
#pragma unroll
                    for (int q = 0; q < 9; ++q) {
                        const T ai = q < 3 ? a0 : (q < 6 ? a1 : a2);
                        T& v = row[q * 32 + (lane ^ q)];
                        v = fma(ai, gb[t][q % 3], v);
                    }
                }
            }
        }
        __syncwarp();

        // K = lambda S + mu S^T + mu tr(S) I per slot; nbw is also the SELL slice width
        const int64_t pbase = kSell ? __ldg(so.ptr + s) : 0;  // first SELL slot of the slice
        const int64_t sbase = 9 * pbase;
        for (int k = 0; k < nbw; ++k) {
            T S[9];
            if (k == dslot) {
                S[0] = d0; S[4] = d1; S[8] = d2;
                S[5] = S[7] = d3;
                S[2] = S[6] = d4;
                S[1] = S[3] = d5;
            } else {
#pragma unroll
                for (int q = 0; q < 9; ++q) S[q] = acc[acc_index(k, q, lane)];
            }
            const T tr = mu * (S[0] + S[4] + S[8]);
            T K[9];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int jj = 0; jj < 3; ++jj)
                    K[3 * i + jj] = lam * S[3 * i + jj] + mu * S[3 * jj + i] + (i == jj ? tr : T(0));
            if (!kSell) {
#pragma unroll
                for (int q = 0; q < 9; ++q) acc[acc_index(k, q, lane)] = K[q];
            } else {
                const bool real = k < nb;
                const int32_t c = __ldg(so.cols + pbase + 32 * k + lane);  // column node of the slot
#pragma unroll
                for (int q = 0; q < 9; ++q) {
                    const int i = q / 3, jj = q % 3;
                    T v = real ? K[q] : T(0);
                    if (real) {
                        const bool mr = __ldg(so.bc_mask + 3 * (int64_t)r + i) != 0;
                        const bool mc = __ldg(so.bc_mask + 3 * (int64_t)c + jj) != 0;
                        if (mr || mc) v = (c == r && i == jj) ? T(1) : T(0);
                    }
                    const int64_t o = sbase + 32 * (9 * k + q) + lane;
                    if (sizeof(T) == 8) so.v64[o] = double(v);
                    if (so.v32) so.v32[o] = float(v);
                    if (so.v16) so.v16[o] = __float2bfloat16_rn(float(v));
                    if (real && k == dslot && i == jj) {
                        if (sizeof(T) == 8) so.dinv[3 * (int64_t)r + i] = 1.0 / double(v);
                        if (so.dinv32) so.dinv32[3 * (int64_t)r + i] = float(1.0 / double(v));
                    }
                }
            }
        }
        if (!kSell) {
            __syncwarp();
            // row-major write-out: the warp writes each row of the slice as one contiguous run
            for (int l = 0; l < 32; ++l) {
                const int32_t rs_l = __shfl_sync(0xffffffffu, rs, l);
                const int nv = 9 * __shfl_sync(0xffffffffu, nb, l);
                double* dst = crs + 9 * (int64_t)rs_l;
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

int launch_assemble_jacobian_rows(plato_problem* h, const double* z, double* entries, int32_t* nwide_out);
int launch_assemble_jacobian_list(plato_problem* h, const double* z, double* entries, const int32_t* rows,
                                  int32_t count);

// Builds the assembly plan and the wide-row list once per mesh.
int assembly_plan(plato_problem* h) {
    if (h->asm_plan) return PLATO_OK;
    cudaStream_t s = h->stream;
    const int64_t ninc = 4 * (int64_t)h->C;
    PLATO_CUDA(h, cudaMalloc(&h->asm_plan, sizeof(uint16_t) * (ninc > 0 ? ninc : 1)));
    PLATO_CUDA(h, cudaMalloc(&h->asm_wide, sizeof(int32_t) * (h->N + 1)));
    PLATO_CUDA(h, cudaMemsetAsync(h->asm_wide + h->N, 0, sizeof(int32_t), s));
    k_asm_plan<<<grid_for(h->N, 128), 128, 0, s>>>(graph_view(h), h->conn, h->asm_plan, h->asm_wide,
                                                   h->asm_wide + h->N);
    PLATO_LAUNCH_CHECK(h);
    PLATO_CUDA(h, cudaMemcpyAsync(&h->asm_nwide, h->asm_wide + h->N, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    PLATO_CUDA(h, cudaStreamSynchronize(s));
    return PLATO_OK;
}

static int asm_grid(plato_problem* h, const void* kernel, int* grid, int warps = kAsmWarps) {
    PLATO_RC(ensure_smem_attribute(h, kernel, int(kAsmSmem)));
    int sms = 0;
    PLATO_CUDA(h, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
    const int64_t nslices = (int64_t(h->N) + 31) / 32;
    *grid = int(std::min<int64_t>(sms, (nslices + warps - 1) / warps));
    if (*grid < 1) *grid = 1;
    return PLATO_OK;
}

// K(z) into the block CRS `entries` (unconstrained): narrow rows here, wide rows by the
// warp-per-row kernel.
int launch_assemble_jacobian(plato_problem* h, const double* z, double* entries) {
    PLATO_RC(assembly_plan(h));
    int grid = 0;
    PLATO_RC(asm_grid(h, reinterpret_cast<const void*>(k_assemble_rows<false, double>), &grid));
    k_assemble_rows<false, double><<<grid, kAsmWarps * 32, kAsmSmem, h->stream>>>(mesh_view(h), graph_view(h), h->material,
                                                                           z, h->asm_plan, entries, SellOut{});
    PLATO_LAUNCH_CHECK(h);
    if (h->asm_nwide > 0) PLATO_RC(launch_assemble_jacobian_list(h, z, entries, h->asm_wide, h->asm_nwide));
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
    int grid = 0;
    PLATO_RC(asm_grid(h, reinterpret_cast<const void*>(k_assemble_rows<true, double>), &grid));
    SellOut so{h->sell.ptr, h->sell.cols, h->bc_mask, v64, v32, static_cast<__nv_bfloat16*>(v16), dinv, dinv32};
    // the solver's assembly timing (instrumentation) brackets this one kernel
    if (h->timing && h->asm_ev[0]) PLATO_CUDA(h, cudaEventRecord(h->asm_ev[0], h->stream));
    k_assemble_rows<true, double><<<grid, kAsmWarps * 32, kAsmSmem, h->stream>>>(mesh_view(h), graph_view(h), h->material,
                                                                          z, h->asm_plan, nullptr, so);
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
    int grid = 0;
    PLATO_RC(asm_grid(h, reinterpret_cast<const void*>(k_assemble_rows<true, float>), &grid, 2 * kAsmWarps));
    SellOut so{h->sell.ptr, h->sell.cols, h->bc_mask, nullptr, v32, nullptr, nullptr, dinv32};
    k_assemble_rows<true, float><<<grid, 2 * kAsmWarps * 32, kAsmSmem, h->stream>>>(
        mesh_view(h), graph_view(h), h->material, z, h->asm_plan, nullptr, so);
    PLATO_LAUNCH_CHECK(h);
    return PLATO_OK;
}

}  // namespace plato
