// Internal declarations of the B200 elliptic path: the handle, error plumbing and the
// device-side element arithmetic shared by every kernel.
#pragma once

#include <cmath>

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "plato_b200.h"
#include "sell.cuh"

namespace plato {

// ---------------------------------------------------------------------------------------
// Material constants of IsotropicLinearElasticMaterial<3>
// (src/IsotropicLinearElasticMaterial.cpp:86-110): C00 = c(1-nu), C01 = c nu,
// C33 = 1/2 c (1-2nu), c = E/((1+nu)(1-2nu)).  Lame form: lambda = C01, mu = C33.
struct Material {
    double c00, c01, c33;
    double p, rho_min;  // MSIMP exponent and minimum value (src/Simp.hpp:130-134)
    int    p_int;       // p when it is a small non-negative integer, else -1
    int    cell_control;  // 0: nodal control, cell density = mean of its 4 nodes
                          // (ApplyWeighting, src/ApplyWeighting.hpp:55-60); 1: one density per cell
};

// Device pointers and sizes the element kernels read.
struct MeshView {
    int32_t       num_nodes;
    int32_t       num_cells;
    const int4*   conn;    // [num_cells]   the 4 node ids of each cell
    const double* coords;  // [3*num_nodes] node-major xyz
};

// Node graph: block pattern plus the node -> (cell, local slot) incidence.
struct GraphView {
    int32_t        num_nodes;
    int64_t        num_blocks;
    const int32_t* row_map;   // [N+1]
    const int32_t* cols;      // [num_blocks]
    const int32_t* diag;      // [N] position of the diagonal block of each row
    const int32_t* n2c_ptr;   // [N+1]
    const int32_t* n2c;       // [4*C] cell*4 + local slot, sorted by cell within a node
};

}  // namespace plato

// Work state of the Jacobi-PCG (device resident).
struct PcgScalars {
    double rz;       // r . z
    double rz_new;
    double pAp;
    double rr;       // r . r
    double bb;       // b . b
    double alpha;
    double beta;
    double tol2;     // tol^2 * b.b
    double zq;       // flexible CG: z_(k+1) . A p_k
    int32_t iter;
    int32_t done;    // 1 once ||r|| <= tol ||b||
    int32_t nonfinite;
    uint32_t ticket; // last-block-done counter of the fused reductions
};

// Size of the next chunk of Krylov iterations the host enqueues while the previous one runs.
// Every iteration enqueued after convergence still launches its kernels (they return at
// once), so near the end the chunks shrink to what the observed residual decay predicts:
// polled state s (its iteration count and r.r), `in_flight` iterations already queued
// behind it; the first poll measures the decay from b.b (the start from x0 = 0; a better
// initial guess only makes the estimate conservative).  Irregular decay keeps the full chunk.
struct ChunkPlanner {
    int32_t full = 16;
    int32_t last_iter = -1;
    double  last_rr = 0.0;
    int32_t next(const PcgScalars& st, int32_t in_flight) {
        int32_t size = full;
        if (last_iter < 0) {  // first poll: measure the decay from the start, r.r = b.b for x0 = 0
            last_iter = 0;
            last_rr = st.bb;
        }
        if (st.iter > last_iter && st.rr > 0.0 && last_rr > 0.0 && st.tol2 > 0.0) {
            const double rate = std::pow(st.rr / last_rr, 1.0 / double(st.iter - last_iter));
            if (rate > 0.0 && rate < 0.999) {
                const double left = std::log(st.tol2 / st.rr) / std::log(rate);  // iterations still needed
                const double after = left - double(in_flight);
                if (after <= 0.0) size = 2;
                else if (after + 2.0 < double(full)) size = int32_t(after) + 2;
            }
        }
        last_iter = st.iter;
        last_rr = st.rr;
        return size;
    }
};

// Per-problem Krylov state of a batched solve (one entry per member problem).
struct SegScalars {
    double pr;       // p . r
    double pq;       // p . A p
    double alpha;
    double beta;
    double zq;       // z . A p
    double rr;       // r . r
    double bb;       // b . b
    double tol2;     // tol^2 * b.b
    int32_t iter;
    int32_t done;
    int32_t nonfinite;
    uint32_t ticket; // last-CTA-done counter of the member's reductions
};

// Batch of independent problems stored as one disjoint-union mesh (batch.cu).  Member s owns
// node rows [node_off[s], node_off[s+1]) and cells [cell_off[s], cell_off[s+1]); the
// segmented solver kernels run one CTA per tile of at most 256 rows of one member.
struct BatchState {
    int32_t  nseg = 0;                 // 0 for a single problem
    std::vector<int32_t> node_off, cell_off;
    int32_t  ncta = 0;                 // tiles of at most tile_rows rows, never across two members
    int32_t  tile_rows = 256;          // rows per tile = threads per CTA of the batched kernels
    int32_t  ctas_per_sm = 8;          // persistent grid of the batched kernels
    int32_t  tuned = 0;                // the pair above comes from plato_batch_autotune
    int32_t* cta_seg = nullptr;        // [ncta] member of each tile
    int32_t* cta_row0 = nullptr;       // [ncta] first row of each tile
    int32_t* cta_row1 = nullptr;       // [ncta] one past its last row
    int32_t* seg_cta0 = nullptr;       // [nseg+1] first tile of each member
    int32_t* cell_off_d = nullptr;     // [nseg+1] on the device
    SegScalars* S = nullptr;           // [nseg] device
    SegScalars* S_host = nullptr;      // [nseg] pinned
    int32_t* ndone = nullptr;          // members done (device)
    double*  partials = nullptr;       // [2*ncta]
    double*  values = nullptr;         // [nseg * kEnergySplit] criterion partial sums
    std::vector<plato_solve_stats> last;  // per-member statistics of the last solve
};

// Two-level preconditioner state (coarse.cu).
struct CoarseSpace {
    int      nc[3] = {0, 0, 0};   // coarse cells per axis
    int      ready = 0;           // mesh-level setup done for nc
    int      active = 0;          // operator built for the current solve
    double   x0[3] = {0, 0, 0};   // grid origin (mesh bounding-box minimum)
    double   h[3] = {0, 0, 0};    // coarse cell size
    int32_t  ncells = 0, nnodes = 0, ndof = 0;
    int32_t* node_ptr = nullptr;  // fine nodes bucketed by coarse cell (CSR)
    int32_t* node_list = nullptr;
    int32_t* elem_ptr = nullptr;  // elements bucketed by coarse cell (CSR)
    int32_t* elem_list = nullptr;
    double*  E = nullptr;         // Galerkin operator, then its Cholesky factor (ndof^2)
    float*   Xf = nullptr;        // L^-1 (lower) then its transpose U (upper), FP32, row stride ldf:
    float*   Uf = nullptr;        // E^-1 = U L^-1, the per-iteration coarse solve (zeros elsewhere)
    int32_t  ldf = 0;             // ndof rounded up to a multiple of 4 (16-byte rows)
    int32_t  band = 0;            // E[i][j] == 0 for |i - j| > band (structural, x-major node order)
    int32_t  tband = 0;           // the same in 64 x 64 tiles: tile (ti, tj) == 0 for ti - tj > tband
    double*  X = nullptr;         // L^-1 while inverting (ndof^2)
    double*  T = nullptr;         // tile-product scratch of the inversion (ndof^2)
    double*  Dt = nullptr;        // inverse diagonal tiles of the Cholesky factor
    int32_t  rsplit = 1, gsplit = 1;  // CTAs per coarse cell in the restriction / Galerkin sum
    double*  rpart = nullptr;     // restriction partial sums (ncells * rsplit * 24)
    double*  rc = nullptr;        // restricted residual
    double*  yc = nullptr;        // coarse correction
    double*  tc = nullptr;        // L^-1 rc
    int32_t* flag = nullptr;
    cudaStream_t side = nullptr;  // trailing Cholesky updates, overlapped with the next panel
    cudaGraphExec_t chain = nullptr;  // the captured factorization + inversion chain
    int          chain_launches = 0;
    cudaEvent_t  ev_panel = nullptr, ev_trail = nullptr;
    // the per-solve set-up runs on a stream of its own, overlapped with the fine-level set-up
    // (assembly, SELL copies, spectrum estimate) on the handle's stream
    cudaStream_t cs = nullptr;
    cudaEvent_t  ev_start = nullptr, ev_ready = nullptr;
    int          start_marked = 0;    // ev_start already recorded for the next set-up
    int32_t*     flag_host = nullptr; // pinned copy of flag (factorization failure)
    int          pending = 0;         // a set-up is in flight: wait for ev_ready before use
};

struct plato_problem {
    int          device = 0;
    cudaStream_t stream = nullptr;
    std::string  last_error;

    int32_t N = 0, C = 0;
    int64_t nblocks = 0;

    plato::Material material{};
    plato_solver_opts opts{};

    // mesh
    int4*   conn = nullptr;
    double* coords = nullptr;
    // graph
    int32_t* row_map = nullptr;
    int32_t* cols = nullptr;
    int32_t* diag = nullptr;
    int32_t* n2c_ptr = nullptr;
    int32_t* n2c = nullptr;
    // loads and BCs
    double*  F = nullptr;          // external load vector (traction), length 3N
    int32_t  nbc = 0;
    int32_t* bc_dofs = nullptr;
    double*  bc_values = nullptr;
    uint8_t* bc_mask = nullptr;    // [3N] 1 where a dof is constrained
    int      bc_nonzero = 0;       // some essential BC value is nonzero
    double   bbox_min[3] = {0, 0, 0};
    double   bbox_max[3] = {0, 0, 0};
    CoarseSpace coarse{};
    // thread-per-row assembly plan (assembly_rows.cu, once per mesh): three 4-bit slots per
    // n2c entry, and the rows with too many blocks for it
    uint16_t* asm_plan = nullptr;
    uint8_t*  asm_mirror = nullptr;   // [nblocks]: slot of the row in each upper neighbour's row
    uint8_t*  asm_wideflag = nullptr; // [N]: rows assembled by the warp-per-row kernel
    int32_t*  asm_wide = nullptr;  // [N + 2]: wide rows, then their count at [N], max upper blocks at [N+1]
    int32_t   asm_nwide = 0;
    int32_t   asm_maxup = 1;       // upper blocks of the widest narrow row
    // assembled operator (allocated on first use)
    double* K = nullptr;           // 9*nblocks
    double* KT = nullptr;          // scratch for transposed / gradient_z matrices
    // PCG work vectors (3N each) and scalars
    double* v_r = nullptr;
    double* v_z = nullptr;
    double* v_p = nullptr;
    double* v_Ap = nullptr;
    double* v_dinv = nullptr;
    double* v_b = nullptr;
    double* v_x = nullptr;
    double* v_tmp = nullptr;
    double* partials = nullptr;    // block partial sums of reductions
    double* cellbuf = nullptr;     // one double per cell (per-cell quantities before a nodal sum)
    int32_t partials_len = 0;
    PcgScalars* scal = nullptr;    // device
    PcgScalars* scal_host = nullptr;  // pinned mirror
    double* red_out = nullptr;     // device scalar result of a reduction
    uint32_t* red_ticket = nullptr;
    // mixed-precision and matrix-free work (allocated on first use)
    float* f_r = nullptr;
    float* f_z = nullptr;
    float* f_p = nullptr;
    float* f_Ap = nullptr;
    float* f_x = nullptr;
    float* f_dinv = nullptr;
    float* f_K = nullptr;          // 9*nblocks FP32 copy of the constrained matrix
    uint16_t* h_K = nullptr;       // 9*nblocks BF16 copy
    float* f_coords = nullptr;
    float* f_z_ctrl = nullptr;     // nodal control in FP32 (matrix-free FP32 apply)
    double* d_z_ctrl = nullptr;    // nodal control the operator was built for
    int     operator_ready = 0;    // K / diag valid for d_z_ctrl
    // host staging for the _host entry points
    double* pinned = nullptr;
    size_t  pinned_len = 0;
    // device scratch for host-buffer calls
    double* d_z_in = nullptr;
    double* d_u_out = nullptr;
    double* d_g_out = nullptr;
    // solver-private SELL-32 copy of the constrained operator (sell.cu)
    plato::SellPattern sell{};
    double* sell64 = nullptr;      // FP64 entries
    float*  sell32 = nullptr;      // FP32 entries (mixed precision)
    void*   sell16 = nullptr;      // BF16 entries (mixed precision)
    void*   sell16s = nullptr;     // FP16 entries of D^-1/2 A D^-1/2 (scaled mixed precision)
    float*  f_sq = nullptr;        // D^1/2 (scaled mixed precision)
    float*  f_isq = nullptr;       // D^-1/2
    // matrix-free operator data (matfree.cu) and mixed-precision work vectors (mixed.cu)
    double* mf_w64 = nullptr;      // per-cell SIMP weight s(rho_e), FP64
    float*  mf_w32 = nullptr;      // same, FP32
    double* v_q = nullptr;         // A p of the flexible CG
    float*  f_res = nullptr;       // Chebyshev residual
    float*  f_d0 = nullptr;        // Chebyshev directions (double buffered)
    float*  f_d1 = nullptr;
    float*  f_y = nullptr;         // preconditioner output
    float*  f_w = nullptr;         // inner operator output
    // multi-step FP16 sweep (k_sell16s_wave in mixed.cu): completion stamps of (step, tile),
    // ticket counters, and the task order for each launch length
    int32_t* wave_flags = nullptr; // [16][wave_tiles] epoch of the last completion
    int32_t* wave_ctl = nullptr;   // ticket, exits, abort, fail
    double* lanczos = nullptr;     // Lanczos coefficients of the Chebyshev interval estimate
    int32_t* wave_order[17] = {};  // per steps-per-launch: task codes (step << 24 | tile)
    int32_t  wave_order_lag[17] = {};
    int32_t  wave_tiles = 0;
    int32_t  wave_halo = -1;       // column reach in tiles (-1: not measured, -2: disabled)
    int32_t  wave_epoch = 0;
    int32_t  sweep_steps_used = 0; // steps per launch of the last flexible-CG solve's sweep
    int32_t  wave_stall = 0;       // test hook: the next launch waits for a stamp nobody writes
    // instrumentation: kernel launches issued, and sampled CUDA-event timings of the
    // solver's operator apply (every kTimingStride-th apply, events on the handle's stream)
    int64_t launches = 0;
    int     timing = 0;
    cudaEvent_t poll_ev[2] = {nullptr, nullptr};  // host polling of the solver scalars (made once)
    std::vector<cudaEvent_t> ev_pool;
    int     ev_used = 0;
    double  op_ms_total = 0.0;
    int64_t op_timed = 0;
    double  inner_ms_total = 0.0;  // preconditioner operator step (mixed-precision solver)
    int64_t inner_timed = 0;       // steps timed
    int32_t inner_record_steps = 1;  // steps in one timed preconditioner launch
    cudaEvent_t asm_ev[2] = {nullptr, nullptr};  // Jacobian assembly of the solve path
    double  asm_ms_total = 0.0;
    int64_t asm_timed = 0;
    cudaEvent_t coarse_ev[3] = {nullptr, nullptr, nullptr};  // coarse operator: Galerkin | dense inverse
    double  coarse_gal_ms = 0.0;
    double  coarse_inv_ms = 0.0;
    int64_t coarse_timed = 0;
    // element kernels timed as one unit per call (kinds 5-8 of plato_get_kernel_timing): the
    // residual (k_internal_force), the energy sum, the control derivative (per-cell pass +
    // nodal sum) and the fused value + derivative; a pair is read when the same kind is timed
    // again or the totals are read
    struct TimedPair {
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        int pending = 0;
        double ms = 0.0;
        int64_t count = 0;
    } elem_timing[4];
    BatchState batch{};
    // subspace initial guess (ritz.cu): columns set for the duration of one solution call
    const double* ritz_W = nullptr;
    int32_t ritz_k = 0;
    double* ritz_scratch = nullptr;
    size_t  ritz_scratch_len = 0;
    double  ritz_rel_gain = 1.0;   // ||r|| after / before the last subspace correction (1: not used)
    int32_t ritz_deflate = 0;      // the subspace also deflates the Krylov directions (this call)
    int32_t ritz_deflating = 0;    // deflation set up for the running solve (Galerkin guess kept)
    double* ritz_small = nullptr;  // G^-1 (k x k) and mu (k) of the deflation
    // Helmholtz density filter (helmholtz.cu): physics 1, one unknown per node
    int32_t physics = 0;           // 0 elastostatics, 1 Helmholtz filter
    double  helm_length = 0.0;     // length scale L
    int32_t helm_ready = 0;        // K, its SELL copy and diagonal built
    double* helm_K = nullptr;      // one value per block of the node pattern
    double* helm_sell = nullptr;   // SELL copy (one value per slot)
    double* helm_D = nullptr;      // (dR/dcontrol)^T = -M, one value per block
    double* helm_Dsell = nullptr;  // its SELL copy
    double* helm_dinv = nullptr;   // inverse diagonal
    double  helm_surface = 0.0;    // surface length scale alpha (0: no surface term)
    int32_t helm_nfaces = 0;       // faces carrying the surface term
    int32_t* helm_fcell = nullptr; // their owning cells
    int32_t* helm_floc = nullptr;  // 3 cell-local node ordinals per face
};

// ---------------------------------------------------------------------------------------
// error plumbing
int plato_fail(plato_problem* h, int status, const std::string& msg);
namespace plato {
int coarse_setup_mesh(plato_problem* h);
int coarse_setup_operator(plato_problem* h, const double* z, double* E_copy = nullptr, int deferred = 0);
int coarse_mark_start(plato_problem* h);  // ev_start: where the next set-up may begin
int coarse_wait(plato_problem* h);    // the handle's stream waits for the set-up (no host wait)
int coarse_finish(plato_problem* h);  // host wait, timing, factorization check
int coarse_apply(plato_problem* h, const float* v, float* y, int accumulate, const PcgScalars* S,
                 const float* sq = nullptr);
void coarse_release(plato_problem* h);
void batch_release(plato_problem* h);
int fcg_batch(plato_problem* h, const double* b, double* x, plato_solve_stats* stats);
int ritz_guess(plato_problem* h, const double* b, double* x);
int deflate_direction(plato_problem* h, double* p, const double* r, int update_pr);
constexpr int kEnergySplit = 32;  // CTAs per member in the batched criterion sum
int launch_energy_segments(plato_problem* h, const double* u, const double* z, double* values);
}  // namespace plato
int plato_cuda_fail(plato_problem* h, cudaError_t e, const char* what, const char* file, int line);
namespace plato {
// Raises a kernel's dynamic shared-memory limit to at least `bytes` on the handle's current
// device.  The attribute belongs to one device, so the granted size is remembered per
// (device, kernel) under a lock (a driver call per launch otherwise); a failed attempt is
// not remembered, so every later call retries and reports the same error.
int ensure_smem_attribute(plato_problem* h, const void* kernel, int bytes);
}  // namespace plato

#define PLATO_CUDA(h, expr)                                                          \
    do {                                                                             \
        cudaError_t _e = (expr);                                                     \
        if (_e != cudaSuccess) return plato_cuda_fail((h), _e, #expr, __FILE__, __LINE__); \
    } while (0)

// Returns a non-zero plato_status of a call from the enclosing function.
#define PLATO_RC(expr)                                                               \
    do {                                                                             \
        const int _rc = (expr);                                                      \
        if (_rc) return _rc;                                                         \
    } while (0)

#define PLATO_LAUNCH_CHECK(h)                                                        \
    do {                                                                             \
        (h)->launches += 1;                                                          \
        cudaError_t _e = cudaGetLastError();                                         \
        if (_e != cudaSuccess) return plato_cuda_fail((h), _e, "kernel launch", __FILE__, __LINE__); \
    } while (0)

namespace plato {

constexpr int kNumSMs = 148;

inline int grid_for(int64_t n, int threads, int64_t max_blocks = 148 * 32) {
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > max_blocks) b = max_blocks;
    return int(b);
}

// Programmatic dependent launch (sm_90 and later).  The Krylov loop's kernels are launched with
// launch_pdl: each may be scheduled onto SMs that the kernel before it in the stream has left,
// while that kernel's last CTAs still run, instead of after its completion has reached the
// host-side launch queue.  Every such kernel starts with pdl_wait(), which returns once the
// previous kernel has completed and its memory operations are visible, before it touches any
// memory; pdl_trigger() then lets the next kernel be scheduled.  Launched without the
// attribute, both are no-ops.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl_smem(void (*kernel)(KArgs...), int grid, int block, size_t smem, cudaStream_t stream,
                                   Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(unsigned(grid));
    cfg.blockDim = dim3(unsigned(block));
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), int grid, int block, cudaStream_t stream, Args... args) {
    return launch_pdl_smem(kernel, grid, block, 0, stream, args...);
}

// ---------------------------------------------------------------------------------------
// device element arithmetic

// Basis gradients and weighted volume of a linear tet: ComputeGradientWorkset<3>
// (src/ImplicitFunctors.hpp:169-221) times the 1/6 cubature weight
// (src/LinearTetCubRuleDegreeOne.hpp:72-78).  g[a][d] = d N_a / d x_d.
template <typename T>
struct TetGeom {
    T g[4][3];
    T vol;
};

template <typename T>
__device__ __forceinline__ void tet_geometry(const T x[4][3], TetGeom<T>& G) {
    const T j11 = x[0][0] - x[3][0], j12 = x[1][0] - x[3][0], j13 = x[2][0] - x[3][0];
    const T j21 = x[0][1] - x[3][1], j22 = x[1][1] - x[3][1], j23 = x[2][1] - x[3][1];
    const T j31 = x[0][2] - x[3][2], j32 = x[1][2] - x[3][2], j33 = x[2][2] - x[3][2];
    const T c11 = j22 * j33 - j23 * j32, c12 = j13 * j32 - j12 * j33, c13 = j12 * j23 - j13 * j22;
    const T detj = j11 * c11 + j21 * c12 + j31 * c13;
    const T inv = T(1) / detj;
    G.g[0][0] = c11 * inv;
    G.g[0][1] = c12 * inv;
    G.g[0][2] = c13 * inv;
    G.g[1][0] = (j23 * j31 - j21 * j33) * inv;
    G.g[1][1] = (j11 * j33 - j13 * j31) * inv;
    G.g[1][2] = (j13 * j21 - j11 * j23) * inv;
    G.g[2][0] = (j21 * j32 - j22 * j31) * inv;
    G.g[2][1] = (j12 * j31 - j11 * j32) * inv;
    G.g[2][2] = (j11 * j22 - j12 * j21) * inv;
    G.g[3][0] = -(G.g[0][0] + G.g[1][0] + G.g[2][0]);
    G.g[3][1] = -(G.g[0][1] + G.g[1][1] + G.g[2][1]);
    G.g[3][2] = -(G.g[0][2] + G.g[1][2] + G.g[2][2]);
    G.vol = fabs(detj) * (T(1) / T(6));
}

__device__ __forceinline__ void load_cell_coords(const double* __restrict__ coords, int4 n,
                                                 double x[4][3]) {
    const int ids[4] = {n.x, n.y, n.z, n.w};
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const double* p = coords + 3 * (int64_t)ids[a];
        x[a][0] = __ldg(p + 0);
        x[a][1] = __ldg(p + 1);
        x[a][2] = __ldg(p + 2);
    }
}

// Density of cell c: the mean of its nodal control (ApplyWeighting, src/ApplyWeighting.hpp:
// 55-60), or the cell's own entry with element control.
__device__ __forceinline__ double cell_rho(const Material& m, const double* __restrict__ z, int64_t c, int4 n) {
    if (m.cell_control) return __ldg(z + c);
    return (__ldg(z + n.x) + __ldg(z + n.y) + __ldg(z + n.z) + __ldg(z + n.w)) * 0.25;
}

// d rho_e / d z: 1/4 for each of the cell's nodes, or 1 for the cell's own entry.
__device__ __forceinline__ double rho_dz(const Material& m) { return m.cell_control ? 1.0 : 0.25; }

__device__ __forceinline__ int node_of(int4 n, int a) {
    return a == 0 ? n.x : (a == 1 ? n.y : (a == 2 ? n.z : n.w));
}

// MSIMP s(rho) = rho_min + (1 - rho_min) rho^p and its derivative (src/Simp.hpp:130-134).
// Integer exponents use repeated products (within 2 ulp of pow).
template <typename T>
__device__ __forceinline__ T ipow(T r, int p) {
    T v = T(1);
    for (int i = 0; i < p; ++i) v *= r;
    return v;
}

template <typename T>
__device__ __forceinline__ T simp(const Material& m, T rho) {
    const T pw = m.p_int >= 0 ? ipow(rho, m.p_int) : T(pow(double(rho), m.p));
    return T(m.rho_min) + (T(1) - T(m.rho_min)) * pw;
}

template <typename T>
__device__ __forceinline__ T simp_dx(const Material& m, T rho) {
    T pw;
    if (m.p_int >= 1) pw = ipow(rho, m.p_int - 1);
    else if (m.p_int == 0) pw = T(0);
    else pw = T(pow(double(rho), m.p - 1.0));
    return (T(1) - T(m.rho_min)) * (T(m.p) * pw);
}

// Voigt strain (xx, yy, zz, yz, xz, xy) with engineering shear, Strain<3>
// (src/Strain.hpp:70-95).
template <typename T>
__device__ __forceinline__ void strain_voigt(const T g[4][3], const T u[4][3], T e[6]) {
#pragma unroll
    for (int v = 0; v < 6; ++v) e[v] = T(0);
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        e[0] += u[a][0] * g[a][0];
        e[1] += u[a][1] * g[a][1];
        e[2] += u[a][2] * g[a][2];
        e[3] += u[a][2] * g[a][1] + u[a][1] * g[a][2];
        e[4] += u[a][2] * g[a][0] + u[a][0] * g[a][2];
        e[5] += u[a][1] * g[a][0] + u[a][0] * g[a][1];
    }
}

// Isotropic stress sigma = C eps, LinearStress (src/LinearStress.hpp:102-120).
template <typename T>
__device__ __forceinline__ void stress_voigt(const Material& m, const T e[6], T s[6]) {
    const T c00 = T(m.c00), c01 = T(m.c01), c33 = T(m.c33);
    s[0] = e[0] * c00 + e[1] * c01 + e[2] * c01;
    s[1] = e[0] * c01 + e[1] * c00 + e[2] * c01;
    s[2] = e[0] * c01 + e[1] * c01 + e[2] * c00;
    s[3] = e[3] * c33;
    s[4] = e[4] * c33;
    s[5] = e[5] * c33;
}

// f_a = vol * B_a^T sigma: StressDivergence<3> (src/StressDivergence.hpp:70-90) for node a.
template <typename T>
__device__ __forceinline__ void divergence_node(const T ga[3], const T s[6], T w, T f[3]) {
    f[0] = w * (s[0] * ga[0] + s[5] * ga[1] + s[4] * ga[2]);
    f[1] = w * (s[5] * ga[0] + s[1] * ga[1] + s[3] * ga[2]);
    f[2] = w * (s[4] * ga[0] + s[3] * ga[1] + s[2] * ga[2]);
}

// 3x3 block (a,b) of the element stiffness w * B_a^T C B_b for isotropic C:
// K_ab[i][j] = w (lambda ga_i gb_j + mu ga_j gb_i + mu (ga . gb) delta_ij).
template <typename T>
__device__ __forceinline__ void stiffness_block(const Material& m, const T ga[3], const T gb[3],
                                                T w, T K[9]) {
    const T lam = T(m.c01) * w, mu = T(m.c33) * w;
    const T dot = ga[0] * gb[0] + ga[1] * gb[1] + ga[2] * gb[2];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            T v = lam * ga[i] * gb[j] + mu * ga[j] * gb[i];
            if (i == j) v += mu * dot;
            K[3 * i + j] = v;
        }
}

}  // namespace plato
