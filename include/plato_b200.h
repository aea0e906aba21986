/*
 * plato_b200.h -- C ABI of the B200 elliptic mechanics path.
 *
 * Drop-in replacement for the Plato Analyze elliptic hot path: SIMP-penalised linear
 * elastostatics on 4-node tetrahedra (SimplexMechanics<3> + LinearTetCubRuleDegreeOne),
 * its residual and block-CRS Jacobian, the linear solve behind Problem::solution, and the
 * "Internal Elastic Energy" criterion (compliance) with its adjoint sensitivity dC/dz.
 * Each entry point names the reference interface it replaces (paths relative to the
 * reference project).
 *
 * Conventions (same as the reference, src/PlatoTypes.hpp:15-20 and
 * src/ImplicitFunctors.hpp:47-89): Scalar = double, ordinals = int32, dof = 3*node + dim,
 * connectivity cell*4 + k, coordinates node*3 + dim, control z nodal (length num_nodes).
 * Block CRS ("CrsMatrix", src/alg/CrsMatrix.hpp:20-111): row_map over node rows (N+1),
 * column_indices node ids sorted with the diagonal included (CreateBlockMatrix,
 * src/ImplicitFunctors.hpp:932-1005), entries row-major per block.
 *
 * Pointers marked [device] are CUDA device pointers on the handle's device; [host] are host
 * pointers.  Every function returns a plato_status; no exception crosses the ABI.  A handle
 * is bound to one CUDA stream; calls on one handle must not run concurrently.
 */
#ifndef PLATO_B200_H
#define PLATO_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum plato_status {
    PLATO_OK             = 0,
    PLATO_BAD_INPUT      = 1, /* invalid sizes, pointers, inverted/degenerate cells, bad options */
    PLATO_NOT_CONVERGED  = 2, /* solver hit max_iterations; outputs hold the last iterate   */
    PLATO_NONFINITE      = 3, /* NaN/Inf met in an input or a solver scalar                 */
    PLATO_DEVICE_TIMEOUT = 4, /* a bounded device-side wait ran out                         */
    PLATO_CUDA_ERROR     = 5, /* CUDA runtime error; see plato_last_error                   */
    PLATO_OUT_OF_MEMORY  = 6,
    PLATO_NOT_SUPPORTED  = 7
} plato_status;

typedef enum plato_operator_kind {
    PLATO_OPERATOR_ASSEMBLED   = 0, /* assembled 3x3 block CRS, FP64 SpMV                  */
    PLATO_OPERATOR_MATRIX_FREE = 1  /* element-by-element apply recomputed from the mesh   */
} plato_operator_kind;

typedef enum plato_precision {
    PLATO_PRECISION_FP64       = 0, /* plain FP64 Jacobi-PCG                                */
    PLATO_PRECISION_MIXED_FP32 = 1, /* FP32 inner PCG inside FP64 iterative refinement      */
    PLATO_PRECISION_MIXED_BF16 = 2, /* as MIXED_FP32 with the block CRS stored in BF16      */
    PLATO_PRECISION_MIXED_FP16 = 3, /* as MIXED_FP32 with the Jacobi-scaled matrix
                                       D^-1/2 A D^-1/2 stored in FP16 (unit diagonal, entries
                                       in [-1, 1]); the Chebyshev sweep runs in scaled
                                       variables (assembled operator only)                 */
    PLATO_PRECISION_MIXED_FP32_ASSEMBLED = 4 /* matrix-free operator only: the FP64 outer
                                       operator is the element-by-element apply and the
                                       preconditioner's matrix is assembled by FP32 element
                                       kernels (gradients, weights and sums in FP32) straight
                                       into an FP32 SELL copy; no FP64 matrix exists        */
} plato_precision;

typedef struct plato_problem plato_problem; /* opaque handle */

typedef struct plato_mesh_desc {
    int32_t        num_nodes;
    int32_t        num_cells;
    const double*  coords;       /* [host] num_nodes*3 */
    const int32_t* connectivity; /* [host] num_cells*4 */
} plato_mesh_desc;

/* "Isotropic Linear Elastic" (src/IsotropicLinearElasticMaterial.cpp:86-110) */
typedef struct plato_material {
    double youngs_modulus;
    double poissons_ratio;
} plato_material;

/* "Penalty Function" Type SIMP -> MSIMP (src/Simp.hpp:41-52) */
typedef struct plato_penalty {
    double exponent;      /* reference default 3   */
    double minimum_value; /* reference default 1e-9 */
} plato_penalty;

/* One "Uniform" natural BC on a side set (src/NaturalBC.hpp:87-113): the side set is
 * given as GetSideSetElements / GetSideSetLocalNodes would return it. */
typedef struct plato_natural_bc {
    int32_t        num_faces;
    const int32_t* face_cells;       /* [host] owning cell of each face              */
    const int32_t* face_local_nodes; /* [host] 3 cell-local node ordinals per face    */
    double         vector[3];        /* traction ("Vector")                          */
} plato_natural_bc;

/* Essential BCs as the Problem holds them (mBcDofs / mBcValues, src/EssentialBCs.hpp:79-88) */
typedef struct plato_essential_bcs {
    int32_t        num_dofs;
    const int32_t* dofs;   /* [host] */
    const double*  values; /* [host] */
} plato_essential_bcs;

typedef struct plato_solver_opts {
    double  tolerance;        /* stop on ||b - A x|| / ||b|| <= tolerance (FP64)          */
    int32_t max_iterations;   /* total inner iterations allowed                          */
    int32_t operator_kind;    /* plato_operator_kind                                      */
    int32_t precision;        /* plato_precision                                          */
    int32_t self_adjoint;     /* Problem "Self-Adjoint" (src/elliptic/Problem.hpp:116)    */
    double  chebyshev_ratio;  /* preconditioner interval [lambda_max/ratio, lambda_max]    */
    int32_t chebyshev_degree; /* Chebyshev steps per preconditioner call (it applies the
                                 operator degree-1 times); 0 with FP64 + assembled = the
                                 plain Jacobi-PCG, 1 = Jacobi inside flexible CG           */
    int32_t coarse_cells[3];  /* two-level preconditioner: coarse box grid of
                                 coarse_cells[0] x [1] x [2] cells over the mesh bounding
                                 box (trilinear coarse space, Galerkin coarse operator);
                                 {0,0,0} = none.  Needs every element inside one coarse
                                 cell (box meshes with divisible cell counts)             */
    int32_t fallback_max_iterations; /* when a flexible-CG method (precision != FP64, a
                                 Chebyshev degree, a coarse grid or the matrix-free operator)
                                 ends without meeting the tolerance or breaks down, the solve
                                 is retried from a zero guess if a subspace guess seeded it,
                                 then falls back to the plain FP64 Jacobi-PCG from a zero
                                 guess; this caps the fallback's iterations (0: the same cap
                                 as max_iterations, < 0: no fallback)                      */
    int32_t chebyshev_kind;   /* polynomial of the Chebyshev preconditioner: 0 or 1 = first
                                 kind on [lambda_max/ratio, lambda_max]; 4 = fourth kind on
                                 (0, lambda_max] (Lottes, Numer. Linear Algebra Appl. 2023;
                                 chebyshev_ratio unused), which damps the upper part of the
                                 spectrum more and leaves the lowest modes to the coarse space */
    int32_t sweep_steps;      /* FP16 scaled sweep (PLATO_PRECISION_MIXED_FP16): Chebyshev steps
                                 per launch.  0 or 1 = one launch per step; 2..16 = that many
                                 steps in one launch, each (step, 512-row tile) task waiting only
                                 for the tiles of the step before that its columns reach, so the
                                 matrix can be re-read from L2 (needs 16-bit column offsets)  */
    int32_t sweep_lag;        /* multi-step sweep: tiles of 512 rows by which each step trails the
                                 one before beyond the column reach (0 = 600 / sweep_steps)  */
} plato_solver_opts;

typedef struct plato_problem_desc {
    plato_mesh_desc         mesh;
    plato_material          material;
    plato_penalty           penalty;
    int32_t                 num_natural_bcs;
    const plato_natural_bc* natural_bcs;  /* [host] */
    plato_essential_bcs     essential_bcs;
    plato_solver_opts       solver;
} plato_problem_desc;

typedef struct plato_solve_stats {
    int32_t iterations;        /* outer (FP64) Krylov iterations            */
    int32_t refinements;       /* preconditioner operator applies in total */
    double  relative_residual; /* FP64 ||b - A x|| / ||b|| at exit          */
    int32_t converged;
    int32_t status;            /* plato_status of the solve                */
    int32_t fallback;          /* 0: the configured method converged; 1: it converged after a
                                  retry from a zero guess (the subspace guess failed); 2: the
                                  plain FP64 Jacobi-PCG fallback ran (iterations and residual
                                  are the fallback's)                                     */
} plato_solve_stats;

/* ---- lifetime -------------------------------------------------------------------------
 * Replaces the construction of Elliptic::Problem + VectorFunction + the criterion
 * (src/elliptic/Problem.hpp:99-125).  Copies mesh and BCs to the device, builds the node
 * graph and block pattern once, precomputes the traction load vector. */
int plato_create(const plato_problem_desc* desc, plato_problem** out);
int plato_destroy(plato_problem* h);
/* Last error text of a handle (or of the last failed plato_create when h is NULL). */
const char* plato_last_error(const plato_problem* h);
/* Bind the handle to a CUDA stream (cudaStream_t); NULL means the legacy default stream. */
int plato_set_stream(plato_problem* h, void* cuda_stream);
int plato_set_solver_opts(plato_problem* h, const plato_solver_opts* opts);
/* Control layout (no reference counterpart: the reference's control is nodal and each cell
 * takes the mean of its nodes, ApplyWeighting, src/ApplyWeighting.hpp:55-64).
 * PLATO_CONTROL_ELEMENT gives every cell its own density: from then on every entry point's
 * control z has num_cells entries (cell order) and every control derivative (sf_gradient_z,
 * vf_gradient_z_apply, problem_criterion_gradient, volume_gradient_z) has num_cells entries,
 * d/dz_e of the cell's own terms.  The (dR/dz)^T block matrix (vf_gradient_z) and batches
 * are nodal only (PLATO_NOT_SUPPORTED). */
typedef enum plato_control_layout {
    PLATO_CONTROL_NODAL   = 0,
    PLATO_CONTROL_ELEMENT = 1
} plato_control_layout;
int plato_set_control_layout(plato_problem* h, int32_t layout);
int plato_get_sizes(const plato_problem* h, int32_t* num_nodes, int32_t* num_cells,
                    int64_t* num_blocks);
/* Instrumentation (no reference counterpart; the reference times phases with
 * Teuchos::TimeMonitor, src/alg/EpetraLinearSolver.cpp:16-17).  With timing enabled, every
 * 8th operator apply inside the solver is bracketed by CUDA events on the handle's stream;
 * op_ms_total / op_timed is the average apply duration.  launches counts every kernel the
 * handle has launched. */
int plato_set_timing(plato_problem* h, int32_t enable);
int plato_get_instrumentation(const plato_problem* h, int64_t* launches, double* op_ms_total,
                              int64_t* op_timed);
int plato_reset_instrumentation(plato_problem* h);
/* Sampled CUDA-event time of one kernel class inside the solvers: kind 0 = the FP64 operator
 * apply of the Krylov loop, kind 1 = the Chebyshev steps of the low-precision preconditioner
 * (one step = one preconditioner-operator apply fused with its update; a sampled call is timed
 * over its whole run of step launches and counts as its number of steps),
 * kind 2 = the Jacobian assembly of each assembled solve, kind 3 = the Galerkin product of
 * the two-level coarse operator, kind 4 = its dense factorization and inverse (kinds 3 and 4
 * count coarse operator set-ups); kinds 5-8 time every call with timing on: 5 = the residual
 * of plato_vf_value (load copy + element force kernel), 6 = the energy sum of plato_sf_value,
 * 7 = the self-adjoint dC/dz of plato_problem_criterion_gradient (per-cell pass + nodal
 * sums), 8 = plato_problem_criterion_value_and_gradient's one pass (+ nodal sums).  Reading
 * kinds 5-8 waits for the last timed launch of that kind.  With the multi-step FP16 sweep
 * (sweep_steps) kind 1 times the first launch of the sampled preconditioner calls and counts
 * it as its number of steps; either way ms_total / count is the time per step. */
int plato_get_kernel_timing(const plato_problem* h, int32_t kind, double* ms_total, int64_t* count);
/* The FP16 sweep of the last flexible-CG solve: Chebyshev steps per launch (1 = one launch
 * per step; > 1 = the multi-step sweep) and its column reach in tiles of 512 rows (-1 when
 * not measured). */
int plato_get_sweep_info(const plato_problem* h, int32_t* steps_per_launch, int32_t* halo_tiles);
/* Test hook for the bounded device waits (no reference counterpart): the next multi-step sweep
 * launch of this handle waits for a completion stamp that none of its tasks writes, so its
 * first dependency wait gives up after its poll limit (about a second).  The launch then ends,
 * the solve reports the timeout to the host, the multi-step sweep is switched off for the
 * handle and the plain FP64 Jacobi-PCG fallback finishes the solve (fallback_max_iterations). */
int plato_test_stall_next_sweep(plato_problem* h);
/* The solver's SELL-32 layout of the block matrix: slots (blocks plus the padding of each
 * 32-row slice to its widest row) and the bytes per column index the FP16 preconditioner
 * sweep reads (2 when every column lies within 32767 of its slice's first row, else 4). */
int plato_get_sell_info(const plato_problem* h, int64_t* total_slots, int32_t* column_bytes);

/* ---- block pattern ---------------------------------------------------------------------
 * CreateBlockMatrix (src/ImplicitFunctors.hpp:932-1005) over the node-node graph
 * (src/EngineMesh.cpp:223-320).  Copies row_map (N+1) and column_indices (num_blocks). */
int plato_jacobian_pattern(plato_problem* h, int32_t* row_map, int32_t* column_indices /*[device]*/);

/* ---- Elliptic::VectorFunction (src/elliptic/VectorFunction.hpp) ------------------------ */
/* value(u,z): R = K(z) u - F, :251-334 */
int plato_vf_value(plato_problem* h, const double* u, const double* z, double* R /*[device]*/);
/* gradient_u(u,z): 3x3 block entries on the handle's pattern, :525-615 */
int plato_vf_gradient_u(plato_problem* h, const double* u, const double* z, double* entries);
/* gradient_u_T(u,z): transpose assembly, :432-523 */
int plato_vf_gradient_u_T(plato_problem* h, const double* u, const double* z, double* entries);
/* gradient_z(u,z): (dR/dz)^T, N x 3N with 1x3 blocks on the same pattern, :618-710 */
int plato_vf_gradient_z(plato_problem* h, const double* u, const double* z, double* entries);
/* out += gradient_z(u,z) * lambda without forming the matrix (Problem.hpp:445-448 fused) */
int plato_vf_gradient_z_apply(plato_problem* h, const double* u, const double* z,
                              const double* lambda, double* out /*[device]*/);

/* ---- Elliptic::PhysicsScalarFunction "Internal Elastic Energy" -------------------------
 * (src/elliptic/PhysicsScalarFunction.hpp, src/elliptic/InternalElasticEnergy.hpp) */
int plato_sf_value(plato_problem* h, const double* u, const double* z, double* value /*[host]*/);
int plato_sf_gradient_u(plato_problem* h, const double* u, const double* z, double* dfdu);
int plato_sf_gradient_z(plato_problem* h, const double* u, const double* z, double* dfdz);

/* ---- Geometric "Volume" criterion (src/geometric/Volume.hpp:83-110) --------------------
 * V(z) = sum_e |det J_e| / 6 * s_v(rho_e) with the criterion's own penalty s_v (MSIMP
 * parameters; exponent 1 and minimum 0 give the material volume sum_e vol_e rho_e), and
 * dV/dz on the nodes (GeometryScalarFunction::gradient_z, SFad<4> control derivative). */
int plato_volume_value(plato_problem* h, const double* z, const plato_penalty* penalty, double* value /*[host]*/);
int plato_volume_gradient_z(plato_problem* h, const double* z, const plato_penalty* penalty, double* dvdz);

/* ---- helpers ----------------------------------------------------------------------------
 * applyBlockConstraints<3> with the handle's essential BCs (src/ApplyConstraints.hpp:40-112);
 * scale multiplies the BC values (0 for the adjoint, src/elliptic/Problem.hpp:701-713). */
int plato_apply_constraints(plato_problem* h, double* entries, double* rhs, double scale);
/* y += A x on the handle's pattern, blocks rows_per_block x cols_per_block (3x3 or 1x3);
 * MatrixTimesVectorPlusVector, src/PlatoMathHelpers.hpp:78-159 */
int plato_matvec_plus(plato_problem* h, int32_t rows_per_block, int32_t cols_per_block,
                      const double* entries, const double* x, double* y);

/* y = K_c(z) x with K_c the Dirichlet-constrained stiffness that Problem::solution hands to
 * the solver (gradient_u + applyBlockConstraints, src/elliptic/Problem.hpp:262-266), applied
 * either from the assembled block matrix (operator_kind = PLATO_OPERATOR_ASSEMBLED) or
 * element by element without a matrix (PLATO_OPERATOR_MATRIX_FREE). */
int plato_apply_operator(plato_problem* h, const double* z, int32_t operator_kind, const double* x,
                         double* y /*[device]*/);

/* ---- AbstractSolver::solve (src/alg/PlatoAbstractSolver.hpp:38-106) ---------------------
 * Jacobi-PCG on an assembled, constrained 3x3 block matrix: A x = b, x holds the initial
 * guess on entry. */
int plato_solver_solve(plato_problem* h, const double* entries, double* x, const double* b,
                       plato_solve_stats* stats);

/* ---- two-level preconditioner diagnostics (no reference counterpart) ------------------
 * The Galerkin coarse operator E = (PZ)^T K(z) (PZ) of the solver options' coarse grid
 * (Z trilinear on the box grid, P masking the constrained dofs; a dof whose column
 * vanishes gets a unit diagonal) and the E^-1 the preconditioner applies, both [host]
 * row-major ndof x ndof.  With E and Einv NULL only *ndof is set.  z [device]. */
int plato_coarse_operator(plato_problem* h, const double* z, int32_t* ndof, double* E, double* Einv);

/* ---- Elliptic::Problem (src/elliptic/Problem.hpp) --------------------------------------- */
/* solution(z), :237-292; u [device] receives the state.  u0 (may be NULL) seeds the solve. */
int plato_problem_solution(plato_problem* h, const double* z, const double* u0, double* u,
                           plato_solve_stats* stats);
/* criterionValue(z, u), :300-354 */
int plato_problem_criterion_value(plato_problem* h, const double* z, const double* u,
                                  double* value /*[host]*/);
/* criterionGradient(z, u), :395-450 (self-adjoint shortcut or adjoint solve) */
int plato_problem_criterion_gradient(plato_problem* h, const double* z, const double* u,
                                     double* dfdz, plato_solve_stats* stats);
/* criterionValue and criterionGradient together (what an MPMD ComputeCriterion operation
 * computes, src/Analyze_App.cpp:727-1014): with the self-adjoint shortcut one pass over the
 * cells gives the compliance (*value, host) and dC/dz [device]; otherwise the two calls above. */
int plato_problem_criterion_value_and_gradient(plato_problem* h, const double* z, const double* u,
                                               double* value /*[host]*/, double* dfdz, plato_solve_stats* stats);
/* One optimisation step on HOST buffers: z -> u, compliance value, dC/dz.  Host<->device
 * copies are part of the call (what an MPMD ComputeSolution + ComputeCriterion +
 * ComputeCriterionGradient sequence does, src/Analyze_App.cpp:727-1201). */
int plato_problem_solve_and_gradient_host(plato_problem* h, const double* z_host,
                                          const double* u0_host, double* u_host,
                                          double* value_host, double* dfdz_host,
                                          plato_solve_stats* stats);

/* ---- allocation-free compliance value ---------------------------------------------------
 * No counterpart in the reference.  Same value as plato_sf_value (internal elastic energy,
 * 1/2 u^T K(z) u over the cells) for callers that cannot allocate device memory when they
 * need it (their device memory belongs to another allocator's pool, or they must not risk
 * the implicit synchronisation of cudaMalloc/cudaFree).  No handle: connectivity
 * (num_cells*4 int32, 16-byte aligned), coords (num_nodes*3), u (num_nodes*3) and z
 * (num_nodes) are caller-owned [device] arrays; value is a [device] double written on
 * cuda_stream (NULL = legacy stream).  The call waits for its kernel (it synchronises
 * cuda_stream) so that its status reports what the kernel found: a connectivity id outside
 * [0, num_nodes) gives PLATO_BAD_INPUT (such cells are skipped on the device, never read,
 * and *value is NaN), a non-finite value gives PLATO_NONFINITE.  Material and penalty are
 * checked as plato_create checks them.
 * The call allocates nothing: its reduction scratch is a static device array of 65,536 block
 * partial sums plus two counters (512 KiB, held by every GPU that loads the library until
 * exit), so num_cells is limited to 16,777,216; larger meshes get PLATO_BAD_INPUT.  The first
 * call on a device looks up the scratch address on the current device; make that first call
 * before any stream capture.  Every call shares the one scratch array, which keeps the last
 * call's contents (the counters are cleared at the start of each call): calls whose kernels
 * overlap on the GPU (different streams, or different host threads on one device) race and
 * must be serialised by the caller.  Errors read through plato_last_error(NULL). */
int plato_sf_value_noalloc(int32_t num_nodes, int32_t num_cells, const int32_t* connectivity,
                           const double* coords, const double* u, const double* z,
                           const plato_material* material, const plato_penalty* penalty,
                           double* value, void* cuda_stream);

/* ---- batches of independent problems (no reference counterpart: the reference builds one
 * Elliptic::Problem per design and load case, src/elliptic/Problem.hpp:80-140) -----------
 * plato_create_batch returns ONE handle over the disjoint union of `count` problems: member
 * s's nodes, cells, essential-BC dofs and traction faces follow those of members 0..s-1
 * (plato_batch_info gives the offsets).  Every entry point above then acts on the union:
 * vectors are the members' vectors concatenated, the block pattern is block diagonal, and
 * the solves (problem_solution, the adjoint, solver_solve) run every member to its own stop
 * test ||r_s|| <= tol ||b_s|| in one batched flexible CG (one launch per stage for all
 * members; Chebyshev-Jacobi preconditioner of solver.chebyshev_degree, Jacobi when it is 0).
 * Members must share material and penalty; the solver options are descs[0].solver; the
 * matrix-free operator and the coarse space are PLATO_NOT_SUPPORTED for batches.  The
 * aggregate statistics of a solve carry the maximum iterations and relative residual. */
int plato_create_batch(int32_t count, const plato_problem_desc* descs, plato_problem** out);
/* count (1 for a single problem) and the member offsets node_offsets[count+1],
 * cell_offsets[count+1] (either may be NULL) */
int plato_batch_info(const plato_problem* h, int32_t* count, int32_t* node_offsets, int32_t* cell_offsets);
/* per-member statistics of the last solve on a batch handle: stats[count] (host) */
int plato_batch_last_stats(const plato_problem* h, plato_solve_stats* stats);
/* per-member criterion values (internal elastic energy, PhysicsScalarFunction::value for
 * each member) into values[count] [device]; synchronises the handle's stream */
int plato_batch_criterion_values(plato_problem* h, const double* z, const double* u, double* values);

/* Autotuner of the batched solve (no reference counterpart).  The batched Krylov kernels are
 * persistent: a grid of ctas_per_sm x SMs CTAs walks the members' row tiles (tiles of
 * tile_rows rows, never across two members, one row per thread), skipping converged members.
 * plato_batch_autotune times every pair tile_rows in {128, 256, 512} x ctas_per_sm in
 * {2, 4, 8, 16} on 8 flexible-CG iterations of this batch with control z [device] (the
 * handle's solver options; the callers' vectors are untouched), keeps the fastest for the
 * handle's later solves and reports all timings.  Without it a batch uses 256 x 8. */
typedef struct plato_batch_tuning {
    int32_t tile_rows;            /* chosen */
    int32_t ctas_per_sm;          /* chosen */
    int32_t candidates;           /* pairs timed */
    int32_t iterations;           /* flexible-CG iterations per timing */
    int32_t tile_rows_tried[16];
    int32_t ctas_per_sm_tried[16];
    double  ms_tried[16];         /* set-up + iterations of each pair (second of two runs) */
} plato_batch_tuning;
int plato_batch_autotune(plato_problem* h, const double* z, plato_batch_tuning* out);

/* Problem::solution with an initial guess improved on a subspace (no reference counterpart;
 * the learned warm start uses it).  W holds k <= 8 columns of 3N values [device]; after the
 * operator is assembled and constrained, the iterate x (u0, or zero) becomes x + P W c with
 * (W^T P K P W) c = W^T P (b - K x) (P zeroes the constrained dofs): the minimiser of the
 * energy error over x + span(P W).  The correction is dropped (x kept) when the Gram matrix
 * is not positive definite or ||b - K x|| would become non-finite or grow more than 10x; the
 * solve then runs to the usual tolerance.  *residual_ratio (may be NULL) receives ||b - K x||
 * after / before the correction (1 when it was dropped).  Single problems on the assembled
 * operator only. */
int plato_problem_solution_subspace(plato_problem* h, const double* z, const double* u0, const double* W, int32_t k,
                                    double* u, plato_solve_stats* stats, double* residual_ratio);
/* The same, with the subspace also deflating the Krylov iteration (no reference counterpart;
 * the learned network's fields use it): after the Galerkin guess above, every search
 * direction is made A-orthogonal to P W (deflated CG), so the solver never searches span(P W)
 * again.  Plain Jacobi-PCG and the flexible-CG methods on the assembled operator; deflation is
 * skipped (the plain solve runs) when the Gram matrix is not positive definite or the guess
 * was dropped.  A failed deflated solve falls back like the others (fallback_max_iterations). */
int plato_problem_solution_deflated(plato_problem* h, const double* z, const double* u0, const double* W,
                                    int32_t k, double* u, plato_solve_stats* stats, double* residual_ratio);

/* ---- learned warm start (no reference counterpart) -------------------------------------
 * A 3-level 3D U-Net (16-32-64 channels; 3x3x3 convolutions with ReLU, 2x2x2 average pooling,
 * nearest upsampling, skip concatenation, 1x1x1 head) on the nodes of an n0 x n1 x n2 box
 * node grid (zero-padded to multiples of 4).  Input: 8 FP32 features per node
 * [batch][n0][n1][n2][8]; output: 9 FP32 values per node [batch][n0][n1][n2][9].  BF16
 * tensor-core kernels with FP32 accumulation for every convolution, forward and backward;
 * FP32 parameters trained with Adam.  All array arguments are [device]; work is issued on the
 * network's stream; errors read through plato_unet_last_error(). */
typedef struct plato_unet plato_unet;
typedef enum plato_unet_conv_kernel {
    PLATO_UNET_CONV_TCGEN05  = 0, /* default: tcgen05.mma from shared-memory descriptors, FP32
                                     accumulator in tensor memory, 128 voxels x all output
                                     channels per CTA, two cp.async-filled stages per tap     */
    PLATO_UNET_CONV_MMA_SYNC = 1  /* warp-level mma.sync.m16n8k16 tiles, register accumulators */
} plato_unet_conv_kernel;
int plato_unet_create(const int32_t nodes[3], int32_t max_batch, plato_unet** out);
/* the kernel family of the forward and data-gradient convolutions (plato_unet_conv_kernel) */
int plato_unet_set_conv_kernel(plato_unet* net, int32_t kind);
/* waits for the network's stream; PLATO_DEVICE_TIMEOUT when a tensor-core convolution's bounded
 * wait for its MMAs ran out since the last check (its outputs were then not written) */
int plato_unet_check(plato_unet* net);
int plato_unet_destroy(plato_unet* net);
int plato_unet_set_stream(plato_unet* net, void* cuda_stream);
const char* plato_unet_last_error(void);
int plato_unet_num_params(const plato_unet* net, int64_t* count);
/* parameters: per layer, weights [taps][cout][cin] then bias [cout]; setting them resets Adam */
int plato_unet_set_params(plato_unet* net, const float* params);
int plato_unet_get_params(const plato_unet* net, float* params);
int plato_unet_forward(plato_unet* net, int32_t batch, const float* input, float* output);
/* mean squared error against target [batch][n0][n1][n2][9] and the parameter gradient (kept
 * for plato_unet_adam_step; also copied to grads when non-NULL); *loss is a [host] double */
int plato_unet_loss_and_gradients(plato_unet* net, int32_t batch, const float* input, const float* target,
                                  double* loss, float* grads);
int plato_unet_adam_step(plato_unet* net, float learning_rate, int32_t step);
/* network input for a box design: the 8 features per node of the net_nodes grid (density
 * interpolated trilinearly from the src_nodes grid's nodal z, loaded-face and clamped-face
 * masks at the two x ends, normalised coordinates, density cubed, zero) into features [device] */
int plato_unet_features(const int32_t src_nodes[3], const double* z, const int32_t net_nodes[3], float* features,
                        void* cuda_stream);
/* the 3 subspace columns W [3][3 * dst nodes] (column d = predicted response to a unit
 * traction along axis d, trilinear from the network output [net nodes][9]) */
int plato_unet_subspace(const int32_t net_nodes[3], const float* output, const int32_t dst_nodes[3], double* W,
                        void* cuda_stream);
/* `passes` 7-point averaging passes (each node becomes the mean of itself and its face
 * neighbours) over FP32 data [nodes][channels] in place; scratch holds as many floats */
int plato_box_smooth(const int32_t nodes[3], int32_t channels, int32_t passes, float* data, float* scratch,
                     void* cuda_stream);
/* trilinear resampling of `channels` FP64 values per node between two node grids spanning the
 * same box (nodes ordered z fastest) */
int plato_box_resample(const int32_t src_nodes[3], const int32_t dst_nodes[3], int32_t channels, const double* src,
                       double* dst, void* cuda_stream);

/* ---- Helmholtz density filter (src/helmholtz/Problem.hpp, VectorFunction.hpp,
 * HelmholtzResidual.hpp) ------------------------------------------------------------------
 * A filter handle over the mesh: one unknown per node, the same node pattern as the
 * mechanics (plato_jacobian_pattern), every array [device] of num_nodes values, entries one
 * value per block.  Solves are FP64 Jacobi-PCG to solver.tolerance (0: 1e-12) within
 * solver.max_iterations (0: 100000); the other solver fields are ignored.  plato_destroy
 * releases the handle. */
typedef struct plato_helmholtz_desc {
    plato_mesh_desc    mesh;
    double             length_scale;         /* "Length Scale" L > 0 (HelmholtzResidual.hpp:81)     */
    double             surface_length_scale; /* "Surface Length Scale" alpha >= 0 (:82); 0 = none   */
    int32_t            num_surface_faces;    /* faces carrying the surface term: the exterior faces
                                                outside the "Symmetry Plane Sides" (:197-198)       */
    const int32_t*     surface_face_cells;       /* [host] owning cell of each face              */
    const int32_t*     surface_face_local_nodes; /* [host] 3 cell-local node ordinals per face    */
    plato_solver_opts  solver;
} plato_helmholtz_desc;
int plato_create_helmholtz(const plato_helmholtz_desc* desc, plato_problem** out);
/* VectorFunction::value: R = K filtered - M control, K including the surface term
 * alpha L sum over faces of (area / 9) for the face's node pairs (evaluate_boundary) */
int plato_helmholtz_value(plato_problem* h, const double* filtered, const double* control, double* R);
/* VectorFunction::gradient_u: K_ab = sum vol (L^2 g_a . g_b + 1/16) + the surface term
 * (assembled once per handle) */
int plato_helmholtz_gradient_u(plato_problem* h, double* entries);
/* VectorFunction::gradient_z, transposed as the reference returns it: -sum vol / 16 */
int plato_helmholtz_gradient_z(plato_problem* h, double* entries);
/* Problem::solution (src/helmholtz/Problem.hpp:158-176): filtered = K^-1 M control */
int plato_helmholtz_solution(plato_problem* h, const double* control, double* filtered, plato_solve_stats* stats);
/* Problem::criterionGradient (src/helmholtz/Problem.hpp:187-208): from the criterion's
 * derivative with respect to the filtered density to the one with respect to the control,
 * dfdcontrol = (dR/dcontrol)^T K^-1 (-dfdfiltered) = M K^-1 dfdfiltered.  Unlike the reference,
 * the input is not negated in place. */
int plato_helmholtz_criterion_gradient(plato_problem* h, const double* dfdfiltered, double* dfdcontrol,
                                       plato_solve_stats* stats);

/* ---- MPMD application (src/Analyze_App.hpp, src/Analyze_App.cpp; Plato::Application) --
 * The reference's Analyze application driven by PlatoEngine: an input deck (Teuchos
 * ParameterList XML: "Input Mesh", "Physics", "PDE Constraint", "Spatial Model", "Material
 * Models", "Elliptic" > "Penalty Function", "Criteria", "Natural Boundary Conditions",
 * "Essential Boundary Conditions", "Linear Solver", "Self-Adjoint"; for the filter
 * "Parameters" > "Length Scale", "Surface Length Scale", "Symmetry Plane Sides") and an
 * operations file (<Operation> elements: Function, Name, Criterion, Target, ProblemDefinition,
 * Output > Argument/ArgumentName, Parameter > ArgumentName/Target/InitialValue).
 * Functions built: ComputeSolution, ComputeCriterion, ComputeCriterionValue,
 * ComputeCriterionGradient, ApplyHelmholtz, ApplyHelmholtzGradient, UpdateProblem.
 * "Input Mesh" = an Exodus II file (plato_mesh_file_open; relative to base_dir) or
 * "box:NX,NY,NZ[:LX,LY,LZ]" (generated; node and side sets x-, x+, y-, y+, z-, z+).
 * Shared data crosses as host arrays: fields of num_nodes values, values of one. */
typedef struct plato_app plato_app;
typedef enum plato_data_layout {
    PLATO_LAYOUT_SCALAR_FIELD     = 0, /* nodal field ("Topology", gradients, state components) */
    PLATO_LAYOUT_SCALAR_VALUE     = 1, /* one number (criterion value minus its Target)         */
    PLATO_LAYOUT_SCALAR_PARAMETER = 2  /* operation parameter; context = the operation's Name    */
} plato_data_layout;
/* MPMD_App constructor + initialize (src/Analyze_App.cpp:301-366).  input_config and
 * operations are XML text (first non-blank character '<') or file names, relative to
 * base_dir (may be NULL).  On failure *out is NULL and plato_app_last_error(NULL) says why. */
int plato_app_create(const char* input_config, const char* operations, const char* base_dir, plato_app** out);
/* Host-only check of a deck and operations file: parses both, generates the mesh, resolves
 * every problem definition (material, penalties, boundary conditions against the mesh's
 * sets, criteria, solver) and each operation's criterion, without touching the GPU.
 * message (may be NULL) receives the first error, truncated to capacity. */
int plato_app_validate(const char* input_config, const char* operations, const char* base_dir, char* message,
                       int64_t capacity);
/* The deck as parsed, one "name (type) = value" line per parameter, sublists indented;
 * *needed = bytes including the terminator (call with text NULL to size the buffer). */
int plato_deck_to_text(const char* input_config, char* text, int64_t capacity, int64_t* needed);
int plato_app_destroy(plato_app* app);
const char* plato_app_last_error(const plato_app* app);
int plato_app_num_nodes(const plato_app* app, int32_t* num_nodes);
/* MPMD_App::compute (src/Analyze_App.cpp:566-590) */
int plato_app_compute(plato_app* app, const char* operation);
/* MPMD_App::importDataT (src/Analyze_App.hpp:181-195): "Topology" (or "Solution") fields,
 * operation parameters (context = operation name) */
int plato_app_import(plato_app* app, const char* name, int32_t layout, const char* context, const double* data,
                     int64_t count);
/* MPMD_App::exportDataT (src/Analyze_App.hpp:287-312): criterion values and gradients by
 * their ArgumentName, "Topology", state components ("displacement X" / "Y" / "Z",
 * "filtered density") */
int plato_app_export(plato_app* app, const char* name, int32_t layout, double* data, int64_t count);

/* ---- Exodus II mesh files (the reference's "Input Mesh"; src/EngineMesh.cpp,
 * src/OmegaHMesh.cpp) --------------------------------------------------------------------
 * Host-only reader of netCDF classic encodings (CDF-1, CDF-2, CDF-5; a netCDF-4/HDF5 file is
 * refused): coordinates, the 4-node tetrahedral element blocks in order, node sets and side
 * sets with their names (else "nodelist_<id>" / "sideset_<id>").  Indices are 0-based on
 * output; a side becomes its cell and 3 cell-local node ordinals (Exodus tetrahedron sides
 * 1: (1,2,4), 2: (2,3,4), 3: (1,4,3), 4: (1,3,2)).  Call a getter with NULL arrays to size. */
typedef struct plato_mesh_file plato_mesh_file;
int plato_mesh_file_open(const char* path, plato_mesh_file** out);
const char* plato_mesh_file_last_error(void);
int plato_mesh_file_close(plato_mesh_file* m);
int plato_mesh_file_info(const plato_mesh_file* m, int32_t* num_nodes, int32_t* num_cells, int32_t* num_node_sets,
                         int32_t* num_side_sets);
int plato_mesh_file_mesh(const plato_mesh_file* m, double* coords /*[host] 3N*/, int32_t* connectivity /*[host] 4C*/);
int plato_mesh_file_node_set(const plato_mesh_file* m, int32_t index, char* name, int64_t name_capacity,
                             int32_t* nodes, int32_t* count);
int plato_mesh_file_side_set(const plato_mesh_file* m, int32_t index, char* name, int64_t name_capacity,
                             int32_t* cells, int32_t* local_nodes /*3 per face*/, int32_t* count);

/* ---- box mesh generator (host only; stands in for BamG, unit_tests/PlatoTestHelpers.hpp) */
int plato_box_mesh_sizes(int32_t nx, int32_t ny, int32_t nz, int32_t* num_nodes, int32_t* num_cells);
int plato_box_mesh_tet4(int32_t nx, int32_t ny, int32_t nz, double lx, double ly, double lz,
                        double* coords, int32_t* connectivity);
/* face: 0 x-, 1 x+, 2 y-, 3 y+, 4 z-, 5 z+; pass NULL outputs to get the count */
int plato_box_nodeset(int32_t nx, int32_t ny, int32_t nz, int32_t face, int32_t* nodes,
                      int32_t* count);
int plato_box_sideset(int32_t nx, int32_t ny, int32_t nz, int32_t face, int32_t* cells,
                      int32_t* local_nodes, int32_t* count);

#ifdef __cplusplus
}
#endif
#endif /* PLATO_B200_H */
