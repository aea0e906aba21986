/*
 * plato_oracle.h -- CPU FP64 oracle for the SIMP linear-tet elastostatic path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker that the CUDA library is compared
 * against; it is never linked into, called by, or shipped with the product path.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 *
 * It restates, in plain C++ with OpenMP, the arithmetic of Plato Analyze's elliptic
 * mechanics path (file:line citations into the reference are on each function in
 * plato_oracle.cpp).  Its results are pinned against the gold vectors of the
 * reference's own unit tests (unit_tests/DerivativeTests.cpp), see
 * tests/test_oracle_golden.py.
 *
 * Conventions follow the reference: Scalar = double, ordinals = int32
 * (src/PlatoTypes.hpp:15-20); dof = 3*node + dim (src/ImplicitFunctors.hpp:61-62);
 * connectivity cell*4 + k; coordinates node*3 + d; block CRS rowMap over nodes,
 * columnIndices node ids, entries row-major per block.
 */
#ifndef PLATO_ORACLE_H
#define PLATO_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_problem {
    int32_t        num_nodes;
    int32_t        num_cells;
    const double*  coords;            /* num_nodes*3 */
    const int32_t* connectivity;      /* num_cells*4 */
    double         youngs_modulus;
    double         poissons_ratio;
    double         penalty_exponent;  /* MSIMP "Exponent" */
    double         penalty_minimum;   /* MSIMP "Minimum Value" */
    int32_t        num_traction_faces;
    const int32_t* face_cells;        /* owning cell of each face */
    const int32_t* face_local_nodes;  /* 3 cell-local node ordinals per face */
    double         traction[3];       /* uniform traction "Vector" */
    int32_t        num_bc_dofs;
    const int32_t* bc_dofs;
    const double*  bc_values;
    int32_t        cell_control;      /* 0: nodal control (ApplyWeighting mean); 1: one density per
                                         cell, z and dz have num_cells entries */
} oracle_problem;

typedef struct oracle_solve_stats {
    int32_t iterations;
    double  relative_residual;     /* ||b - A x|| / ||b|| recomputed at exit */
    int32_t converged;
} oracle_solve_stats;

/* per-cell intermediates of DerivativeTests.3D: grad (C*4*3), weighted volume (C),
 * strain (C*6), stress (C*6), unweighted cell residual (C*12).  Any output may be NULL. */
void oracle_cell_fields(const oracle_problem* P, const double* u,
                        double* grad, double* volume, double* strain,
                        double* stress, double* cell_result);

/* node-node graph + CreateBlockMatrix pattern (diagonal included). */
int64_t oracle_graph_nnz(const oracle_problem* P);
void    oracle_graph(const oracle_problem* P, int32_t* row_map, int32_t* column_indices);

/* Elliptic::VectorFunction */
void oracle_vf_value(const oracle_problem* P, const double* u, const double* z, double* R);
void oracle_vf_gradient_u(const oracle_problem* P, const double* u, const double* z,
                          const int32_t* row_map, const int32_t* column_indices, double* entries);
void oracle_vf_gradient_u_T(const oracle_problem* P, const double* u, const double* z,
                            const int32_t* row_map, const int32_t* column_indices, double* entries);
void oracle_vf_gradient_z(const oracle_problem* P, const double* u, const double* z,
                          const int32_t* row_map, const int32_t* column_indices, double* entries);

/* Elliptic::PhysicsScalarFunction, "Internal Elastic Energy" */
double oracle_sf_value(const oracle_problem* P, const double* u, const double* z);
void   oracle_sf_gradient_u(const oracle_problem* P, const double* u, const double* z, double* dfdu);
void   oracle_sf_gradient_z(const oracle_problem* P, const double* u, const double* z, double* dfdz);

/* Geometric "Volume" criterion with its own MSIMP penalty (exponent p, minimum m). */
double oracle_volume_value(const oracle_problem* P, const double* z, double p, double m);
void   oracle_volume_gradient_z(const oracle_problem* P, const double* z, double p, double m, double* dvdz);

/* helpers */
void oracle_apply_block_constraints(int32_t num_node_rows, const int32_t* row_map,
                                    const int32_t* column_indices, double* entries, double* rhs,
                                    int32_t num_bc, const int32_t* bc_dofs, const double* bc_values,
                                    double scale);
void oracle_matvec_plus(int32_t num_node_rows, int32_t rows_per_block, int32_t cols_per_block,
                        const int32_t* row_map, const int32_t* column_indices, const double* entries,
                        const double* x, double* y);
/* Iterative refinement of A u = b with a long double iterate u (in/out), long double
 * residuals and FP64 Jacobi-PCG corrections to inner_tol; stops at ||b - A u||/||b|| <= tol.
 * stats->iterations counts the inner iterations, relative_residual is the long double one. */
int oracle_refine_solution(int32_t N, const int32_t* row_map, const int32_t* cols, const double* A,
                           const double* b, long double* u, double tol, double inner_tol, int32_t max_rounds,
                           int32_t max_it, oracle_solve_stats* stats);
int  oracle_pcg_jacobi(int32_t num_node_rows, const int32_t* row_map, const int32_t* column_indices,
                       const double* entries, const double* b, double* x, double tolerance,
                       int32_t max_iterations, oracle_solve_stats* stats);

/* Elliptic::Problem */
int oracle_problem_solution(const oracle_problem* P, const double* z, double* u,
                            double tolerance, int32_t max_iterations, oracle_solve_stats* stats);
int oracle_problem_criterion_gradient(const oracle_problem* P, const double* z, const double* u,
                                      int32_t self_adjoint, double tolerance, int32_t max_iterations,
                                      double* dfdz, oracle_solve_stats* stats);

/* Helmholtz density filter (src/helmholtz): "Length Scale" L, "Surface Length Scale" alpha
 * (0 = no surface term) and the faces that carry it (the exterior faces outside the
 * "Symmetry Plane Sides"; HelmholtzResidual.hpp evaluate_boundary). */
typedef struct oracle_helmholtz {
    double         length_scale;
    double         surface_length_scale;
    int32_t        num_faces;
    const int32_t* face_cells;       /* owning cell of each face */
    const int32_t* face_local_nodes; /* 3 cell-local node ordinals per face */
} oracle_helmholtz;

/* Residual, Jacobian and (dR/dcontrol)^T entries (one value per block of the node pattern),
 * solution, and the chain rule from the filtered to the unfiltered density. */
void oracle_helmholtz_value(const oracle_problem* P, const oracle_helmholtz* H, const double* filtered,
                            const double* control, double* R);
void oracle_helmholtz_gradient_u(const oracle_problem* P, const oracle_helmholtz* H, const int32_t* row_map,
                                 const int32_t* column_indices, double* entries);
void oracle_helmholtz_gradient_z(const oracle_problem* P, const int32_t* row_map, const int32_t* column_indices,
                                 double* entries);
int oracle_helmholtz_solution(const oracle_problem* P, const oracle_helmholtz* H, const double* control,
                              double* filtered, double tolerance, int32_t max_iterations, oracle_solve_stats* stats);
int oracle_helmholtz_criterion_gradient(const oracle_problem* P, const oracle_helmholtz* H, const double* dfdfiltered,
                                        double* dfdcontrol, double tolerance, int32_t max_iterations,
                                        oracle_solve_stats* stats);
int oracle_num_threads(void);
void oracle_set_num_threads(int n); /* OpenMP threads of the later calls (n > 0) */

#ifdef __cplusplus
}
#endif
#endif
