/*
 * plato_oracle.cpp -- CPU FP64 oracle for the SIMP linear-tet elastostatic path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA library, never part of the
 * product.  Each routine restates the arithmetic of one piece of the Plato Analyze
 * reference (paths are relative to that project) in the same loop order, so that
 * results agree with the reference to rounding.  Where the reference differentiates
 * with Sacado forward AD, the oracle propagates the same derivative components
 * through the same sequence of operations (one "dx" component per pass).
 *
 * Parallelism: OpenMP over cells / node rows.  Scatter-adds use atomics, like the
 * reference's Kokkos::atomic_add, so sums over cells can differ in the last bits from
 * run to run; every comparison in the tests carries a relative tolerance.
 */
#include "plato_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int kNodesPerCell = 4;
constexpr int kDofsPerNode  = 3;
constexpr int kDofsPerCell  = 12;
constexpr int kVoigt        = 6;

/* Voigt index of tensor component (i,j): StressDivergence ctor,
 * src/StressDivergence.hpp:33-48 (diagonal first, then (1,2),(0,2),(0,1)). */
constexpr int kVoigtIndex[3][3] = {{0, 5, 4}, {5, 1, 3}, {4, 3, 2}};

struct CellGeom {
    double g[4][3];  /* basis-function gradients */
    double vol;      /* |det J| * cubature weight */
};

/* Cubature weight of the degree-one simplex rule, src/LinearTetCubRuleDegreeOne.hpp:72-78:
 * start at 1 and divide by 2..dim. */
double cub_weight(int dim) {
    double w = 1.0;
    for (int d = 2; d <= dim; ++d) w /= double(d);
    return w;
}

/* ComputeGradientWorkset<3>, src/ImplicitFunctors.hpp:169-221, followed by
 * "tCellVolume(c) *= tQuadratureWeight" (src/elliptic/ElastostaticResidual.hpp:201-202). */
void cell_geometry(const oracle_problem* P, int32_t c, CellGeom& G) {
    const int32_t* n = P->connectivity + 4 * (int64_t)c;
    auto X = [&](int a, int d) { return P->coords[3 * (int64_t)n[a] + d]; };
    double j11 = X(0, 0) - X(3, 0), j12 = X(1, 0) - X(3, 0), j13 = X(2, 0) - X(3, 0);
    double j21 = X(0, 1) - X(3, 1), j22 = X(1, 1) - X(3, 1), j23 = X(2, 1) - X(3, 1);
    double j31 = X(0, 2) - X(3, 2), j32 = X(1, 2) - X(3, 2), j33 = X(2, 2) - X(3, 2);
    double detj = j11 * j22 * j33 + j12 * j23 * j31 + j13 * j21 * j32
                - j11 * j23 * j32 - j12 * j21 * j33 - j13 * j22 * j31;
    double i11 = (j22 * j33 - j23 * j32) / detj;
    double i12 = (j13 * j32 - j12 * j33) / detj;
    double i13 = (j12 * j23 - j13 * j22) / detj;
    double i21 = (j23 * j31 - j21 * j33) / detj;
    double i22 = (j11 * j33 - j13 * j31) / detj;
    double i23 = (j13 * j21 - j11 * j23) / detj;
    double i31 = (j21 * j32 - j22 * j31) / detj;
    double i32 = (j12 * j31 - j11 * j32) / detj;
    double i33 = (j11 * j22 - j12 * j21) / detj;
    G.vol = std::fabs(detj);
    G.g[0][0] = i11; G.g[0][1] = i12; G.g[0][2] = i13;
    G.g[1][0] = i21; G.g[1][1] = i22; G.g[1][2] = i23;
    G.g[2][0] = i31; G.g[2][1] = i32; G.g[2][2] = i33;
    G.g[3][0] = -(i11 + i21 + i31);
    G.g[3][1] = -(i12 + i22 + i32);
    G.g[3][2] = -(i13 + i23 + i33);
    G.vol *= cub_weight(3);
}

/* IsotropicLinearElasticMaterial<3>, src/IsotropicLinearElasticMaterial.cpp:86-110. */
void material_matrix(const oracle_problem* P, double C[6][6]) {
    std::memset(C, 0, sizeof(double) * 36);
    const double nu = P->poissons_ratio, E = P->youngs_modulus;
    const double coef = E / ((1.0 + nu) * (1.0 - 2.0 * nu));
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) C[i][j] = (i == j) ? coef * (1.0 - nu) : coef * nu;
    for (int i = 3; i < 6; ++i) C[i][i] = 1.0 / 2.0 * coef * (1.0 - 2.0 * nu);
}

/* Strain<3>::operator(), src/Strain.hpp:70-95 (engineering shear strain). */
void strain_of(const CellGeom& G, const double ue[12], double eps[6]) {
    int v = 0;
    for (int d = 0; d < 3; ++d) {
        eps[v] = 0.0;
        for (int a = 0; a < kNodesPerCell; ++a) eps[v] += ue[a * kDofsPerNode + d] * G.g[a][d];
        ++v;
    }
    for (int J = 2; J >= 1; --J)
        for (int I = J - 1; I >= 0; --I) {
            eps[v] = 0.0;
            for (int a = 0; a < kNodesPerCell; ++a)
                eps[v] += (ue[a * kDofsPerNode + J] * G.g[a][I] + ue[a * kDofsPerNode + I] * G.g[a][J]);
            ++v;
        }
}

/* LinearStress::operator(), src/LinearStress.hpp:102-120 (reference strain = 0,
 * src/AbstractLinearStress.hpp:45-62). */
void stress_of(const double C[6][6], const double eps[6], double sig[6]) {
    for (int I = 0; I < kVoigt; ++I) {
        sig[I] = 0.0;
        for (int J = 0; J < kVoigt; ++J) sig[I] += (eps[J] - 0.0) * C[I][J];
    }
}

/* ApplyWeighting cell density, src/ApplyWeighting.hpp:55-60: the mean of the cell's nodal
 * control; with element control (no reference counterpart) the cell's own entry. */
double cell_density(const oracle_problem* P, const double* z, int32_t c, const int32_t* n) {
    if (P->cell_control) return z[c];
    double rho = 0.0;
    for (int a = 0; a < kNodesPerCell; ++a) rho += z[n[a]];
    return rho / kNodesPerCell;
}
/* d rho_c / d z: 1/4 per node of the cell, or 1 for the cell's own entry */
double density_dz(const oracle_problem* P) { return P->cell_control ? 1.0 : 1.0 / kNodesPerCell; }

/* MSIMP::operator(), src/Simp.hpp:130-134. */
double msimp(const oracle_problem* P, double rho) {
    return P->penalty_minimum + ((1.0 - P->penalty_minimum) * std::pow(rho, P->penalty_exponent));
}
/* d MSIMP / d rho (what Sacado propagates through pow). */
double msimp_dx(const oracle_problem* P, double rho) {
    const double p = P->penalty_exponent;
    return (1.0 - P->penalty_minimum) * (p * std::pow(rho, p - 1.0));
}

/* StressDivergence<3>::operator(), src/StressDivergence.hpp:70-90 (accumulates). */
void divergence_add(const CellGeom& G, const double sig[6], double out[12], double scale = 1.0) {
    for (int i = 0; i < 3; ++i)
        for (int a = 0; a < kNodesPerCell; ++a) {
            const int local = a * kDofsPerNode + i;
            for (int j = 0; j < 3; ++j) out[local] += scale * G.vol * sig[kVoigtIndex[i][j]] * G.g[a][j];
        }
}

void gather_cell_state(const double* u, const int32_t* n, double ue[12]) {
    for (int a = 0; a < kNodesPerCell; ++a)
        for (int d = 0; d < kDofsPerNode; ++d) ue[a * 3 + d] = u[3 * (int64_t)n[a] + d];
}

inline void atomic_add(double* p, double v) {
#pragma omp atomic
    *p += v;
}

/* Element residual of ElastostaticResidual::evaluate, src/elliptic/ElastostaticResidual.hpp:
 * 165-234: gradient, strain, stress ("Cauchy stress" kernel), then weighting and stress
 * divergence ("Apply weighting and compute divergence" kernel). */
void cell_residual(const oracle_problem* P, const double C[6][6], int32_t c, const double* u,
                   const double* z, double out[12]) {
    CellGeom G;
    cell_geometry(P, c, G);
    const int32_t* n = P->connectivity + 4 * (int64_t)c;
    double ue[12], eps[6], sig[6];
    gather_cell_state(u, n, ue);
    strain_of(G, ue, eps);
    stress_of(C, eps, sig);
    const double s = msimp(P, cell_density(P, z, c, n));
    for (int v = 0; v < kVoigt; ++v) sig[v] *= s;
    for (int k = 0; k < 12; ++k) out[k] = 0.0;
    divergence_add(G, sig, out);
}

/* Element stiffness as Sacado SFad<double,12> computes it: seeding du_j/du_j = 1
 * (src/Assembly.hpp:858-935) and pushing the j-th derivative component through
 * strain, stress, weighting and divergence.  Column j of Ke is R_e.dx(j). */
void cell_stiffness(const oracle_problem* P, const double C[6][6], int32_t c, const double* z,
                    double Ke[12][12]) {
    CellGeom G;
    cell_geometry(P, c, G);
    const int32_t* n = P->connectivity + 4 * (int64_t)c;
    const double s = msimp(P, cell_density(P, z, c, n));
    for (int j = 0; j < kDofsPerCell; ++j) {
        double seed[12] = {0};
        seed[j] = 1.0;
        double eps[6], sig[6], col[12] = {0};
        strain_of(G, seed, eps);
        stress_of(C, eps, sig);
        for (int v = 0; v < kVoigt; ++v) sig[v] *= s;
        divergence_add(G, sig, col);
        for (int i = 0; i < kDofsPerCell; ++i) Ke[i][j] = col[i];
    }
}

/* BlockMatrixEntryOrdinal, src/ImplicitFunctors.hpp:730-766: linear search of the
 * row for the column node. */
int64_t block_entry(const int32_t* row_map, const int32_t* cols, int32_t row_node, int32_t col_node) {
    for (int32_t e = row_map[row_node]; e < row_map[row_node + 1]; ++e)
        if (cols[e] == col_node) return e;
    return -1;
}

/* SurfaceLoadIntegral<3>::operator() with scale -1, src/SurfaceLoadIntegral.hpp:97-150;
 * CalculateSurfaceJacobians<3> src/SurfaceIntegralUtilities.hpp:100-117;
 * CalculateSurfaceArea<3> src/SurfaceIntegralUtilities.hpp:217-227.  Adds into R. */
void add_boundary_load(const oracle_problem* P, double* R, double scale) {
    const double cub = cub_weight(2);
    const double c0 = 1.0 / 3.0, c1 = 1.0 / 3.0;  /* face cubature point (1/3,1/3) */
    const double basis[3] = {1.0 - c0 - c1, c0, c1};
    const double mult = scale * cub;
#pragma omp parallel for schedule(static)
    for (int32_t f = 0; f < P->num_traction_faces; ++f) {
        const int32_t c = P->face_cells[f];
        const int32_t* loc = P->face_local_nodes + 3 * (int64_t)f;
        const int32_t* n = P->connectivity + 4 * (int64_t)c;
        double J[2][3];
        for (int a = 0; a < 2; ++a)
            for (int d = 0; d < 3; ++d)
                J[a][d] = P->coords[3 * (int64_t)n[loc[a]] + d] - P->coords[3 * (int64_t)n[loc[2]] + d];
        double J23 = J[0][1] * J[1][2] - J[0][2] * J[1][1];
        double J31 = J[0][2] * J[1][0] - J[0][0] * J[1][2];
        double J12 = J[0][0] * J[1][1] - J[0][1] * J[1][0];
        double area = mult * std::sqrt(J23 * J23 + J31 * J31 + J12 * J12);
        for (int a = 0; a < 3; ++a)
            for (int d = 0; d < 3; ++d)
                atomic_add(&R[3 * (int64_t)n[loc[a]] + d], basis[a] * P->traction[d] * area);
    }
}

/* Zeroes a block matrix row by row with the static row partition the solver's passes use
 * (first-touch page placement then matches the threads that stream the rows). */
void zero_rows(int32_t N, const int32_t* row_map, int per_block, double* entries) {
#pragma omp parallel for schedule(static)
    for (int32_t r = 0; r < N; ++r)
        std::fill(entries + (int64_t)per_block * row_map[r], entries + (int64_t)per_block * row_map[r + 1], 0.0);
}

}  // namespace

extern "C" {

void oracle_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int oracle_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void oracle_cell_fields(const oracle_problem* P, const double* u, double* grad, double* volume,
                        double* strain, double* stress, double* cell_result) {
    double C[6][6];
    material_matrix(P, C);
#pragma omp parallel for schedule(static)
    for (int32_t c = 0; c < P->num_cells; ++c) {
        CellGeom G;
        cell_geometry(P, c, G);
        const int32_t* n = P->connectivity + 4 * (int64_t)c;
        double ue[12], eps[6], sig[6], res[12] = {0};
        gather_cell_state(u, n, ue);
        strain_of(G, ue, eps);
        stress_of(C, eps, sig);
        divergence_add(G, sig, res);
        if (grad)
            for (int a = 0; a < 4; ++a)
                for (int d = 0; d < 3; ++d) grad[12 * (int64_t)c + 3 * a + d] = G.g[a][d];
        if (volume) volume[c] = G.vol;
        if (strain) std::memcpy(strain + 6 * (int64_t)c, eps, sizeof eps);
        if (stress) std::memcpy(stress + 6 * (int64_t)c, sig, sizeof sig);
        if (cell_result) std::memcpy(cell_result + 12 * (int64_t)c, res, sizeof res);
    }
}

/* EngineMesh::createNodeNodeGraph, src/EngineMesh.cpp:223-320 (unique neighbours,
 * self excluded, sorted) followed by CreateBlockMatrix, src/ImplicitFunctors.hpp:
 * 932-1005 (diagonal inserted in front of the first larger column). */
static void build_graph(const oracle_problem* P, std::vector<int32_t>& row_map,
                        std::vector<int32_t>& cols) {
    const int32_t N = P->num_nodes;
    std::vector<int32_t> elem_count(N + 1, 0);
    for (int64_t k = 0; k < 4 * (int64_t)P->num_cells; ++k) elem_count[P->connectivity[k] + 1]++;
    for (int32_t i = 0; i < N; ++i) elem_count[i + 1] += elem_count[i];
    std::vector<int32_t> node_elems(elem_count[N]);
    {
        std::vector<int32_t> fill(elem_count.begin(), elem_count.end() - 1);
        for (int32_t c = 0; c < P->num_cells; ++c)
            for (int a = 0; a < 4; ++a) node_elems[fill[P->connectivity[4 * (int64_t)c + a]]++] = c;
    }
    std::vector<std::vector<int32_t>> neigh(N);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int32_t i = 0; i < N; ++i) {
        std::vector<int32_t>& nb = neigh[i];
        for (int32_t e = elem_count[i]; e < elem_count[i + 1]; ++e) {
            const int32_t* n = P->connectivity + 4 * (int64_t)node_elems[e];
            for (int a = 0; a < 4; ++a)
                if (n[a] != i && std::find(nb.begin(), nb.end(), n[a]) == nb.end()) nb.push_back(n[a]);
        }
        std::sort(nb.begin(), nb.end());
    }
    row_map.assign(N + 1, 0);
    for (int32_t i = 0; i < N; ++i) row_map[i + 1] = row_map[i] + (int32_t)neigh[i].size() + 1;
    cols.resize(row_map[N]);
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < N; ++i) {
        int32_t out = row_map[i];
        bool diag_done = false;
        for (int32_t c : neigh[i]) {
            if (!diag_done && c > i) { cols[out++] = i; diag_done = true; }
            cols[out++] = c;
        }
        if (!diag_done) cols[out++] = i;
    }
}

int64_t oracle_graph_nnz(const oracle_problem* P) {
    std::vector<int32_t> rm, cols;
    build_graph(P, rm, cols);
    return (int64_t)cols.size();
}

void oracle_graph(const oracle_problem* P, int32_t* row_map, int32_t* column_indices) {
    std::vector<int32_t> rm, cols;
    build_graph(P, rm, cols);
    std::memcpy(row_map, rm.data(), rm.size() * sizeof(int32_t));
    std::memcpy(column_indices, cols.data(), cols.size() * sizeof(int32_t));
}

/* VectorFunction::value, src/elliptic/VectorFunction.hpp:251-334: domain cells are
 * evaluated and assembled (assemble_residual, src/Assembly.hpp:1222-1281), then the
 * boundary term (evaluate_boundary with scale -1, ElastostaticResidual.hpp:248-262). */
void oracle_vf_value(const oracle_problem* P, const double* u, const double* z, double* R) {
    double C[6][6];
    material_matrix(P, C);
    const int64_t n = 3 * (int64_t)P->num_nodes;
    std::fill(R, R + n, 0.0);
#pragma omp parallel for schedule(static)
    for (int32_t c = 0; c < P->num_cells; ++c) {
        double out[12];
        cell_residual(P, C, c, u, z, out);
        const int32_t* nd = P->connectivity + 4 * (int64_t)c;
        for (int a = 0; a < 4; ++a)
            for (int d = 0; d < 3; ++d) atomic_add(&R[3 * (int64_t)nd[a] + d], out[3 * a + d]);
    }
    add_boundary_load(P, R, -1.0);
}

/* VectorFunction::gradient_u, src/elliptic/VectorFunction.hpp:525-615, assembled by
 * assemble_jacobian_fad (src/Assembly.hpp:1374-1438) with BlockMatrixEntryOrdinal. */
void oracle_vf_gradient_u(const oracle_problem* P, const double* u, const double* z,
                          const int32_t* row_map, const int32_t* cols, double* entries) {
    (void)u;
    double C[6][6];
    material_matrix(P, C);
    zero_rows(P->num_nodes, row_map, 9, entries);
#pragma omp parallel for schedule(static)
    for (int32_t c = 0; c < P->num_cells; ++c) {
        double Ke[12][12];
        cell_stiffness(P, C, c, z, Ke);
        const int32_t* nd = P->connectivity + 4 * (int64_t)c;
        for (int i = 0; i < 12; ++i)
            for (int j = 0; j < 12; ++j) {
                int64_t e = block_entry(row_map, cols, nd[i / 3], nd[j / 3]);
                atomic_add(&entries[9 * e + 3 * (i % 3) + (j % 3)], Ke[i][j]);
            }
    }
}

/* VectorFunction::gradient_u_T, src/elliptic/VectorFunction.hpp:432-523, with
 * BlockMatrixTransposeEntryOrdinal (src/ImplicitFunctors.hpp:610-647). */
void oracle_vf_gradient_u_T(const oracle_problem* P, const double* u, const double* z,
                            const int32_t* row_map, const int32_t* cols, double* entries) {
    (void)u;
    double C[6][6];
    material_matrix(P, C);
    zero_rows(P->num_nodes, row_map, 9, entries);
#pragma omp parallel for schedule(static)
    for (int32_t c = 0; c < P->num_cells; ++c) {
        double Ke[12][12];
        cell_stiffness(P, C, c, z, Ke);
        const int32_t* nd = P->connectivity + 4 * (int64_t)c;
        for (int i = 0; i < 12; ++i)
            for (int j = 0; j < 12; ++j) {
                int64_t e = block_entry(row_map, cols, nd[j / 3], nd[i / 3]);
                atomic_add(&entries[9 * e + 3 * (j % 3) + (i % 3)], Ke[i][j]);
            }
    }
}

/* VectorFunction::gradient_z, src/elliptic/VectorFunction.hpp:618-710: (dR/dz)^T as an
 * N x 3N block matrix with 1x3 blocks on the node graph, from SFad<double,4> control
 * derivatives (src/elliptic/EllipticSimplexFadTypes.hpp:22-70), assembled by
 * assemble_transpose_jacobian (src/Assembly.hpp:1455-1521). */
void oracle_vf_gradient_z(const oracle_problem* P, const double* u, const double* z,
                          const int32_t* row_map, const int32_t* cols, double* entries) {
    double C[6][6];
    material_matrix(P, C);
    zero_rows(P->num_nodes, row_map, 3, entries);
#pragma omp parallel for schedule(static)
    for (int32_t c = 0; c < P->num_cells; ++c) {
        CellGeom G;
        cell_geometry(P, c, G);
        const int32_t* nd = P->connectivity + 4 * (int64_t)c;
        double ue[12], eps[6], sig[6];
        gather_cell_state(u, nd, ue);
        strain_of(G, ue, eps);
        stress_of(C, eps, sig);
        /* cell density rho = sum(z)/4 has d rho/d z_k = 1/4 for every local node k */
        const double sdx = msimp_dx(P, cell_density(P, z, c, nd)) * density_dz(P);
        double dsig[6], dres[12] = {0};
        for (int v = 0; v < 6; ++v) dsig[v] = sig[v] * sdx;
        divergence_add(G, dsig, dres);
        for (int i = 0; i < 12; ++i)        /* residual row (state dof) */
            for (int k = 0; k < 4; ++k) {   /* control node */
                int64_t e = block_entry(row_map, cols, nd[k], nd[i / 3]);
                atomic_add(&entries[3 * e + (i % 3)], dres[i]);
            }
    }
}

/* InternalElasticEnergy::evaluate, src/elliptic/InternalElasticEnergy.hpp:132-199 with
 * ScalarProduct (src/ScalarProduct.hpp:26-41, scale 0.5), summed by local_result_sum
 * (src/Assembly.hpp:20-33) in PhysicsScalarFunction::value
 * (src/elliptic/PhysicsScalarFunction.hpp:226-289). */
double oracle_sf_value(const oracle_problem* P, const double* u, const double* z) {
    double C[6][6];
    material_matrix(P, C);
    double total = 0.0;
#pragma omp parallel for reduction(+ : total) schedule(static)
    for (int32_t c = 0; c < P->num_cells; ++c) {
        CellGeom G;
        cell_geometry(P, c, G);
        const int32_t* nd = P->connectivity + 4 * (int64_t)c;
        double ue[12], eps[6], sig[6];
        gather_cell_state(u, nd, ue);
        strain_of(G, ue, eps);
        stress_of(C, eps, sig);
        const double s = msimp(P, cell_density(P, z, c, nd));
        for (int v = 0; v < 6; ++v) sig[v] *= s;
        double inc = 0.0;
        for (int v = 0; v < 6; ++v) inc += sig[v] * eps[v];
        total += 0.5 * inc * G.vol;
    }
    return total;
}

/* PhysicsScalarFunction::gradient_u, src/elliptic/PhysicsScalarFunction.hpp:365-428:
 * SFad<12> state derivative of the cell energy, scattered per dof. */
void oracle_sf_gradient_u(const oracle_problem* P, const double* u, const double* z, double* dfdu) {
    double C[6][6];
    material_matrix(P, C);
    std::fill(dfdu, dfdu + 3 * (int64_t)P->num_nodes, 0.0);
#pragma omp parallel for schedule(static)
    for (int32_t c = 0; c < P->num_cells; ++c) {
        CellGeom G;
        cell_geometry(P, c, G);
        const int32_t* nd = P->connectivity + 4 * (int64_t)c;
        double ue[12], eps[6], sig[6];
        gather_cell_state(u, nd, ue);
        strain_of(G, ue, eps);
        stress_of(C, eps, sig);
        const double s = msimp(P, cell_density(P, z, c, nd));
        for (int v = 0; v < 6; ++v) sig[v] *= s;
        for (int j = 0; j < 12; ++j) {
            double seed[12] = {0};
            seed[j] = 1.0;
            double deps[6], dsig[6];
            strain_of(G, seed, deps);
            stress_of(C, deps, dsig);
            for (int v = 0; v < 6; ++v) dsig[v] *= s;
            double dinc = 0.0;  /* d(sig . eps) = sig.val*eps.dx + sig.dx*eps.val */
            for (int v = 0; v < 6; ++v) dinc += sig[v] * deps[v] + dsig[v] * eps[v];
            atomic_add(&dfdu[3 * (int64_t)nd[j / 3] + j % 3], 0.5 * dinc * G.vol);
        }
    }
}

/* PhysicsScalarFunction::gradient_z, src/elliptic/PhysicsScalarFunction.hpp:432-495, with
 * assemble_scalar_gradient_fad (src/Assembly.hpp:592-627). */
void oracle_sf_gradient_z(const oracle_problem* P, const double* u, const double* z, double* dfdz) {
    double C[6][6];
    material_matrix(P, C);
    std::fill(dfdz, dfdz + (int64_t)(P->cell_control ? P->num_cells : P->num_nodes), 0.0);
#pragma omp parallel for schedule(static)
    for (int32_t c = 0; c < P->num_cells; ++c) {
        CellGeom G;
        cell_geometry(P, c, G);
        const int32_t* nd = P->connectivity + 4 * (int64_t)c;
        double ue[12], eps[6], sig[6];
        gather_cell_state(u, nd, ue);
        strain_of(G, ue, eps);
        stress_of(C, eps, sig);
        const double sdx = msimp_dx(P, cell_density(P, z, c, nd)) * density_dz(P);
        double dinc = 0.0;
        for (int v = 0; v < 6; ++v) dinc += (sig[v] * sdx) * eps[v];
        const double val = 0.5 * dinc * G.vol;
        if (P->cell_control) dfdz[c] = val;
        else
            for (int k = 0; k < 4; ++k) atomic_add(&dfdz[nd[k]], val);
    }
}

/* Geometric Volume criterion, src/geometric/Volume.hpp:83-110: ComputeCellVolume<3>
 * (src/ImplicitFunctors.hpp:292-315, |det J|) times the cubature weight, weighted by the
 * criterion's penalty of the cell density (ApplyWeighting); summed over cells.  The gradient
 * is the SFad<4> control derivative vol * s'(rho) * 1/4 scattered to the cell's nodes. */
static double cell_volume(const oracle_problem* P, int32_t c) {
    const int32_t* n = P->connectivity + 4 * (int64_t)c;
    auto X = [&](int a, int d) { return P->coords[3 * (int64_t)n[a] + d]; };
    double j11 = X(0, 0) - X(3, 0), j12 = X(1, 0) - X(3, 0), j13 = X(2, 0) - X(3, 0);
    double j21 = X(0, 1) - X(3, 1), j22 = X(1, 1) - X(3, 1), j23 = X(2, 1) - X(3, 1);
    double j31 = X(0, 2) - X(3, 2), j32 = X(1, 2) - X(3, 2), j33 = X(2, 2) - X(3, 2);
    double detj = j11 * j22 * j33 + j12 * j23 * j31 + j13 * j21 * j32
                - j11 * j23 * j32 - j12 * j21 * j33 - j13 * j22 * j31;
    return std::fabs(detj) * cub_weight(3);
}

double oracle_volume_value(const oracle_problem* P, const double* z, double p, double m) {
    oracle_problem Q = *P;
    Q.penalty_exponent = p;
    Q.penalty_minimum = m;
    double total = 0.0;
#pragma omp parallel for reduction(+ : total) schedule(static)
    for (int32_t c = 0; c < P->num_cells; ++c) {
        double v = cell_volume(P, c);
        v *= msimp(&Q, cell_density(P, z, c, P->connectivity + 4 * (int64_t)c));
        total += v;
    }
    return total;
}

void oracle_volume_gradient_z(const oracle_problem* P, const double* z, double p, double m, double* dvdz) {
    oracle_problem Q = *P;
    Q.penalty_exponent = p;
    Q.penalty_minimum = m;
    std::fill(dvdz, dvdz + (int64_t)(P->cell_control ? P->num_cells : P->num_nodes), 0.0);
#pragma omp parallel for schedule(static)
    for (int32_t c = 0; c < P->num_cells; ++c) {
        const int32_t* nd = P->connectivity + 4 * (int64_t)c;
        const double val = cell_volume(P, c) * (msimp_dx(&Q, cell_density(P, z, c, nd)) * density_dz(P));
        if (P->cell_control) dvdz[c] = val;
        else
            for (int k = 0; k < 4; ++k) atomic_add(&dvdz[nd[k]], val);
    }
}

/* applyBlockConstraints<3>, src/ApplyConstraints.hpp:40-112 (both loops). */
void oracle_apply_block_constraints(int32_t num_node_rows, const int32_t* row_map,
                                    const int32_t* cols, double* entries, double* rhs,
                                    int32_t num_bc, const int32_t* bc_dofs, const double* bc_values,
                                    double scale) {
    (void)num_node_rows;
    const int B = 3;
    for (int32_t b = 0; b < num_bc; ++b) {
        const int32_t row_dof = bc_dofs[b];
        const double value = scale * bc_values[b];
        const int32_t row_node = row_dof / B, local_row = row_dof % B;
        for (int32_t off = row_map[row_node]; off < row_map[row_node + 1]; ++off)
            for (int lc = 0; lc < B; ++lc) {
                const int32_t col_node = cols[off];
                const int64_t e = (int64_t)B * B * off + B * local_row + lc;
                const int32_t col_dof = B * col_node + lc;
                if (col_dof == row_dof) {
                    entries[e] = 1.0;
                } else {
                    rhs[col_dof] += -entries[e] * value;
                    entries[e] = 0.0;
                    for (int32_t off2 = row_map[col_node]; off2 < row_map[col_node + 1]; ++off2) {
                        const int32_t cr_node = cols[off2];
                        const int64_t e2 = (int64_t)B * B * off2 + B * lc + local_row;
                        if (B * cr_node + local_row == row_dof) entries[e2] = 0.0;
                    }
                }
            }
    }
    for (int32_t b = 0; b < num_bc; ++b) rhs[bc_dofs[b]] = scale * bc_values[b];
}

/* MatrixTimesVectorPlusVector (block branch), src/PlatoMathHelpers.hpp:78-159. */
void oracle_matvec_plus(int32_t num_node_rows, int32_t rb, int32_t cb, const int32_t* row_map,
                        const int32_t* cols, const double* entries, const double* x, double* y) {
#pragma omp parallel for schedule(static)
    for (int32_t r = 0; r < num_node_rows; ++r)
        for (int32_t k = row_map[r]; k < row_map[r + 1]; ++k) {
            int64_t e = (int64_t)rb * cb * k;
            for (int32_t i = 0; i < rb; ++i) {
                double sum = 0.0;
                for (int32_t j = 0; j < cb; ++j) sum += entries[e++] * x[(int64_t)cb * cols[k] + j];
                y[(int64_t)rb * r + i] += sum;
            }
        }
}

}  // extern "C"

/* Jacobi-preconditioned CG.  The reference hands the solve to third-party back ends
 * (src/alg/PlatoAbstractSolver.hpp:38-106); this is the textbook method (Hestenes-
 * Stiefel CG with M = diag(A)), FP64 throughout, stopping when the iterated residual meets
 * ||r_k||/||b|| <= tol (AztecOO's AZ_r0 test) and then confirming with the recomputed
 * residual b - A x: the solve converges only when that true residual meets tol.  When the
 * recurrence has drifted from it (thousands of iterations), CG restarts from the current
 * iterate with a fresh direction, at most kMaxRestarts times.
 *
 * Two fused passes per iteration over the vectors, parallel over node rows with one static
 * partition for every pass (so each thread touches the same rows, and first-touch page
 * placement follows it): (A) p = z + beta p_old formed at every gathered column, Ap = A p
 * and p.Ap; (B) x += alpha p, r -= alpha Ap, z = Dinv r, r.r and r.z. */
namespace {

constexpr int kMaxRestarts = 8;

template <int D>
struct PcgWork {
    int64_t n;
    std::vector<double> dinv, r, zv, p0, p1, Ap;
    explicit PcgWork(int32_t N) : n(D * (int64_t)N) {
        for (auto* v : {&dinv, &r, &zv, &p0, &p1, &Ap}) v->resize(n);
    }
};

/* y = A x, parallel over rows. */
template <int D>
void spmv_rows(int32_t N, const int32_t* row_map, const int32_t* cols, const double* A, const double* x, double* y) {
#pragma omp parallel for schedule(static)
    for (int32_t r = 0; r < N; ++r) {
        double acc[D] = {};
        for (int32_t k = row_map[r]; k < row_map[r + 1]; ++k) {
            const double* blk = A + (int64_t)D * D * k;
            const double* xv = x + (int64_t)D * cols[k];
            for (int i = 0; i < D; ++i)
                for (int j = 0; j < D; ++j) acc[i] += blk[D * i + j] * xv[j];
        }
        for (int i = 0; i < D; ++i) y[(int64_t)D * r + i] = acc[i];
    }
}

/* pass A: pn = z + beta po (own rows), Ap = A pn with pn formed at each gathered column; p.Ap */
template <int D>
double pass_direction_apply(int32_t N, const int32_t* row_map, const int32_t* cols, const double* A,
                            const double* z, const double* po, double beta, double* pn, double* Ap) {
    double pAp = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : pAp)
    for (int32_t r = 0; r < N; ++r) {
        double acc[D] = {};
        for (int32_t k = row_map[r]; k < row_map[r + 1]; ++k) {
            const double* blk = A + (int64_t)D * D * k;
            const int64_t c = (int64_t)D * cols[k];
            double pc[D];
            for (int j = 0; j < D; ++j) pc[j] = z[c + j] + beta * po[c + j];
            for (int i = 0; i < D; ++i)
                for (int j = 0; j < D; ++j) acc[i] += blk[D * i + j] * pc[j];
        }
        for (int i = 0; i < D; ++i) {
            const int64_t q = (int64_t)D * r + i;
            const double pv = z[q] + beta * po[q];
            pn[q] = pv;
            Ap[q] = acc[i];
            pAp += pv * acc[i];
        }
    }
    return pAp;
}

/* x = 0 start, or the residual of a given x: r = b - A x, z = Dinv r, p_old = 0; r.r, r.z */
template <int D>
void pass_residual(int32_t N, const int32_t* row_map, const int32_t* cols, const double* A, const double* b,
                   const double* x, PcgWork<D>& w, double* rr, double* rz) {
    spmv_rows<D>(N, row_map, cols, A, x, w.Ap.data());
    double s_rr = 0.0, s_rz = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : s_rr, s_rz)
    for (int32_t r = 0; r < N; ++r)
        for (int i = 0; i < D; ++i) {
            const int64_t q = (int64_t)D * r + i;
            const double rv = b[q] - w.Ap[q];
            w.r[q] = rv;
            w.zv[q] = w.dinv[q] * rv;
            w.p0[q] = 0.0;
            s_rr += rv * rv;
            s_rz += rv * w.zv[q];
        }
    *rr = s_rr;
    *rz = s_rz;
}

template <int D>
int pcg_jacobi(int32_t N, const int32_t* row_map, const int32_t* cols, const double* A, const double* b, double* x,
               double tol, int32_t max_it, oracle_solve_stats* st) {
    PcgWork<D> w(N);
    double bb = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : bb)
    for (int32_t i = 0; i < N; ++i) {
        int64_t e = block_entry(row_map, cols, i, i);
        for (int d = 0; d < D; ++d) {
            const int64_t q = (int64_t)D * i + d;
            w.dinv[q] = 1.0 / A[(int64_t)D * D * e + (D + 1) * d];
            bb += b[q] * b[q];
        }
    }
    const double bnorm = std::sqrt(bb);
    st->iterations = 0;
    st->converged = 0;
    if (bnorm == 0.0) {
        std::fill(x, x + w.n, 0.0);
        st->relative_residual = 0.0;
        st->converged = 1;
        return 0;
    }
    double rr = 0.0, rz = 0.0;
    pass_residual<D>(N, row_map, cols, A, b, x, w, &rr, &rz);
    int32_t it = 0, restarts = 0;
    double true_rel = std::sqrt(rr) / bnorm;
    double* po = w.p0.data();
    double* pn = w.p1.data();
    for (;;) {
        double beta = 0.0;
        while (it < max_it && std::sqrt(rr) / bnorm > tol) {
            const double pAp = pass_direction_apply<D>(N, row_map, cols, A, w.zv.data(), po, beta, pn, w.Ap.data());
            if (!(pAp > 0.0) || !std::isfinite(pAp)) break;
            const double alpha = rz / pAp;
            double s_rr = 0.0, s_rz = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : s_rr, s_rz)
            for (int32_t r = 0; r < N; ++r)
                for (int i = 0; i < D; ++i) {
                    const int64_t q = (int64_t)D * r + i;
                    x[q] += alpha * pn[q];
                    const double rv = w.r[q] - alpha * w.Ap[q];
                    w.r[q] = rv;
                    const double zq = w.dinv[q] * rv;
                    w.zv[q] = zq;
                    s_rr += rv * rv;
                    s_rz += rv * zq;
                }
            ++it;
            beta = s_rz / rz;
            rr = s_rr;
            rz = s_rz;
            std::swap(po, pn);
        }
        pass_residual<D>(N, row_map, cols, A, b, x, w, &rr, &rz);
        po = w.p0.data();
        pn = w.p1.data();
        true_rel = std::sqrt(rr) / bnorm;
        if (true_rel <= tol || it >= max_it || restarts >= kMaxRestarts || !std::isfinite(true_rel)) break;
        ++restarts;
    }
    st->iterations = it;
    st->relative_residual = true_rel;
    st->converged = true_rel <= tol ? 1 : 0;
    return st->converged ? 0 : 1;
}

}  // namespace

extern "C" {

static int pcg_jacobi_dpn(int32_t N, int dpn, const int32_t* row_map, const int32_t* cols, const double* A,
                          const double* b, double* x, double tol, int32_t max_it, oracle_solve_stats* st) {
    return dpn == 1 ? pcg_jacobi<1>(N, row_map, cols, A, b, x, tol, max_it, st)
                    : pcg_jacobi<3>(N, row_map, cols, A, b, x, tol, max_it, st);
}

int oracle_pcg_jacobi(int32_t N, const int32_t* row_map, const int32_t* cols, const double* A,
                      const double* b, double* x, double tol, int32_t max_it, oracle_solve_stats* st) {
    return pcg_jacobi_dpn(N, 3, row_map, cols, A, b, x, tol, max_it, st);
}

/* Iterative refinement with an extended-precision iterate: u (long double, 64-bit
 * mantissa) holds the solution, r = b - A u is evaluated in long double, and each
 * correction A d = r is solved by the FP64 Jacobi-PCG above to inner_tol relative to ||r||.
 * An FP64 iterate cannot have a residual much below eps ||A|| ||u|| / ||b|| (rounding u to
 * double alone leaves that much), about 5e-11 on a 3.2M-dof SIMP cantilever; the long
 * double iterate lowers that floor by 2^11, so relative residuals of 1e-13 are reachable.
 * Stops when ||b - A u|| / ||b|| <= tol (long double), after max_rounds corrections, or
 * when a correction fails to reduce the residual. */
int oracle_refine_solution(int32_t N, const int32_t* row_map, const int32_t* cols, const double* A,
                           const double* b, long double* u, double tol, double inner_tol, int32_t max_rounds,
                           int32_t max_it, oracle_solve_stats* st) {
    const int64_t n = 3 * (int64_t)N;
    std::vector<double> rd(n), d(n);
    long double bb = 0.0L;
    for (int64_t i = 0; i < n; ++i) bb += (long double)b[i] * b[i];
    const long double bnorm = std::sqrt(bb);
    auto residual = [&]() -> long double {
        long double tot = 0.0L;
#pragma omp parallel for schedule(static) reduction(+ : tot)
        for (int32_t r = 0; r < N; ++r) {
            long double acc[3] = {0.0L, 0.0L, 0.0L};
            for (int32_t k = row_map[r]; k < row_map[r + 1]; ++k) {
                const double* blk = A + 9 * (int64_t)k;
                const long double* uv = u + 3 * (int64_t)cols[k];
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) acc[i] += (long double)blk[3 * i + j] * uv[j];
            }
            for (int i = 0; i < 3; ++i) {
                const long double rv = (long double)b[3 * (int64_t)r + i] - acc[i];
                rd[3 * (int64_t)r + i] = (double)rv;
                tot += rv * rv;
            }
        }
        return std::sqrt(tot);
    };
    st->iterations = 0;
    st->converged = 0;
    if (bnorm == 0.0L) {
        std::fill(u, u + n, 0.0L);
        st->relative_residual = 0.0;
        st->converged = 1;
        return 0;
    }
    long double rel = residual() / bnorm;
    for (int32_t round = 0; round < max_rounds && rel > tol && std::isfinite((double)rel); ++round) {
        std::fill(d.begin(), d.end(), 0.0);
        oracle_solve_stats inner{};
        pcg_jacobi<3>(N, row_map, cols, A, rd.data(), d.data(), inner_tol, max_it, &inner);
        st->iterations += inner.iterations;
        std::vector<long double> keep(u, u + n);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) u[i] += d[i];
        const long double next = residual() / bnorm;
        if (!(next < rel)) {  // no progress: keep the better iterate
            std::copy(keep.begin(), keep.end(), u);
            residual();
            break;
        }
        rel = next;
    }
    st->relative_residual = (double)rel;
    st->converged = rel <= tol ? 1 : 0;
    return st->converged ? 0 : 1;
}

/* Problem::solution, src/elliptic/Problem.hpp:237-292 (one Newton step):
 * R = value(0, z); R *= -1; J = gradient_u; applyStateConstraints(J, R, 1);
 * solve J d = R; u = 0 + d. */
int oracle_problem_solution(const oracle_problem* P, const double* z, double* u, double tol,
                            int32_t max_it, oracle_solve_stats* st) {
    const int64_t n = 3 * (int64_t)P->num_nodes;
    std::vector<int32_t> rm, cols;
    build_graph(P, rm, cols);
    std::vector<double> zero(n, 0.0), R(n), J(9 * cols.size());
    oracle_vf_value(P, zero.data(), z, R.data());
    for (auto& v : R) v *= -1.0;
    oracle_vf_gradient_u(P, zero.data(), z, rm.data(), cols.data(), J.data());
    oracle_apply_block_constraints(P->num_nodes, rm.data(), cols.data(), J.data(), R.data(),
                                   P->num_bc_dofs, P->bc_dofs, P->bc_values, 1.0);
    std::fill(u, u + n, 0.0);
    return oracle_pcg_jacobi(P->num_nodes, rm.data(), cols.data(), J.data(), R.data(), u, tol, max_it, st);
}

/* Problem::criterionGradient, src/elliptic/Problem.hpp:395-450 (self-adjoint shortcut
 * at :423-427; otherwise adjoint solve with zero-valued constraints, :701-713). */
int oracle_problem_criterion_gradient(const oracle_problem* P, const double* z, const double* u,
                                      int32_t self_adjoint, double tol, int32_t max_it,
                                      double* dfdz, oracle_solve_stats* st) {
    const int64_t n = 3 * (int64_t)P->num_nodes;
    std::vector<int32_t> rm, cols;
    build_graph(P, rm, cols);
    oracle_sf_gradient_z(P, u, z, dfdz);
    std::vector<double> lambda(n, 0.0);
    int rc = 0;
    if (self_adjoint) {
        for (int64_t i = 0; i < n; ++i) lambda[i] = -u[i];
        if (st) { st->iterations = 0; st->relative_residual = 0.0; st->converged = 1; }
    } else {
        std::vector<double> dfdu(n), JT(9 * cols.size());
        oracle_sf_gradient_u(P, u, z, dfdu.data());
        for (auto& v : dfdu) v *= -1.0;
        oracle_vf_gradient_u_T(P, u, z, rm.data(), cols.data(), JT.data());
        std::vector<double> zero_vals(P->num_bc_dofs, 0.0);
        oracle_apply_block_constraints(P->num_nodes, rm.data(), cols.data(), JT.data(), dfdu.data(),
                                       P->num_bc_dofs, P->bc_dofs, zero_vals.data(), 1.0);
        oracle_solve_stats local;
        rc = oracle_pcg_jacobi(P->num_nodes, rm.data(), cols.data(), JT.data(), dfdu.data(),
                               lambda.data(), tol, max_it, st ? st : &local);
    }
    if (P->cell_control) {  /* (dR/dz_c)^T lambda = s'(rho_c) lambda_e . (K_e^0 u_e), per cell */
        double C[6][6];
        material_matrix(P, C);
#pragma omp parallel for schedule(static)
        for (int32_t c = 0; c < P->num_cells; ++c) {
            CellGeom G;
            cell_geometry(P, c, G);
            const int32_t* nd = P->connectivity + 4 * (int64_t)c;
            double ue[12], le[12], eps[6], sig[6], dres[12] = {0};
            gather_cell_state(u, nd, ue);
            gather_cell_state(lambda.data(), nd, le);
            strain_of(G, ue, eps);
            stress_of(C, eps, sig);
            const double sdx = msimp_dx(P, cell_density(P, z, c, nd));
            for (int v = 0; v < 6; ++v) sig[v] *= sdx;
            divergence_add(G, sig, dres);
            double t = 0.0;
            for (int i = 0; i < 12; ++i) t += dres[i] * le[i];
            dfdz[c] += t;
        }
        return rc;
    }
    std::vector<double> dRdz(3 * cols.size());
    oracle_vf_gradient_z(P, u, z, rm.data(), cols.data(), dRdz.data());
    oracle_matvec_plus(P->num_nodes, 1, 3, rm.data(), cols.data(), dRdz.data(), lambda.data(), dfdz);
    return rc;
}

/* ---- Helmholtz density filter (src/helmholtz) ------------------------------------------
 * HelmholtzResidual::evaluate (src/helmholtz/HelmholtzResidual.hpp:103-176): per cell, with
 * the one-point rule (basis functions 1/4 at the centroid) and vol = |det J| / 6: the flux
 * L^2 grad(filtered) (HelmholtzFlux.hpp:32-43) is divided against the basis gradients,
 * R_a += vol (L^2 grad(filtered) . g_a) (FluxDivergence), then the mass term
 * R_a += N_a (filtered_gp - control_gp) vol (AddMassTerm.hpp:35-47). */

/* Triangle area of a face (CalculateSurfaceArea<3>, src/SurfaceIntegralUtilities.hpp:212-227,
 * times the degree-one triangle weight 1/2) and its three global nodes. */
static double face_area(const oracle_problem* P, const oracle_helmholtz* H, int32_t f, int32_t id[3]) {
    const int32_t* n = P->connectivity + 4 * (int64_t)H->face_cells[f];
    for (int a = 0; a < 3; ++a) id[a] = n[H->face_local_nodes[3 * (int64_t)f + a]];
    double J[2][3];
    for (int a = 0; a < 2; ++a)
        for (int d = 0; d < 3; ++d) J[a][d] = P->coords[3 * (int64_t)id[a] + d] - P->coords[3 * (int64_t)id[2] + d];
    const double J23 = J[0][1] * J[1][2] - J[0][2] * J[1][1];
    const double J31 = J[0][2] * J[1][0] - J[0][0] * J[1][2];
    const double J12 = J[0][0] * J[1][1] - J[0][1] * J[1][0];
    return 0.5 * std::sqrt(J23 * J23 + J31 * J31 + J12 * J12);
}

/* evaluate_boundary (src/helmholtz/HelmholtzResidual.hpp:178-241), per face with the
 * degree-one triangle rule (basis 1/3): filtered_face = sum_b filtered_b / 3 and
 * R_a += alpha L filtered_face area / 3 for the face's nodes.  The reference keeps
 * filtered_face in a per-cell slot, shared by the faces of one cell; here it is per face. */
void oracle_helmholtz_value(const oracle_problem* P, const oracle_helmholtz* H, const double* filtered,
                            const double* control, double* R) {
    std::fill(R, R + P->num_nodes, 0.0);
    const double L2 = H->length_scale * H->length_scale;
#pragma omp parallel for schedule(static)
    for (int32_t c = 0; c < P->num_cells; ++c) {
        CellGeom G;
        cell_geometry(P, c, G);
        const int32_t* n = P->connectivity + 4 * (int64_t)c;
        double grad[3] = {0.0, 0.0, 0.0}, fg = 0.0, cg = 0.0;
        for (int a = 0; a < 4; ++a) {
            for (int d = 0; d < 3; ++d) grad[d] += filtered[n[a]] * G.g[a][d];
            fg += 0.25 * filtered[n[a]];
            cg += 0.25 * control[n[a]];
        }
        double flux[3];
        for (int d = 0; d < 3; ++d) flux[d] = L2 * grad[d];
        double out[4] = {0.0, 0.0, 0.0, 0.0};
        for (int a = 0; a < 4; ++a)
            for (int d = 0; d < 3; ++d) out[a] += flux[d] * G.g[a][d] * G.vol;
        for (int a = 0; a < 4; ++a) out[a] += 0.25 * (fg - cg) * G.vol;
        for (int a = 0; a < 4; ++a) atomic_add(&R[n[a]], out[a]);
    }
    if (!(H->surface_length_scale > 0.0)) return;
    const double aL = H->surface_length_scale * H->length_scale;
    for (int32_t f = 0; f < H->num_faces; ++f) {
        int32_t id[3];
        const double area = face_area(P, H, f, id);
        double ff = 0.0;
        for (int b = 0; b < 3; ++b) ff += filtered[id[b]] / 3.0;
        for (int a = 0; a < 3; ++a) R[id[a]] += aL * ff * (area / 3.0);
    }
}

/* VectorFunction::gradient_u (src/helmholtz/VectorFunction.hpp): dR_a/dfiltered_b =
 * vol (L^2 g_a . g_b + 1/16) per cell, plus alpha L area / 9 per surface face. */
void oracle_helmholtz_gradient_u(const oracle_problem* P, const oracle_helmholtz* H, const int32_t* row_map,
                                 const int32_t* cols, double* entries) {
    std::fill(entries, entries + row_map[P->num_nodes], 0.0);
    const double L2 = H->length_scale * H->length_scale;
#pragma omp parallel for schedule(static)
    for (int32_t c = 0; c < P->num_cells; ++c) {
        CellGeom G;
        cell_geometry(P, c, G);
        const int32_t* n = P->connectivity + 4 * (int64_t)c;
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) {
                const double v = G.vol * (L2 * (G.g[a][0] * G.g[b][0] + G.g[a][1] * G.g[b][1] + G.g[a][2] * G.g[b][2]) +
                                          0.0625);
                atomic_add(&entries[block_entry(row_map, cols, n[a], n[b])], v);
            }
    }
    if (!(H->surface_length_scale > 0.0)) return;
    const double aL = H->surface_length_scale * H->length_scale;
    for (int32_t f = 0; f < H->num_faces; ++f) {
        int32_t id[3];
        const double area = face_area(P, H, f, id);
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) entries[block_entry(row_map, cols, id[a], id[b])] += aL * (area / 3.0) / 3.0;
    }
}

/* VectorFunction::gradient_z, transposed as the reference returns it: dR_a/dcontrol_b =
 * -vol / 16 (the mass term; symmetric). */
void oracle_helmholtz_gradient_z(const oracle_problem* P, const int32_t* row_map, const int32_t* cols,
                                 double* entries) {
    std::fill(entries, entries + row_map[P->num_nodes], 0.0);
#pragma omp parallel for schedule(static)
    for (int32_t c = 0; c < P->num_cells; ++c) {
        CellGeom G;
        cell_geometry(P, c, G);
        const int32_t* n = P->connectivity + 4 * (int64_t)c;
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) atomic_add(&entries[block_entry(row_map, cols, n[b], n[a])], -0.0625 * G.vol);
    }
}

/* Helmholtz Problem::solution (src/helmholtz/Problem.hpp:158-176): R = value(0, control),
 * R *= -1, J = gradient_u, solve J filtered = R from zero. */
int oracle_helmholtz_solution(const oracle_problem* P, const oracle_helmholtz* H, const double* control,
                              double* filtered, double tol, int32_t max_it, oracle_solve_stats* st) {
    const int64_t N = P->num_nodes;
    std::vector<int32_t> rm, cols;
    build_graph(P, rm, cols);
    std::vector<double> zero(N, 0.0), R(N), J(cols.size());
    oracle_helmholtz_value(P, H, zero.data(), control, R.data());
    for (auto& v : R) v *= -1.0;
    oracle_helmholtz_gradient_u(P, H, rm.data(), cols.data(), J.data());
    std::fill(filtered, filtered + N, 0.0);
    return pcg_jacobi_dpn(P->num_nodes, 1, rm.data(), cols.data(), J.data(), R.data(), filtered, tol, max_it, st);
}

/* Helmholtz Problem::criterionGradient (src/helmholtz/Problem.hpp:187-208): given the
 * criterion's derivative with respect to the filtered density g, solve J x = -g and return
 * (dR/dcontrol)^T x (= M J^-1 g). */
int oracle_helmholtz_criterion_gradient(const oracle_problem* P, const oracle_helmholtz* H, const double* dfdfiltered,
                                        double* dfdcontrol, double tol, int32_t max_it, oracle_solve_stats* st) {
    const int64_t N = P->num_nodes;
    std::vector<int32_t> rm, cols;
    build_graph(P, rm, cols);
    std::vector<double> J(cols.size()), dRdz(cols.size()), rhs(N), x(N, 0.0);
    oracle_helmholtz_gradient_u(P, H, rm.data(), cols.data(), J.data());
    oracle_helmholtz_gradient_z(P, rm.data(), cols.data(), dRdz.data());
    for (int64_t i = 0; i < N; ++i) rhs[i] = -dfdfiltered[i];
    const int rc = pcg_jacobi_dpn(P->num_nodes, 1, rm.data(), cols.data(), J.data(), rhs.data(), x.data(), tol,
                                  max_it, st);
    std::fill(dfdcontrol, dfdcontrol + N, 0.0);
    oracle_matvec_plus(P->num_nodes, 1, 1, rm.data(), cols.data(), dRdz.data(), x.data(), dfdcontrol);
    return rc;
}

}  // extern "C"
