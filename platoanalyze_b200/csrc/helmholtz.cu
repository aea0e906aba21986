// Helmholtz density filter (src/helmholtz): the PDE filter that turns the optimiser's nodal
// density into the filtered density the mechanics sees,
//   R(filtered, control)_a = sum over cells of vol (L^2 grad(filtered) . g_a + N_a (filtered_gp - control_gp))
// with the one-point rule (N_a = 1/4 at the centroid) and vol = |det J| / 6
// (HelmholtzResidual::evaluate, src/helmholtz/HelmholtzResidual.hpp; HelmholtzFlux.hpp,
// FluxDivergence.hpp, AddMassTerm.hpp).  R is linear: R = K filtered - M control with
// K_ab = sum vol (L^2 g_a . g_b + 1/16) and M_ab = sum vol / 16 on the node pattern.
//
// A filter handle is a plato_problem over the mesh (same node graph and SELL pattern as the
// mechanics) with one unknown per node.  K and D = (dR/dcontrol)^T = -M depend on the mesh
// and L only, so both are assembled once per handle (warp per row, deterministic per-slot
// sums in cell order) and kept with their SELL copies and K's Jacobi diagonal.  Every call
// is then SELL SpMVs and, for the two solves, a scalar Jacobi-PCG in FP64 (solver.cu): the
// residual is K filtered + D control, the right-hand side of the solution -D control, the
// chain rule D K^-1 (-dF/dfiltered).
//
// Surface term (evaluate_boundary, src/helmholtz/HelmholtzResidual.hpp:178-241; "Surface
// Length Scale" alpha, default 0): on each face that carries it, with the degree-one triangle
// rule, R_a += alpha L (area / 3) (sum_b filtered_b / 3), i.e. K_ab += alpha L area / 9.
// The reference holds the face's filtered value in a per-cell slot that the faces of one
// cell share; it is per face here.  Faces are few and K is assembled once per handle, so the
// term adds with atomics after the deterministic cell sums.
#include <cmath>

#include "plato_internal.cuh"

namespace plato {

MeshView mesh_view(const plato_problem* h);
GraphView graph_view(const plato_problem* h);
int launch_axpby(plato_problem* h, int64_t n, double a, const double* x, double b, double* y);
int pcg_scalar(plato_problem* h, const double* vals, const double* dinv, const double* b, double* x,
               plato_solve_stats* stats);
int launch_sell1_spmv(plato_problem* h, const double* vals, const double* x, double* y);

namespace {

constexpr int kThreads = 256;

// One value per block of the node pattern, warp per row.  MODE 0: K_ab = sum vol (L^2 g_a.g_b
// + 1/16); MODE 1: (dR/dcontrol)^T, -sum vol / 16.  The row's cells are staged 32 at a time
// (nodes and per-node values), each lane owns a block slot and sums the matching
// contributions in cell order.
template <int MODE>
__global__ void __launch_bounds__(128)
k_helm_rows(MeshView m, GraphView g, double L2, double* __restrict__ entries) {
    __shared__ int32_t nodes_s[4][32][4];
    __shared__ double q_s[4][32][4];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t warps_total = (int64_t)gridDim.x * 4;
    for (int64_t row = blockIdx.x * 4LL + wib; row < g.num_nodes; row += warps_total) {
        const int32_t rs = g.row_map[row], nbk = g.row_map[row + 1] - rs;
        const int32_t ks = g.n2c_ptr[row], ncell = g.n2c_ptr[row + 1] - ks;
        for (int sc = 0; sc < nbk; sc += 32) {
            const int j = sc + lane;
            const int32_t col = j < nbk ? g.cols[rs + j] : -1;
            double acc = 0.0;
            for (int cc = 0; cc < ncell; cc += 32) {
                const int c = cc + lane;
                if (c < ncell) {
                    const int32_t packed = g.n2c[ks + c];
                    const int la = packed & 3;
                    const int4 n = m.conn[packed >> 2];
                    double x[4][3];
                    load_cell_coords(m.coords, n, x);
                    TetGeom<double> G;
                    tet_geometry(x, G);
                    double ga[3];
#pragma unroll
                    for (int d = 0; d < 3; ++d)
                        ga[d] = la == 0 ? G.g[0][d] : la == 1 ? G.g[1][d] : la == 2 ? G.g[2][d] : G.g[3][d];
                    const int ids[4] = {n.x, n.y, n.z, n.w};
#pragma unroll
                    for (int b = 0; b < 4; ++b) {
                        nodes_s[wib][lane][b] = ids[b];
                        q_s[wib][lane][b] =
                            MODE == 0 ? G.vol * (L2 * (ga[0] * G.g[b][0] + ga[1] * G.g[b][1] + ga[2] * G.g[b][2]) + 0.0625)
                                      : -0.0625 * G.vol;
                    }
                }
                __syncwarp();
                const int cnt = min(32, ncell - cc);
                for (int t = 0; t < cnt; ++t)
#pragma unroll
                    for (int b = 0; b < 4; ++b)
                        if (nodes_s[wib][t][b] == col) acc += q_s[wib][t][b];
                __syncwarp();
            }
            if (j < nbk) entries[rs + j] = acc;
        }
    }
}

__device__ __forceinline__ double face_nodes_area(MeshView m, const int32_t* fcell, const int32_t* floc, int64_t f,
                                                  int32_t id[3]) {
    const int4 n = m.conn[fcell[f]];
#pragma unroll
    for (int a = 0; a < 3; ++a) id[a] = node_of(n, floc[3 * f + a]);
    double J[2][3];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int d = 0; d < 3; ++d) J[a][d] = m.coords[3 * (int64_t)id[a] + d] - m.coords[3 * (int64_t)id[2] + d];
    const double J23 = J[0][1] * J[1][2] - J[0][2] * J[1][1];
    const double J31 = J[0][2] * J[1][0] - J[0][0] * J[1][2];
    const double J12 = J[0][0] * J[1][1] - J[0][1] * J[1][0];
    return 0.5 * sqrt(J23 * J23 + J31 * J31 + J12 * J12);
}

// K_ab += aL area / 9 for the node pairs of each surface face (rows sorted: binary search)
__global__ void __launch_bounds__(kThreads)
k_helm_surface_entries(MeshView m, GraphView g, int32_t nfaces, const int32_t* __restrict__ fcell,
                       const int32_t* __restrict__ floc, double aL, double* __restrict__ entries) {
    for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f < nfaces; f += (int64_t)gridDim.x * blockDim.x) {
        int32_t id[3];
        const double v = aL * (face_nodes_area(m, fcell, floc, f, id) / 3.0) / 3.0;
        for (int a = 0; a < 3; ++a) {
            const int32_t rs = g.row_map[id[a]];
            const int32_t n = g.row_map[id[a] + 1] - rs;
            for (int b = 0; b < 3; ++b) {
                int lo = 0, hi = n - 1;
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (g.cols[rs + mid] < id[b]) lo = mid + 1; else hi = mid;
                }
                if (g.cols[rs + lo] == id[b]) atomicAdd(entries + rs + lo, v);
            }
        }
    }
}

// Scalar SELL copy (value of slot k of row 32s+l at ptr_s + 32k + l) and the inverse diagonal
__global__ void k_crs_to_sell1(int32_t N, SellView A, const int32_t* __restrict__ row_map,
                               const int32_t* __restrict__ diag, const double* __restrict__ crs,
                               double* __restrict__ sell, double* __restrict__ dinv) {
    const int64_t nslices = (int64_t(N) + 31) / 32;
    for (int64_t s = blockIdx.x; s < nslices; s += gridDim.x) {
        const int w = A.width[s];
        const int64_t base = A.ptr[s];
        for (int t = threadIdx.x; t < 32 * w; t += blockDim.x) {
            const int k = t >> 5, l = t & 31;
            const int64_t r = 32 * s + l;
            double v = 0.0;
            if (r < N) {
                const int32_t rs = row_map[r], nb = row_map[r + 1] - rs;
                if (k < nb) v = crs[rs + k];
            }
            sell[base + t] = v;
        }
        if (dinv && threadIdx.x < 32 && 32 * s + threadIdx.x < N) {
            const int64_t r = 32 * s + threadIdx.x;
            dinv[r] = 1.0 / crs[diag[r]];
        }
    }
}

}  // namespace

SellView sell_view(const plato_problem* h);

// K and D = (dR/dcontrol)^T = -M, their SELL copies and K's Jacobi diagonal (once per handle)
static int helm_prepare(plato_problem* h) {
    if (h->helm_ready) return PLATO_OK;
    if (!h->helm_K) PLATO_CUDA(h, cudaMalloc(&h->helm_K, sizeof(double) * size_t(h->nblocks)));
    if (!h->helm_D) PLATO_CUDA(h, cudaMalloc(&h->helm_D, sizeof(double) * size_t(h->nblocks)));
    if (!h->helm_sell) PLATO_CUDA(h, cudaMalloc(&h->helm_sell, sizeof(double) * size_t(h->sell.total_slots)));
    if (!h->helm_Dsell) PLATO_CUDA(h, cudaMalloc(&h->helm_Dsell, sizeof(double) * size_t(h->sell.total_slots)));
    if (!h->helm_dinv) PLATO_CUDA(h, cudaMalloc(&h->helm_dinv, sizeof(double) * size_t(h->N)));
    const double L2 = h->helm_length * h->helm_length;
    k_helm_rows<0><<<grid_for(h->N, 4, 148 * 32), 128, 0, h->stream>>>(mesh_view(h), graph_view(h), L2, h->helm_K);
    PLATO_LAUNCH_CHECK(h);
    if (h->helm_nfaces > 0) {
        k_helm_surface_entries<<<grid_for(h->helm_nfaces, kThreads), kThreads, 0, h->stream>>>(
            mesh_view(h), graph_view(h), h->helm_nfaces, h->helm_fcell, h->helm_floc, h->helm_surface * h->helm_length,
            h->helm_K);
        PLATO_LAUNCH_CHECK(h);
    }
    k_crs_to_sell1<<<grid_for(h->sell.nslices, 1, 148 * 16), 256, 0, h->stream>>>(
        h->N, sell_view(h), h->row_map, h->diag, h->helm_K, h->helm_sell, h->helm_dinv);
    PLATO_LAUNCH_CHECK(h);
    k_helm_rows<1><<<grid_for(h->N, 4, 148 * 32), 128, 0, h->stream>>>(mesh_view(h), graph_view(h), 0.0, h->helm_D);
    PLATO_LAUNCH_CHECK(h);
    k_crs_to_sell1<<<grid_for(h->sell.nslices, 1, 148 * 16), 256, 0, h->stream>>>(
        h->N, sell_view(h), h->row_map, h->diag, h->helm_D, h->helm_Dsell, nullptr);
    PLATO_LAUNCH_CHECK(h);
    h->helm_ready = 1;
    return PLATO_OK;
}

}  // namespace plato

using namespace plato;

#define RC(expr)                   \
    do {                           \
        int _rc = (expr);          \
        if (_rc) return _rc;       \
    } while (0)

static int helm_check(plato_problem* h) {
    if (!h) return PLATO_BAD_INPUT;
    if (h->physics != 1) return plato_fail(h, PLATO_BAD_INPUT, "not a Helmholtz filter handle");
    return PLATO_OK;
}

extern "C" {

int plato_create_helmholtz(const plato_helmholtz_desc* desc, plato_problem** out) {
    if (!out) return plato_fail(nullptr, PLATO_BAD_INPUT, "null output handle pointer");
    *out = nullptr;
    if (!desc) return plato_fail(nullptr, PLATO_BAD_INPUT, "null Helmholtz description");
    const double L = desc->length_scale, alpha = desc->surface_length_scale;
    if (!(L > 0.0) || !std::isfinite(L))
        return plato_fail(nullptr, PLATO_BAD_INPUT, "Helmholtz length scale must be a positive finite number");
    if (!(alpha >= 0.0) || !std::isfinite(alpha))
        return plato_fail(nullptr, PLATO_BAD_INPUT, "surface length scale must be a non-negative finite number");
    const int32_t nf = alpha > 0.0 ? desc->num_surface_faces : 0;
    if (nf < 0 || (nf > 0 && (!desc->surface_face_cells || !desc->surface_face_local_nodes)))
        return plato_fail(nullptr, PLATO_BAD_INPUT, "surface term needs face cells and local nodes");
    for (int32_t f = 0; f < nf; ++f) {
        if (desc->surface_face_cells[f] < 0 || desc->surface_face_cells[f] >= desc->mesh.num_cells)
            return plato_fail(nullptr, PLATO_BAD_INPUT, "surface face cell out of range");
        for (int a = 0; a < 3; ++a) {
            const int32_t l = desc->surface_face_local_nodes[3 * int64_t(f) + a];
            if (l < 0 || l > 3) return plato_fail(nullptr, PLATO_BAD_INPUT, "surface face local node ordinal out of range");
        }
    }
    plato_problem_desc d{};
    d.mesh = desc->mesh;
    d.material.youngs_modulus = 1.0;  // the filter has no material; the handle needs valid values
    d.material.poissons_ratio = 0.0;
    d.penalty.exponent = 1.0;
    d.penalty.minimum_value = 0.0;
    d.solver = desc->solver;
    if (d.solver.tolerance == 0.0) d.solver.tolerance = 1e-12;
    if (d.solver.max_iterations == 0) d.solver.max_iterations = 100000;
    d.solver.operator_kind = PLATO_OPERATOR_ASSEMBLED;
    d.solver.precision = PLATO_PRECISION_FP64;
    d.solver.chebyshev_degree = 0;
    d.solver.coarse_cells[0] = d.solver.coarse_cells[1] = d.solver.coarse_cells[2] = 0;
    plato_problem* h = nullptr;
    if (int rc = plato_create(&d, &h)) return rc;
    h->physics = 1;
    h->helm_length = L;
    h->helm_surface = alpha;
    if (nf > 0) {
        cudaError_t e = cudaMalloc(&h->helm_fcell, sizeof(int32_t) * size_t(nf));
        if (e == cudaSuccess) e = cudaMalloc(&h->helm_floc, sizeof(int32_t) * 3 * size_t(nf));
        if (e == cudaSuccess)
            e = cudaMemcpy(h->helm_fcell, desc->surface_face_cells, sizeof(int32_t) * size_t(nf), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(h->helm_floc, desc->surface_face_local_nodes, sizeof(int32_t) * 3 * size_t(nf),
                           cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            const int rc = plato_cuda_fail(nullptr, e, "surface face upload", __FILE__, __LINE__);
            plato_destroy(h);
            return rc;
        }
        h->helm_nfaces = nf;
    }
    *out = h;
    return PLATO_OK;
}

int plato_helmholtz_value(plato_problem* h, const double* filtered, const double* control, double* R) {
    RC(helm_check(h));
    if (!filtered || !control || !R) return plato_fail(h, PLATO_BAD_INPUT, "null device pointer");
    RC(helm_prepare(h));
    // R = K filtered + D control (D = (dR/dcontrol)^T = -M, symmetric)
    RC(launch_sell1_spmv(h, h->helm_sell, filtered, R));
    RC(launch_sell1_spmv(h, h->helm_Dsell, control, h->v_tmp));
    return launch_axpby(h, h->N, 1.0, h->v_tmp, 1.0, R);
}

int plato_helmholtz_gradient_u(plato_problem* h, double* entries) {
    RC(helm_check(h));
    if (!entries) return plato_fail(h, PLATO_BAD_INPUT, "null device pointer");
    RC(helm_prepare(h));
    PLATO_CUDA(h, cudaMemcpyAsync(entries, h->helm_K, sizeof(double) * size_t(h->nblocks), cudaMemcpyDeviceToDevice,
                                  h->stream));
    return PLATO_OK;
}

int plato_helmholtz_gradient_z(plato_problem* h, double* entries) {
    RC(helm_check(h));
    if (!entries) return plato_fail(h, PLATO_BAD_INPUT, "null device pointer");
    RC(helm_prepare(h));
    PLATO_CUDA(h, cudaMemcpyAsync(entries, h->helm_D, sizeof(double) * size_t(h->nblocks), cudaMemcpyDeviceToDevice,
                                  h->stream));
    return PLATO_OK;
}

int plato_helmholtz_solution(plato_problem* h, const double* control, double* filtered, plato_solve_stats* stats) {
    RC(helm_check(h));
    if (!control || !filtered) return plato_fail(h, PLATO_BAD_INPUT, "null device pointer");
    plato_solve_stats local{};
    RC(helm_prepare(h));
    // R = value(0, control) = D control; rhs = -R; solve K filtered = rhs from zero
    RC(launch_sell1_spmv(h, h->helm_Dsell, control, h->v_b));
    RC(launch_axpby(h, h->N, -1.0, h->v_b, 0.0, h->v_b));
    PLATO_CUDA(h, cudaMemsetAsync(filtered, 0, sizeof(double) * size_t(h->N), h->stream));
    return pcg_scalar(h, h->helm_sell, h->helm_dinv, h->v_b, filtered, stats ? stats : &local);
}

int plato_helmholtz_criterion_gradient(plato_problem* h, const double* dfdfiltered, double* dfdcontrol,
                                       plato_solve_stats* stats) {
    RC(helm_check(h));
    if (!dfdfiltered || !dfdcontrol) return plato_fail(h, PLATO_BAD_INPUT, "null device pointer");
    plato_solve_stats local{};
    RC(helm_prepare(h));
    // solve K x = -g, then dfdcontrol = (dR/dcontrol)^T x = D x
    RC(launch_axpby(h, h->N, -1.0, dfdfiltered, 0.0, h->v_b));
    PLATO_CUDA(h, cudaMemsetAsync(h->v_x, 0, sizeof(double) * size_t(h->N), h->stream));
    RC(pcg_scalar(h, h->helm_sell, h->helm_dinv, h->v_b, h->v_x, stats ? stats : &local));
    return launch_sell1_spmv(h, h->helm_Dsell, h->v_x, dfdcontrol);
}

}  // extern "C"
