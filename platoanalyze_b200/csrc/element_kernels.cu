// Element kernels of the elastostatic residual, the internal-energy criterion and their
// control derivatives.  Every kernel gathers connectivity (one int4 per cell), nodal
// coordinates, control and state straight from the global arrays (no worksets) and
// recomputes the tet kinematics in registers.
#include <algorithm>

#include "plato_internal.cuh"

namespace plato {
namespace {

constexpr int kThreads = 256;

struct CellState {
    int4   n;
    TetGeom<double> G;
    double rho;  // mean nodal control, ApplyWeighting (src/ApplyWeighting.hpp:55-60)
};

__device__ __forceinline__ void load_cell(const MeshView& m, const Material& mat, const double* __restrict__ z,
                                          int64_t c, CellState& cs) {
    cs.n = m.conn[c];
    double x[4][3];
    load_cell_coords(m.coords, cs.n, x);
    tet_geometry(x, cs.G);
    cs.rho = cell_rho(mat, z, c, cs.n);
}

__device__ __forceinline__ void gather_state(const double* __restrict__ u, int4 n, double ue[4][3]) {
    const int ids[4] = {n.x, n.y, n.z, n.w};
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const double* p = u + 3 * (int64_t)ids[a];
        ue[a][0] = __ldg(p + 0);
        ue[a][1] = __ldg(p + 1);
        ue[a][2] = __ldg(p + 2);
    }
}

// R += K_e(z) u_e over all cells: ElastostaticResidual::evaluate
// (src/elliptic/ElastostaticResidual.hpp:165-234) + assemble_residual
// (src/Assembly.hpp:1222-1281).  Scatter with FP64 atomics into an L2-resident vector.
__global__ void __launch_bounds__(kThreads) k_internal_force(MeshView m, Material mat,
                                                             const double* __restrict__ u,
                                                             const double* __restrict__ z,
                                                             double* __restrict__ R) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < m.num_cells;
         c += (int64_t)gridDim.x * blockDim.x) {
        CellState cs;
        load_cell(m, mat, z, c, cs);
        double ue[4][3], e[6], s[6];
        gather_state(u, cs.n, ue);
        strain_voigt(cs.G.g, ue, e);
        stress_voigt(mat, e, s);
        const double w = cs.G.vol * simp(mat, cs.rho);
        const int ids[4] = {cs.n.x, cs.n.y, cs.n.z, cs.n.w};
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            double f[3];
            divergence_node(cs.G.g[a], s, w, f);
            double* dst = R + 3 * (int64_t)ids[a];
            atomicAdd(dst + 0, f[0]);
            atomicAdd(dst + 1, f[1]);
            atomicAdd(dst + 2, f[2]);
        }
    }
}

// Per-cell strain energy density pieces.  mode 0: cell energy 1/2 vol s(rho) eps.C.eps
// (InternalElasticEnergy::evaluate, src/elliptic/InternalElasticEnergy.hpp:169-192).
// mode 1: its derivative with respect to one nodal control, d/dz_k = 1/2 vol s'(rho)/4 eps.C.eps
// (PhysicsScalarFunction::gradient_z, src/elliptic/PhysicsScalarFunction.hpp:432-495).
// mode 2: compliance sensitivity with the self-adjoint adjoint lambda = -u
// (Problem::criterionGradient, src/elliptic/Problem.hpp:423-448): dfdz + (dR/dz)^T lambda
// = -1/2 vol s'(rho)/4 eps.C.eps per node of the cell.
// mode 3: (dR/dz)^T lambda alone, vol s'(rho)/4 eps(lambda).C.eps(u)
// (VectorFunction::gradient_z, src/elliptic/VectorFunction.hpp:618-710, times lambda).
// mode 4: general adjoint, mode 1 + mode 3.
template <int MODE>
__device__ __forceinline__ double cell_quantity(const MeshView& m, const Material& mat,
                                                const double* __restrict__ u,
                                                const double* __restrict__ z,
                                                const double* __restrict__ lam, int64_t c) {
    CellState cs;
    load_cell(m, mat, z, c, cs);
    double ue[4][3], e[6], s[6];
    gather_state(u, cs.n, ue);
    strain_voigt(cs.G.g, ue, e);
    stress_voigt(mat, e, s);
    const double ese = s[0] * e[0] + s[1] * e[1] + s[2] * e[2] + s[3] * e[3] + s[4] * e[4] + s[5] * e[5];
    if (MODE == 0) return 0.5 * ese * cs.G.vol * simp(mat, cs.rho);
    const double sdx = simp_dx(mat, cs.rho) * rho_dz(mat);
    if (MODE == 1) return 0.5 * ese * cs.G.vol * sdx;
    if (MODE == 2) return -0.5 * ese * cs.G.vol * sdx;
    double le[4][3], el[6];
    gather_state(lam, cs.n, le);
    strain_voigt(cs.G.g, le, el);
    const double esl = s[0] * el[0] + s[1] * el[1] + s[2] * el[2] + s[3] * el[3] + s[4] * el[4] + s[5] * el[5];
    if (MODE == 3) return esl * cs.G.vol * sdx;
    return (0.5 * ese + esl) * cs.G.vol * sdx;
}

// accumulate != 0 adds into out (the element-control gradient goes straight to its output).
template <int MODE>
__global__ void __launch_bounds__(kThreads) k_cell_quantity(MeshView m, Material mat,
                                                            const double* __restrict__ u,
                                                            const double* __restrict__ z,
                                                            const double* __restrict__ lam,
                                                            double* __restrict__ out, int accumulate) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < m.num_cells;
         c += (int64_t)gridDim.x * blockDim.x) {
        const double q = cell_quantity<MODE>(m, mat, u, z, lam, c);
        out[c] = accumulate ? out[c] + q : q;
    }
}

// Nodal sum of a per-cell quantity over the node's incident cells, in incidence order
// (assemble_scalar_gradient_fad, src/Assembly.hpp:592-627, without atomics).
// accumulate != 0 adds into out (MatrixTimesVectorPlusVector semantics).
__global__ void __launch_bounds__(kThreads) k_node_sum(GraphView g, const double* __restrict__ cellval,
                                                       double* __restrict__ out, int accumulate) {
    for (int64_t a = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; a < g.num_nodes;
         a += (int64_t)gridDim.x * blockDim.x) {
        double sum = 0.0;
        for (int32_t k = g.n2c_ptr[a]; k < g.n2c_ptr[a + 1]; ++k) sum += cellval[g.n2c[k] >> 2];
        out[a] = accumulate ? out[a] + sum : sum;
    }
}

// Energy sum with a deterministic two-level reduction: block partials, then the last
// block to finish sums the partials in block order (local_result_sum,
// src/Assembly.hpp:20-33).
__device__ __forceinline__ double block_sum(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x < 32) {
        r = (l < (int)(blockDim.x >> 5)) ? sh[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    __syncthreads();
    return r;  // valid in thread 0
}

__global__ void __launch_bounds__(kThreads, 4) k_energy_sum(MeshView m, Material mat,
                                                         const double* __restrict__ u,
                                                         const double* __restrict__ z,
                                                         double* __restrict__ partials,
                                                         unsigned int* __restrict__ ticket,
                                                         double* __restrict__ result) {
    __shared__ double sh[32];
    __shared__ bool last;
    double v = 0.0;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < m.num_cells;
         c += (int64_t)gridDim.x * blockDim.x)
        v += cell_quantity<0>(m, mat, u, z, nullptr, c);
    v = block_sum(v, sh);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = v;
        __threadfence();
        last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (last) {
        __threadfence();
        double t = 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) t += partials[b];
        t = block_sum(t, sh);
        if (threadIdx.x == 0) {
            *result = t;
            *ticket = 0u;
        }
    }
}

// Compliance and its self-adjoint sensitivity in one pass over the cells (the value and the
// gradient that an MPMD ComputeCriterion operation asks for together, src/Analyze_App.cpp:
// 727-1014): per cell ese = eps.C.eps once; the energy 1/2 vol s(rho) ese is summed as in
// k_energy_sum (block partials, the last block adds them in block order) and the cell's
// sensitivity -1/2 vol s'(rho) drho/dz ese goes to cellq (nodal control: summed per node by
// k_node_sum afterwards; element control: the gradient itself).
__global__ void __launch_bounds__(kThreads, 4) k_energy_and_cell_grad(MeshView m, Material mat,
                                                                   const double* __restrict__ u,
                                                                   const double* __restrict__ z,
                                                                   double* __restrict__ partials,
                                                                   unsigned int* __restrict__ ticket,
                                                                   double* __restrict__ result,
                                                                   double* __restrict__ cellq) {
    __shared__ double sh[32];
    __shared__ bool last;
    double v = 0.0;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < m.num_cells;
         c += (int64_t)gridDim.x * blockDim.x) {
        CellState cs;
        load_cell(m, mat, z, c, cs);
        double ue[4][3], e[6], s[6];
        gather_state(u, cs.n, ue);
        strain_voigt(cs.G.g, ue, e);
        stress_voigt(mat, e, s);
        const double ese = s[0] * e[0] + s[1] * e[1] + s[2] * e[2] + s[3] * e[3] + s[4] * e[4] + s[5] * e[5];
        v += 0.5 * ese * cs.G.vol * simp(mat, cs.rho);
        cellq[c] = -0.5 * ese * cs.G.vol * (simp_dx(mat, cs.rho) * rho_dz(mat));
    }
    v = block_sum(v, sh);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = v;
        __threadfence();
        last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (last) {
        __threadfence();
        double t = 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) t += partials[b];
        t = block_sum(t, sh);
        if (threadIdx.x == 0) {
            *result = t;
            *ticket = 0u;
        }
    }
}

// Geometric "Volume" criterion (src/geometric/Volume.hpp:83-110): cell volume |det J| / 6
// weighted by the criterion's own penalty s_v(rho) (ApplyWeighting); GRAD = 1 gives the
// derivative with respect to one nodal control, vol s_v'(rho) / 4.
template <int GRAD>
__device__ __forceinline__ double cell_volume_quantity(const MeshView& m, const Material& pen,
                                                       const double* __restrict__ z, int64_t c) {
    CellState cs;
    load_cell(m, pen, z, c, cs);
    return GRAD ? cs.G.vol * simp_dx(pen, cs.rho) * rho_dz(pen) : cs.G.vol * simp(pen, cs.rho);
}

__global__ void __launch_bounds__(kThreads) k_volume_sum(MeshView m, Material pen, const double* __restrict__ z,
                                                         double* __restrict__ partials,
                                                         unsigned int* __restrict__ ticket,
                                                         double* __restrict__ result) {
    __shared__ double sh[32];
    __shared__ bool last;
    double v = 0.0;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < m.num_cells;
         c += (int64_t)gridDim.x * blockDim.x)
        v += cell_volume_quantity<0>(m, pen, z, c);
    v = block_sum(v, sh);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = v;
        __threadfence();
        last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (last) {
        __threadfence();
        double t = 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) t += partials[b];
        t = block_sum(t, sh);
        if (threadIdx.x == 0) {
            *result = t;
            *ticket = 0u;
        }
    }
}

__global__ void __launch_bounds__(kThreads) k_volume_cell_grad(MeshView m, Material pen,
                                                               const double* __restrict__ z,
                                                               double* __restrict__ out) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < m.num_cells;
         c += (int64_t)gridDim.x * blockDim.x)
        out[c] = cell_volume_quantity<1>(m, pen, z, c);
}

// Traction load F: SurfaceLoadIntegral<3> (src/SurfaceLoadIntegral.hpp:97-150) with the
// triangle degree-one rule (weight 1/2, basis 1/3 each), area from
// CalculateSurfaceArea<3> (src/SurfaceIntegralUtilities.hpp:217-227).
__global__ void k_traction(int32_t nfaces, const int32_t* __restrict__ fcell,
                           const int32_t* __restrict__ floc, double tx, double ty, double tz,
                           MeshView m, double* __restrict__ F) {
    for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f < nfaces;
         f += (int64_t)gridDim.x * blockDim.x) {
        const int4 n = m.conn[fcell[f]];
        int id[3];
        for (int a = 0; a < 3; ++a) id[a] = node_of(n, floc[3 * f + a]);
        double J[2][3];
        for (int a = 0; a < 2; ++a)
            for (int d = 0; d < 3; ++d) J[a][d] = m.coords[3 * (int64_t)id[a] + d] - m.coords[3 * (int64_t)id[2] + d];
        const double J23 = J[0][1] * J[1][2] - J[0][2] * J[1][1];
        const double J31 = J[0][2] * J[1][0] - J[0][0] * J[1][2];
        const double J12 = J[0][0] * J[1][1] - J[0][1] * J[1][0];
        const double area = 0.5 * sqrt(J23 * J23 + J31 * J31 + J12 * J12);
        const double c = 1.0 / 3.0;
        const double basis[3] = {1.0 - c - c, c, c};
        const double t[3] = {tx, ty, tz};
        for (int a = 0; a < 3; ++a)
            for (int d = 0; d < 3; ++d) atomicAdd(&F[3 * (int64_t)id[a] + d], basis[a] * t[d] * area);
    }
}

__global__ void k_axpby(int64_t n, double a, const double* __restrict__ x, double b,
                        double* __restrict__ y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        y[i] = a * x[i] + (b == 0.0 ? 0.0 : b * y[i]);
}

}  // namespace

MeshView mesh_view(const plato_problem* h) { return MeshView{h->N, h->C, h->conn, h->coords}; }
GraphView graph_view(const plato_problem* h) {
    return GraphView{h->N, h->nblocks, h->row_map, h->cols, h->diag, h->n2c_ptr, h->n2c};
}

int launch_axpby(plato_problem* h, int64_t n, double a, const double* x, double b, double* y) {
    k_axpby<<<grid_for(n, kThreads), kThreads, 0, h->stream>>>(n, a, x, b, y);
    PLATO_LAUNCH_CHECK(h);
    return PLATO_OK;
}

// R = K(z) u + scale_F * F   (scale_F = -1 gives VectorFunction::value, 0 gives dfdu)
int launch_internal_force(plato_problem* h, const double* u, const double* z, double* R, double scale_F) {
    const int64_t n = 3 * (int64_t)h->N;
    int rc = launch_axpby(h, n, scale_F, h->F, 0.0, R);
    if (rc) return rc;
    k_internal_force<<<grid_for(h->C, kThreads), kThreads, 0, h->stream>>>(mesh_view(h), h->material, u, z, R);
    PLATO_LAUNCH_CHECK(h);
    return PLATO_OK;
}

int launch_traction(plato_problem* h, int32_t nfaces, const int32_t* fcell, const int32_t* floc,
                    const double t[3]) {
    if (nfaces == 0) return PLATO_OK;
    k_traction<<<grid_for(nfaces, kThreads), kThreads, 0, h->stream>>>(nfaces, fcell, floc, t[0], t[1],
                                                                        t[2], mesh_view(h), h->F);
    PLATO_LAUNCH_CHECK(h);
    return PLATO_OK;
}

// Nodal control derivative: mode 1 (dfdz), 2 (self-adjoint dC/dz), 3 ((dR/dz)^T lam),
// 4 (dfdz + (dR/dz)^T lam).  cellbuf holds num_cells doubles.
int launch_nodal_control_derivative(plato_problem* h, int mode, const double* u, const double* z,
                                    const double* lam, double* cellbuf, double* out, int accumulate) {
    const MeshView m = mesh_view(h);
    const int G = grid_for(h->C, kThreads);
    // element control: the per-cell quantity is the derivative itself
    const bool cells = h->material.cell_control != 0;
    double* dst = cells ? out : cellbuf;
    const int acc = cells ? accumulate : 0;
    switch (mode) {
        case 1: k_cell_quantity<1><<<G, kThreads, 0, h->stream>>>(m, h->material, u, z, lam, dst, acc); break;
        case 2: k_cell_quantity<2><<<G, kThreads, 0, h->stream>>>(m, h->material, u, z, lam, dst, acc); break;
        case 3: k_cell_quantity<3><<<G, kThreads, 0, h->stream>>>(m, h->material, u, z, lam, dst, acc); break;
        case 4: k_cell_quantity<4><<<G, kThreads, 0, h->stream>>>(m, h->material, u, z, lam, dst, acc); break;
        default: return plato_fail(h, PLATO_BAD_INPUT, "unknown control-derivative mode");
    }
    PLATO_LAUNCH_CHECK(h);
    if (cells) return PLATO_OK;
    k_node_sum<<<grid_for(h->N, kThreads), kThreads, 0, h->stream>>>(graph_view(h), cellbuf, out, accumulate);
    PLATO_LAUNCH_CHECK(h);
    return PLATO_OK;
}

// Volume criterion value into *result (device scalar) and its nodal gradient.
int launch_volume(plato_problem* h, const Material& pen, const double* z, double* result) {
    const int G = grid_for(h->C, kThreads, h->partials_len);
    k_volume_sum<<<G, kThreads, 0, h->stream>>>(mesh_view(h), pen, z, h->partials, h->red_ticket, result);
    PLATO_LAUNCH_CHECK(h);
    return PLATO_OK;
}

int launch_volume_gradient(plato_problem* h, const Material& pen, const double* z, double* dvdz) {
    const bool cells = pen.cell_control != 0;
    k_volume_cell_grad<<<grid_for(h->C, kThreads), kThreads, 0, h->stream>>>(mesh_view(h), pen, z,
                                                                              cells ? dvdz : h->cellbuf);
    PLATO_LAUNCH_CHECK(h);
    if (cells) return PLATO_OK;
    k_node_sum<<<grid_for(h->N, kThreads), kThreads, 0, h->stream>>>(graph_view(h), h->cellbuf, dvdz, 0);
    PLATO_LAUNCH_CHECK(h);
    return PLATO_OK;
}

// Internal elastic energy of each member of a batch: CTA (member, piece) sums its share of
// the member's cells, then one thread per member adds the pieces in order (deterministic).
__global__ void __launch_bounds__(kThreads) k_energy_pieces(MeshView m, Material mat, const double* __restrict__ u,
                                                            const double* __restrict__ z,
                                                            const int32_t* __restrict__ cell_off,
                                                            double* __restrict__ pieces) {
    __shared__ double sh[32];
    const int s = blockIdx.x / kEnergySplit, piece = blockIdx.x - s * kEnergySplit;
    const int64_t c0 = cell_off[s], c1 = cell_off[s + 1];
    const int64_t len = (c1 - c0 + kEnergySplit - 1) / kEnergySplit;
    const int64_t a = c0 + piece * len, e = a + len < c1 ? a + len : c1;
    double v = 0.0;
    for (int64_t c = a + threadIdx.x; c < e; c += blockDim.x) v += cell_quantity<0>(m, mat, u, z, nullptr, c);
    v = block_sum(v, sh);
    if (threadIdx.x == 0) pieces[blockIdx.x] = v;
}

__global__ void k_sum_pieces(int32_t nseg, const double* __restrict__ pieces, double* __restrict__ values) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nseg; s += gridDim.x * blockDim.x) {
        double t = 0.0;
        for (int k = 0; k < kEnergySplit; ++k) t += pieces[(int64_t)s * kEnergySplit + k];
        values[s] = t;
    }
}

// The energy sums run one resident wave (4 CTAs of 256 threads per SM at 64 registers): each
// thread accumulates several cells before the block sums, so the per-block reduction and the
// partial written per block are paid once per CTA rather than once per 256 cells.
static int energy_grid(plato_problem* h) {
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device) != cudaSuccess || sms < 1) sms = 148;
    return grid_for(h->C, kThreads, std::min(h->partials_len, 4 * sms));
}

// Internal elastic energy into *result (device scalar).
int launch_energy(plato_problem* h, const double* u, const double* z, double* result) {
    const int G = energy_grid(h);
    k_energy_sum<<<G, kThreads, 0, h->stream>>>(mesh_view(h), h->material, u, z, h->partials,
                                                 h->red_ticket, result);
    PLATO_LAUNCH_CHECK(h);
    return PLATO_OK;
}

// Compliance into *result (device scalar) and the self-adjoint dC/dz into dfdz, one pass.
int launch_energy_and_gradient(plato_problem* h, const double* u, const double* z, double* result, double* dfdz) {
    const int G = energy_grid(h);
    const bool cells = h->material.cell_control != 0;
    k_energy_and_cell_grad<<<G, kThreads, 0, h->stream>>>(mesh_view(h), h->material, u, z, h->partials,
                                                           h->red_ticket, result, cells ? dfdz : h->cellbuf);
    PLATO_LAUNCH_CHECK(h);
    if (cells) return PLATO_OK;
    k_node_sum<<<grid_for(h->N, kThreads), kThreads, 0, h->stream>>>(graph_view(h), h->cellbuf, dfdz, 0);
    PLATO_LAUNCH_CHECK(h);
    return PLATO_OK;
}

// Energy of every batch member into values[nseg] (device).
int launch_energy_segments(plato_problem* h, const double* u, const double* z, double* values) {
    const int nseg = h->batch.nseg;
    k_energy_pieces<<<nseg * kEnergySplit, kThreads, 0, h->stream>>>(mesh_view(h), h->material, u, z,
                                                                      h->batch.cell_off_d, h->batch.values);
    PLATO_LAUNCH_CHECK(h);
    k_sum_pieces<<<grid_for(nseg, 128), 128, 0, h->stream>>>(nseg, h->batch.values, values);
    PLATO_LAUNCH_CHECK(h);
    return PLATO_OK;
}

}  // namespace plato
