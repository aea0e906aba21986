// Matrix-free element-by-element operator: y = K(z) x for the Dirichlet-constrained
// stiffness, recomputed from the mesh on every apply (no assembled matrix).
//
// K(z) = sum_e s(rho_e) vol_e B_e^T C B_e (ElastostaticResidual, src/elliptic/
// ElastostaticResidual.hpp:165-234, differentiated in closed form).  The constrained
// operator is the one applyBlockConstraints produces (src/ApplyConstraints.hpp:40-112):
// rows and columns of constrained dofs are cleared and their diagonal set to 1, i.e.
// y = P K P x + (I - P) x with P the free-dof mask.
//
// One thread per cell: connectivity (one int4), the four node coordinates and the cell's
// precomputed SIMP weight, the masked state gather, strain, stress, and a 12-entry scatter
// with FP32/FP64 atomics into y (an L2-resident vector).  Constrained rows are written
// afterwards by the consumer (y_d = x_d).  Templated on the arithmetic type: FP64 for the
// outer Krylov operator, FP32 (with FP32 coordinates) for the mixed-precision
// preconditioner.
#include "plato_internal.cuh"

namespace plato {

MeshView mesh_view(const plato_problem* h);
GraphView graph_view(const plato_problem* h);

namespace {

constexpr int kThreads = 256;

// Per-cell SIMP weight s(rho_e) (ApplyWeighting, src/ApplyWeighting.hpp:55-64) in T.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_cell_weights(int32_t C, const int4* __restrict__ conn,
                                                           const double* __restrict__ z, Material mat,
                                                           T* __restrict__ w) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < C;
         c += (int64_t)gridDim.x * blockDim.x) {
        const int4 n = conn[c];
        const double rho = cell_rho(mat, z, c, n);
        w[c] = T(simp(mat, rho));
    }
}

template <typename T>
__device__ __forceinline__ void load_coords_t(const T* __restrict__ coords, int4 n, T x[4][3]) {
    const int ids[4] = {n.x, n.y, n.z, n.w};
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const T* p = coords + 3 * (int64_t)ids[a];
        x[a][0] = __ldg(p + 0);
        x[a][1] = __ldg(p + 1);
        x[a][2] = __ldg(p + 2);
    }
}

template <typename T>
__global__ void __launch_bounds__(kThreads)
k_ebe_apply(int32_t C, const int4* __restrict__ conn, const T* __restrict__ coords, const T* __restrict__ wcell,
            Material mat, const uint8_t* __restrict__ mask, const T* __restrict__ x, T* __restrict__ y,
            const PcgScalars* S) {
    if (S && S->done) return;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < C;
         c += (int64_t)gridDim.x * blockDim.x) {
        const int4 n = conn[c];
        T xc[4][3];
        load_coords_t(coords, n, xc);
        TetGeom<T> G;
        tet_geometry(xc, G);
        const int ids[4] = {n.x, n.y, n.z, n.w};
        T ue[4][3];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const int64_t dof = 3 * (int64_t)ids[a] + d;
                ue[a][d] = (mask && __ldg(mask + dof)) ? T(0) : __ldg(x + dof);
            }
        T e[6], s[6];
        strain_voigt(G.g, ue, e);
        stress_voigt(mat, e, s);
        const T w = G.vol * __ldg(wcell + c);
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            T f[3];
            divergence_node(G.g[a], s, w, f);
            T* dst = y + 3 * (int64_t)ids[a];
            atomicAdd(dst + 0, f[0]);
            atomicAdd(dst + 1, f[1]);
            atomicAdd(dst + 2, f[2]);
        }
    }
}

// Diagonal of the constrained operator, node-centric over the incidence lists (no atomics):
// K_aa[d][d] = sum_e w_e vol_e ((lambda + mu) g_ad^2 + mu |g_a|^2); 1 on constrained dofs.
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_diag_inverse(GraphView g, const int4* __restrict__ conn, const double* __restrict__ coords,
               const double* __restrict__ wcell, Material mat, const uint8_t* __restrict__ mask,
               double* __restrict__ dinv64, float* __restrict__ dinv32) {
    for (int64_t a = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; a < g.num_nodes;
         a += (int64_t)gridDim.x * blockDim.x) {
        double dg[3] = {0.0, 0.0, 0.0};
        for (int32_t k = g.n2c_ptr[a]; k < g.n2c_ptr[a + 1]; ++k) {
            const int32_t packed = g.n2c[k];
            const int32_t c = packed >> 2, la = packed & 3;
            const int4 n = conn[c];
            double x[4][3];
            load_cell_coords(coords, n, x);
            TetGeom<double> G;
            tet_geometry(x, G);
            const double w = G.vol * wcell[c];
            const double* ga = G.g[la];
            const double gg = ga[0] * ga[0] + ga[1] * ga[1] + ga[2] * ga[2];
#pragma unroll
            for (int d = 0; d < 3; ++d) dg[d] += w * ((mat.c01 + mat.c33) * ga[d] * ga[d] + mat.c33 * gg);
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const int64_t dof = 3 * a + d;
            const double v = mask[dof] ? 1.0 : 1.0 / dg[d];
            if (dinv64) dinv64[dof] = v;
            if (dinv32) dinv32[dof] = float(v);
        }
    }
    (void)sizeof(T);
}

template <typename T>
__global__ void k_zero(int64_t n, T* __restrict__ y, const PcgScalars* S) {
    if (S && S->done) return;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = T(0);
}

__global__ void k_mask_copy(int64_t n, const uint8_t* __restrict__ mask, const double* __restrict__ x,
                            double* __restrict__ y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (mask[i]) y[i] = x[i];
}

__global__ void k_masked_axpy(int64_t n, const uint8_t* __restrict__ mask, double a, const double* __restrict__ x,
                              double* __restrict__ y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (!mask[i]) y[i] += a * x[i];
}

__global__ void k_to_float(int64_t n, const double* __restrict__ a, float* __restrict__ b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = float(a[i]);
}

}  // namespace

// Precomputes what the matrix-free operator needs for control z: per-cell weights (FP64
// and FP32) and the inverse diagonal (FP64 into h->v_dinv, FP32 into h->f_dinv).
int matfree_setup(plato_problem* h, const double* z) {
    const int64_t n = 3 * (int64_t)h->N;
    if (!h->mf_w64) PLATO_CUDA(h, cudaMalloc(&h->mf_w64, sizeof(double) * h->C));
    if (!h->mf_w32) PLATO_CUDA(h, cudaMalloc(&h->mf_w32, sizeof(float) * h->C));
    if (!h->f_dinv) PLATO_CUDA(h, cudaMalloc(&h->f_dinv, sizeof(float) * n));
    if (!h->f_coords) {
        PLATO_CUDA(h, cudaMalloc(&h->f_coords, sizeof(float) * n));
        k_to_float<<<grid_for(n, kThreads), kThreads, 0, h->stream>>>(n, h->coords, h->f_coords);
        PLATO_LAUNCH_CHECK(h);
    }
    const int G = grid_for(h->C, kThreads);
    k_cell_weights<double><<<G, kThreads, 0, h->stream>>>(h->C, h->conn, z, h->material, h->mf_w64);
    PLATO_LAUNCH_CHECK(h);
    k_cell_weights<float><<<G, kThreads, 0, h->stream>>>(h->C, h->conn, z, h->material, h->mf_w32);
    PLATO_LAUNCH_CHECK(h);
    k_diag_inverse<double><<<grid_for(h->N, kThreads), kThreads, 0, h->stream>>>(
        graph_view(h), h->conn, h->coords, h->mf_w64, h->material, h->bc_mask, h->v_dinv, h->f_dinv);
    PLATO_LAUNCH_CHECK(h);
    return PLATO_OK;
}

// y = P K P x (constrained rows of y are NOT written; the caller overwrites them with x).
// With S != nullptr both kernels return at once after the solver has converged.
int launch_ebe_apply64(plato_problem* h, const double* x, double* y, const PcgScalars* S) {
    const int64_t n = 3 * (int64_t)h->N;
    k_zero<double><<<grid_for(n, kThreads), kThreads, 0, h->stream>>>(n, y, S);
    k_ebe_apply<double><<<grid_for(h->C, kThreads, 148 * 64), kThreads, 0, h->stream>>>(
        h->C, h->conn, h->coords, h->mf_w64, h->material, h->bc_mask, x, y, S);
    h->launches += 1;
    PLATO_LAUNCH_CHECK(h);
    return PLATO_OK;
}

int launch_ebe_apply32(plato_problem* h, const float* x, float* y, const PcgScalars* S) {
    const int64_t n = 3 * (int64_t)h->N;
    k_zero<float><<<grid_for(n, kThreads), kThreads, 0, h->stream>>>(n, y, S);
    k_ebe_apply<float><<<grid_for(h->C, kThreads, 148 * 64), kThreads, 0, h->stream>>>(
        h->C, h->conn, h->f_coords, h->mf_w32, h->material, h->bc_mask, x, y, S);
    h->launches += 1;
    PLATO_LAUNCH_CHECK(h);
    return PLATO_OK;
}

// K x without the constraint mask (for the Dirichlet lift of inhomogeneous values).
int launch_ebe_apply64_unmasked(plato_problem* h, const double* x, double* y) {
    const int64_t n = 3 * (int64_t)h->N;
    k_zero<double><<<grid_for(n, kThreads), kThreads, 0, h->stream>>>(n, y, nullptr);
    k_ebe_apply<double><<<grid_for(h->C, kThreads, 148 * 64), kThreads, 0, h->stream>>>(
        h->C, h->conn, h->coords, h->mf_w64, h->material, nullptr, x, y, nullptr);
    h->launches += 1;
    PLATO_LAUNCH_CHECK(h);
    return PLATO_OK;
}

// y_free += a x_free.
int launch_masked_axpy(plato_problem* h, double a, const double* x, double* y) {
    const int64_t n = 3 * (int64_t)h->N;
    k_masked_axpy<<<grid_for(n, kThreads), kThreads, 0, h->stream>>>(n, h->bc_mask, a, x, y);
    PLATO_LAUNCH_CHECK(h);
    return PLATO_OK;
}

// y_d = x_d on constrained dofs.
int launch_mask_copy(plato_problem* h, const double* x, double* y) {
    const int64_t n = 3 * (int64_t)h->N;
    k_mask_copy<<<grid_for(n, kThreads), kThreads, 0, h->stream>>>(n, h->bc_mask, x, y);
    PLATO_LAUNCH_CHECK(h);
    return PLATO_OK;
}

}  // namespace plato
