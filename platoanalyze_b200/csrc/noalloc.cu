// Compliance value (internal elastic energy) without any device allocation.
//
// plato_sf_value needs a handle, and plato_create allocates device memory for the mesh, the
// graph and the solver.  Some callers cannot allocate at the point they need the criterion:
// for instance code whose device memory is owned up front by another allocator (a Kokkos
// memory pool, a framework arena) that must not grow behind its back, or code that must
// not risk the implicit device synchronisation cudaMalloc / cudaFree can cause.  This entry
// point takes everything as caller-owned device pointers and keeps its only scratch -- the
// per-block partial sums of the reduction, the last-block ticket and an error word -- in a
// file-scope static __device__ array, which every GPU that loads the library holds until
// the process exits.
//
// The computation is the same as plato_sf_value: 1/2 vol s(rho) eps.C.eps per cell
// (InternalElasticEnergy::evaluate, src/elliptic/InternalElasticEnergy.hpp:169-192) summed
// over cells (local_result_sum, src/Assembly.hpp:20-33), here one thread per cell, block
// sums, then the last block to finish sums the block partials in block order.  A cell with
// a node id outside [0, num_nodes) is skipped before any of its loads and marks the error
// word; the result is then NaN and the call returns PLATO_BAD_INPUT, as plato_create does
// for such a mesh.
#include <cmath>
#include <cstddef>
#include <mutex>
#include <string>

#include "plato_internal.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 65536;
constexpr int64_t kMaxCells = int64_t(kMaxBlocks) * kThreads;  // 16,777,216 cells
constexpr int kMaxDevices = 64;

struct NoAllocScratch {
    double partials[kMaxBlocks];  // one partial sum per block (512 KiB)
    unsigned int ticket;          // blocks finished; must be 0 when a call starts
    unsigned int bad_ids;         // cells skipped for an out-of-range node id; 0 when a call starts
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

std::mutex g_scratch_mutex;
NoAllocScratch* g_scratch_addr[kMaxDevices] = {};

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ void __launch_bounds__(kThreads)
k_energy_noalloc(int32_t N, int32_t C, const int4* __restrict__ conn, const double* __restrict__ coords,
                 const double* __restrict__ u, const double* __restrict__ z, plato::Material mat,
                 NoAllocScratch* __restrict__ scratch, double* __restrict__ result) {
    __shared__ double sh[kThreads / 32];
    __shared__ bool last;
    const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    double v = 0.0;
    unsigned int bad = 0u;
    int4 n = make_int4(0, 0, 0, 0);
    if (c < C) {
        n = conn[c];
        bad = (unsigned(n.x) >= unsigned(N)) | (unsigned(n.y) >= unsigned(N)) | (unsigned(n.z) >= unsigned(N)) |
              (unsigned(n.w) >= unsigned(N));
    }
    if (bad) atomicAdd(&scratch->bad_ids, 1u);
    if (c < C && !bad) {
        double x[4][3], ue[4][3];
        plato::load_cell_coords(coords, n, x);
        plato::TetGeom<double> G;
        plato::tet_geometry(x, G);
        const int ids[4] = {n.x, n.y, n.z, n.w};
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int d = 0; d < 3; ++d) ue[a][d] = __ldg(u + 3 * (int64_t)ids[a] + d);
        double e[6], s[6];
        plato::strain_voigt(G.g, ue, e);
        plato::stress_voigt(mat, e, s);
        const double rho = (__ldg(z + n.x) + __ldg(z + n.y) + __ldg(z + n.z) + __ldg(z + n.w)) * 0.25;
        const double ese = s[0] * e[0] + s[1] * e[1] + s[2] * e[2] + s[3] * e[3] + s[4] * e[4] + s[5] * e[5];
        v = 0.5 * ese * G.vol * plato::simp(mat, rho);
    }
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) b += sh[w];
        scratch->partials[blockIdx.x] = b;
        __threadfence();
        last = (atomicAdd(&scratch->ticket, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (last) {
        __threadfence();
        double t = 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) t += scratch->partials[b];
        t = warp_sum(t);
        __syncthreads();
        if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = t;
        __syncthreads();
        if (threadIdx.x == 0) {
            double total = 0.0;
            for (int w = 0; w < kThreads / 32; ++w) total += sh[w];
            // every block's bad-id increment precedes its ticket (fence), so the count is final
            *result = atomicAdd(&scratch->bad_ids, 0u) ? __longlong_as_double(0x7ff8000000000000LL) : total;
            scratch->ticket = 0u;
        }
    }
}

// Device address of the static scratch for the current device, looked up once per device.
int scratch_address(NoAllocScratch** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return plato_cuda_fail(nullptr, e, "cudaGetDevice", __FILE__, __LINE__);
    if (dev < 0 || dev >= kMaxDevices)
        return plato_fail(nullptr, PLATO_NOT_SUPPORTED, "device ordinal beyond the no-alloc scratch table");
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return plato_cuda_fail(nullptr, e, "cudaGetSymbolAddress", __FILE__, __LINE__);
        g_scratch_addr[dev] = static_cast<NoAllocScratch*>(p);
    }
    *out = g_scratch_addr[dev];
    return PLATO_OK;
}

}  // namespace

extern "C" int plato_sf_value_noalloc(int32_t num_nodes, int32_t num_cells, const int32_t* connectivity,
                                      const double* coords, const double* u, const double* z,
                                      const plato_material* material, const plato_penalty* penalty,
                                      double* value, void* cuda_stream) {
    if (num_cells < 1 || int64_t(num_cells) > kMaxCells)
        return plato_fail(nullptr, PLATO_BAD_INPUT,
                          "plato_sf_value_noalloc: num_cells must be in [1, 16777216] (the static scratch holds "
                          "one partial sum per 256 cells, 65536 blocks)");
    if (num_nodes < 1 || !connectivity || !coords || !u || !z || !material || !penalty || !value)
        return plato_fail(nullptr, PLATO_BAD_INPUT, "plato_sf_value_noalloc: null pointer or empty mesh");
    if (reinterpret_cast<uintptr_t>(connectivity) % 16 != 0)
        return plato_fail(nullptr, PLATO_BAD_INPUT, "plato_sf_value_noalloc: connectivity must be 16-byte aligned");
    const double E = material->youngs_modulus, nu = material->poissons_ratio;
    // the same checks as plato_create
    if (!std::isfinite(E) || !std::isfinite(nu) || nu <= -1.0 || nu >= 0.5)
        return plato_fail(nullptr, PLATO_BAD_INPUT, "plato_sf_value_noalloc: material needs finite E and -1 < nu < 0.5");
    if (!std::isfinite(penalty->exponent) || !std::isfinite(penalty->minimum_value))
        return plato_fail(nullptr, PLATO_BAD_INPUT, "plato_sf_value_noalloc: non-finite penalty parameter");
    // IsotropicLinearElasticMaterial<3> constants (src/IsotropicLinearElasticMaterial.cpp:86-110)
    plato::Material mat{};
    const double coef = E / ((1.0 + nu) * (1.0 - 2.0 * nu));
    mat.c00 = coef * (1.0 - nu);
    mat.c01 = coef * nu;
    mat.c33 = 1.0 / 2.0 * coef * (1.0 - 2.0 * nu);
    mat.p = penalty->exponent;
    mat.rho_min = penalty->minimum_value;
    mat.p_int = (mat.p >= 0.0 && mat.p <= 16.0 && double(int(mat.p)) == mat.p) ? int(mat.p) : -1;

    NoAllocScratch* scratch = nullptr;
    int rc = scratch_address(&scratch);
    if (rc) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    // ticket and error word are adjacent: one memset clears both
    static_assert(offsetof(NoAllocScratch, bad_ids) == offsetof(NoAllocScratch, ticket) + sizeof(unsigned int),
                  "ticket and bad_ids must be adjacent");
    cudaError_t e = cudaMemsetAsync(&scratch->ticket, 0, 2 * sizeof(unsigned int), s);
    if (e != cudaSuccess) return plato_cuda_fail(nullptr, e, "cudaMemsetAsync", __FILE__, __LINE__);
    const int blocks = int((int64_t(num_cells) + kThreads - 1) / kThreads);
    k_energy_noalloc<<<blocks, kThreads, 0, s>>>(num_nodes, num_cells, reinterpret_cast<const int4*>(connectivity),
                                                 coords, u, z, mat, scratch, value);
    e = cudaGetLastError();
    if (e != cudaSuccess) return plato_cuda_fail(nullptr, e, "k_energy_noalloc launch", __FILE__, __LINE__);
    // wait for the kernel so that the status can report what it found (pageable copies of
    // two words: no allocation)
    unsigned int bad = 0u;
    double result = 0.0;
    e = cudaMemcpyAsync(&bad, &scratch->bad_ids, sizeof(bad), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&result, value, sizeof(result), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return plato_cuda_fail(nullptr, e, "plato_sf_value_noalloc result", __FILE__, __LINE__);
    if (bad)
        return plato_fail(nullptr, PLATO_BAD_INPUT,
                          "plato_sf_value_noalloc: " + std::to_string(bad) +
                              " cell(s) reference a node id outside [0, num_nodes); value set to NaN");
    if (!std::isfinite(result))
        return plato_fail(nullptr, PLATO_NONFINITE, "plato_sf_value_noalloc: non-finite compliance value");
    return PLATO_OK;
}
