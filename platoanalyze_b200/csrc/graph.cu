// Node graph and block pattern, built once per mesh on the device.
//
// Reference semantics (bit-exact): row a of the block matrix holds every node that shares
// a cell with a, sorted ascending, with the diagonal inserted in sorted position --
// EngineMesh::createNodeNodeGraph (src/EngineMesh.cpp:223-320: unique, self excluded,
// sorted) followed by CreateBlockMatrix (src/ImplicitFunctors.hpp:932-1005: diagonal put
// in front of the first larger column).  That is exactly the sorted set
// {nodes sharing a cell with a} U {a}, which is what the radix sort + unique below builds
// from the (row, col) pairs of every cell, plus (a, a) for every node so that nodes in no
// cell still get their diagonal, as in the reference.
//
// The node -> (cell, local slot) incidence is built the same way and sorted by cell, so
// every node-centric kernel accumulates in a fixed order (bit-reproducible results).
#include <cub/cub.cuh>

#include "plato_internal.cuh"

namespace plato {
namespace {

__global__ void k_pair_keys(int32_t C, int32_t N, const int4* __restrict__ conn,
                            uint64_t* __restrict__ keys) {
    const int64_t total = 16 * (int64_t)C + N;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        uint64_t key;
        if (t < 16 * (int64_t)C) {
            const int64_t c = t >> 4;
            const int a = int(t >> 2) & 3, b = int(t) & 3;
            const int4 n = conn[c];
            key = ((uint64_t)(uint32_t)node_of(n, a) << 32) | (uint32_t)node_of(n, b);
        } else {
            const uint32_t i = uint32_t(t - 16 * (int64_t)C);
            key = ((uint64_t)i << 32) | i;
        }
        keys[t] = key;
    }
}

__global__ void k_pattern_from_keys(int64_t nb, int32_t N, const uint64_t* __restrict__ keys,
                                    int32_t* __restrict__ row_map, int32_t* __restrict__ cols,
                                    int32_t* __restrict__ diag) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nb;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t k = keys[i];
        const int32_t r = int32_t(k >> 32), c = int32_t(k & 0xffffffffu);
        cols[i] = c;
        if (r == c) diag[r] = int32_t(i);
        if (i == 0 || int32_t(keys[i - 1] >> 32) != r) row_map[r] = int32_t(i);
        if (i == nb - 1) row_map[N] = int32_t(nb);
    }
}

__global__ void k_incidence_keys(int32_t C, const int4* __restrict__ conn,
                                 uint64_t* __restrict__ keys, int32_t* __restrict__ count) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < 4 * (int64_t)C;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = t >> 2;
        const int a = int(t) & 3;
        const int32_t node = node_of(conn[c], a);
        keys[t] = ((uint64_t)(uint32_t)node << 32) | (uint32_t)(c * 4 + a);
        atomicAdd(&count[node], 1);
    }
}

__global__ void k_low_words(int64_t n, const uint64_t* __restrict__ keys, int32_t* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = int32_t(keys[i] & 0xffffffffu);
}

__global__ void k_check_conn(int32_t C, int32_t N, const int4* __restrict__ conn, int32_t* bad) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < C;
         c += (int64_t)gridDim.x * blockDim.x) {
        const int4 n = conn[c];
        const bool ok = n.x >= 0 && n.x < N && n.y >= 0 && n.y < N && n.z >= 0 && n.z < N &&
                        n.w >= 0 && n.w < N && n.x != n.y && n.x != n.z && n.x != n.w &&
                        n.y != n.z && n.y != n.w && n.z != n.w;
        if (!ok) atomicExch(bad, 1);
    }
}

int end_bit_for(int64_t max_value) {
    int bits = 1;
    while (bits < 63 && (int64_t(1) << bits) <= max_value) ++bits;
    return bits;
}

}  // namespace

// Builds row_map / cols / diag and n2c_ptr / n2c on the handle.
int build_graph(plato_problem* h) {
    const int32_t N = h->N, C = h->C;
    cudaStream_t s = h->stream;
    const int T = 256;

    // connectivity sanity (ids in range, 4 distinct nodes per cell)
    int32_t* d_bad = nullptr;
    PLATO_CUDA(h, cudaMallocAsync(&d_bad, sizeof(int32_t), s));
    PLATO_CUDA(h, cudaMemsetAsync(d_bad, 0, sizeof(int32_t), s));
    k_check_conn<<<grid_for(C, T), T, 0, s>>>(C, N, h->conn, d_bad);
    PLATO_LAUNCH_CHECK(h);
    int32_t bad = 0;
    PLATO_CUDA(h, cudaMemcpyAsync(&bad, d_bad, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    PLATO_CUDA(h, cudaStreamSynchronize(s));
    PLATO_CUDA(h, cudaFreeAsync(d_bad, s));
    if (bad) return plato_fail(h, PLATO_BAD_INPUT, "connectivity has an out-of-range or repeated node id");

    // ---- block pattern --------------------------------------------------------------
    const int64_t npairs = 16 * (int64_t)C + N;
    uint64_t *k_in = nullptr, *k_out = nullptr, *k_uniq = nullptr;
    int64_t* d_num = nullptr;
    PLATO_CUDA(h, cudaMallocAsync(&k_in, npairs * sizeof(uint64_t), s));
    PLATO_CUDA(h, cudaMallocAsync(&k_out, npairs * sizeof(uint64_t), s));
    PLATO_CUDA(h, cudaMallocAsync(&d_num, sizeof(int64_t), s));
    k_pair_keys<<<grid_for(npairs, T, 148 * 64), T, 0, s>>>(C, N, h->conn, k_in);
    PLATO_LAUNCH_CHECK(h);
    const int ebits = 32 + end_bit_for(N);
    size_t tmp_sort = 0, tmp_uniq = 0;
    PLATO_CUDA(h, cub::DeviceRadixSort::SortKeys(nullptr, tmp_sort, k_in, k_out, npairs, 0, ebits, s));
    PLATO_CUDA(h, cub::DeviceSelect::Unique(nullptr, tmp_uniq, k_out, k_in, d_num, npairs, s));
    void* tmp = nullptr;
    const size_t tmp_bytes = tmp_sort > tmp_uniq ? tmp_sort : tmp_uniq;
    PLATO_CUDA(h, cudaMallocAsync(&tmp, tmp_bytes, s));
    size_t tb = tmp_bytes;
    PLATO_CUDA(h, cub::DeviceRadixSort::SortKeys(tmp, tb, k_in, k_out, npairs, 0, ebits, s));
    tb = tmp_bytes;
    PLATO_CUDA(h, cub::DeviceSelect::Unique(tmp, tb, k_out, k_in, d_num, npairs, s));
    k_uniq = k_in;
    int64_t nb = 0;
    PLATO_CUDA(h, cudaMemcpyAsync(&nb, d_num, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    PLATO_CUDA(h, cudaStreamSynchronize(s));
    if (nb > INT32_MAX / 9)
        return plato_fail(h, PLATO_BAD_INPUT, "block pattern too large for int32 entry offsets");
    h->nblocks = nb;
    PLATO_CUDA(h, cudaMalloc(&h->row_map, (N + 1) * sizeof(int32_t)));
    PLATO_CUDA(h, cudaMalloc(&h->cols, nb * sizeof(int32_t)));
    PLATO_CUDA(h, cudaMalloc(&h->diag, N * sizeof(int32_t)));
    k_pattern_from_keys<<<grid_for(nb, T, 148 * 64), T, 0, s>>>(nb, N, k_uniq, h->row_map, h->cols, h->diag);
    PLATO_LAUNCH_CHECK(h);

    // ---- node -> (cell, slot) incidence ----------------------------------------------
    const int64_t ninc = 4 * (int64_t)C;
    int32_t* counts = nullptr;
    PLATO_CUDA(h, cudaMallocAsync(&counts, (N + 1) * sizeof(int32_t), s));
    PLATO_CUDA(h, cudaMemsetAsync(counts, 0, (N + 1) * sizeof(int32_t), s));
    k_incidence_keys<<<grid_for(ninc, T, 148 * 64), T, 0, s>>>(C, h->conn, k_in, counts);
    PLATO_LAUNCH_CHECK(h);
    tb = tmp_bytes;
    PLATO_CUDA(h, cub::DeviceRadixSort::SortKeys(tmp, tb, k_in, k_out, ninc, 0, ebits, s));
    PLATO_CUDA(h, cudaMalloc(&h->n2c_ptr, (N + 1) * sizeof(int32_t)));
    PLATO_CUDA(h, cudaMalloc(&h->n2c, (ninc > 0 ? ninc : 1) * sizeof(int32_t)));
    size_t tmp_scan = 0;
    PLATO_CUDA(h, cub::DeviceScan::ExclusiveSum(nullptr, tmp_scan, counts, h->n2c_ptr, N + 1, s));
    if (tmp_scan > tmp_bytes) return plato_fail(h, PLATO_OUT_OF_MEMORY, "scan scratch larger than sort scratch");
    tb = tmp_bytes;
    PLATO_CUDA(h, cub::DeviceScan::ExclusiveSum(tmp, tb, counts, h->n2c_ptr, N + 1, s));
    k_low_words<<<grid_for(ninc, T, 148 * 64), T, 0, s>>>(ninc, k_out, h->n2c);
    PLATO_LAUNCH_CHECK(h);

    PLATO_CUDA(h, cudaFreeAsync(counts, s));
    PLATO_CUDA(h, cudaFreeAsync(tmp, s));
    PLATO_CUDA(h, cudaFreeAsync(k_in, s));
    PLATO_CUDA(h, cudaFreeAsync(k_out, s));
    PLATO_CUDA(h, cudaFreeAsync(d_num, s));
    PLATO_CUDA(h, cudaStreamSynchronize(s));
    return PLATO_OK;
}

}  // namespace plato
