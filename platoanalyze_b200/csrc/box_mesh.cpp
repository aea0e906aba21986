// Structured box mesh of linear tetrahedra (host code, no device work).
//
// The reference builds its unit-test meshes with PlatoEngine's BamG generator
// (unit_tests/PlatoTestHelpers.hpp:31-84), which is not part of the reference tree.
// This generator reproduces the numbering those tests' gold values imply:
//   * nodes lexicographic with z fastest: id = k + (nz+1)*(j + (ny+1)*i);
//   * hexes in the same order, each cut into 6 tets around its (0,0,0)-(1,1,1)
//     diagonal (Kuhn split): tet t = [v000, P_t, P_{t+1}, v111] with the ring
//     P = (1,1,0),(0,1,0),(0,1,1),(0,0,1),(1,0,1),(1,0,0).
// The per-cell gradients of unit_tests/DerivativeTests.cpp:155-162 and the assembled
// residual of :339-367 pin this ordering.
#include <cstdint>

#include "plato_b200.h"

namespace {

constexpr int kRing[6][3] = {{1, 1, 0}, {0, 1, 0}, {0, 1, 1}, {0, 0, 1}, {1, 0, 1}, {1, 0, 0}};

inline void tet_offsets(int t, int local, int off[3]) {
    if (local == 0) { off[0] = off[1] = off[2] = 0; return; }
    if (local == 3) { off[0] = off[1] = off[2] = 1; return; }
    const int* r = kRing[(t + local - 1) % 6];
    off[0] = r[0]; off[1] = r[1]; off[2] = r[2];
}

bool dims_ok(int32_t nx, int32_t ny, int32_t nz) {
    if (nx < 1 || ny < 1 || nz < 1) return false;
    const int64_t nodes = int64_t(nx + 1) * (ny + 1) * (nz + 1);
    const int64_t cells = int64_t(6) * nx * ny * nz;
    return nodes < INT32_MAX && 4 * cells < INT32_MAX;
}

}  // namespace

extern "C" {

int plato_box_mesh_sizes(int32_t nx, int32_t ny, int32_t nz, int32_t* num_nodes, int32_t* num_cells) {
    if (!dims_ok(nx, ny, nz) || !num_nodes || !num_cells) return PLATO_BAD_INPUT;
    *num_nodes = (nx + 1) * (ny + 1) * (nz + 1);
    *num_cells = 6 * nx * ny * nz;
    return PLATO_OK;
}

int plato_box_mesh_tet4(int32_t nx, int32_t ny, int32_t nz, double lx, double ly, double lz,
                        double* coords, int32_t* connectivity) {
    if (!dims_ok(nx, ny, nz) || !coords || !connectivity) return PLATO_BAD_INPUT;
    const int32_t NY = ny + 1, NZ = nz + 1;
    auto nid = [&](int32_t i, int32_t j, int32_t k) { return k + NZ * (j + NY * i); };
    for (int32_t i = 0; i <= nx; ++i)
        for (int32_t j = 0; j <= ny; ++j)
            for (int32_t k = 0; k <= nz; ++k) {
                double* x = coords + 3 * int64_t(nid(i, j, k));
                x[0] = lx * double(i) / double(nx);
                x[1] = ly * double(j) / double(ny);
                x[2] = lz * double(k) / double(nz);
            }
    int64_t c = 0;
    for (int32_t i = 0; i < nx; ++i)
        for (int32_t j = 0; j < ny; ++j)
            for (int32_t k = 0; k < nz; ++k)
                for (int t = 0; t < 6; ++t, ++c)
                    for (int a = 0; a < 4; ++a) {
                        int off[3];
                        tet_offsets(t, a, off);
                        connectivity[4 * c + a] = nid(i + off[0], j + off[1], k + off[2]);
                    }
    return PLATO_OK;
}

// face: 0 x-, 1 x+, 2 y-, 3 y+, 4 z-, 5 z+.  Nodes in increasing id order.
int plato_box_nodeset(int32_t nx, int32_t ny, int32_t nz, int32_t face, int32_t* nodes,
                      int32_t* count) {
    if (!dims_ok(nx, ny, nz) || face < 0 || face > 5 || !count) return PLATO_BAD_INPUT;
    const int32_t n[3] = {nx, ny, nz};
    const int axis = face / 2;
    const int32_t fixed = (face % 2) ? n[axis] : 0;
    int32_t m = 0;
    for (int32_t i = 0; i <= nx; ++i)
        for (int32_t j = 0; j <= ny; ++j)
            for (int32_t k = 0; k <= nz; ++k) {
                const int32_t ijk[3] = {i, j, k};
                if (ijk[axis] != fixed) continue;
                if (nodes) nodes[m] = k + (nz + 1) * (j + (ny + 1) * i);
                ++m;
            }
    *count = m;
    return PLATO_OK;
}

// Side set of a box face: the tet faces lying on it, as (cell, 3 cell-local node
// ordinals in increasing order), the layout of GetSideSetElements /
// GetSideSetLocalNodes (src/AbstractPlatoMesh.hpp:22-191).
int plato_box_sideset(int32_t nx, int32_t ny, int32_t nz, int32_t face, int32_t* cells,
                      int32_t* local_nodes, int32_t* count) {
    if (!dims_ok(nx, ny, nz) || face < 0 || face > 5 || !count) return PLATO_BAD_INPUT;
    const int32_t n[3] = {nx, ny, nz};
    const int axis = face / 2;
    const int side = face % 2;
    int32_t m = 0;
    int64_t c = 0;
    for (int32_t i = 0; i < nx; ++i)
        for (int32_t j = 0; j < ny; ++j)
            for (int32_t k = 0; k < nz; ++k) {
                const int32_t ijk[3] = {i, j, k};
                const bool on_boundary = side ? (ijk[axis] == n[axis] - 1) : (ijk[axis] == 0);
                for (int t = 0; t < 6; ++t, ++c) {
                    if (!on_boundary) continue;
                    int loc[4], cnt = 0;
                    for (int a = 0; a < 4; ++a) {
                        int off[3];
                        tet_offsets(t, a, off);
                        if (off[axis] == side) loc[cnt++] = a;
                    }
                    if (cnt != 3) continue;
                    if (cells) cells[m] = int32_t(c);
                    if (local_nodes)
                        for (int a = 0; a < 3; ++a) local_nodes[3 * int64_t(m) + a] = loc[a];
                    ++m;
                }
            }
    *count = m;
    return PLATO_OK;
}

}  // extern "C"
