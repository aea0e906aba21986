"""The benchmark's cantilever problem built on the host with numpy alone.

TEST INFRASTRUCTURE ONLY: the reference arm of bench.py and the tests build the oracle's
copy of the problem here, so that a CPU-only run of the reference path never loads the
product's CUDA library.  tests/test_workloads_cpu.py checks that these arrays equal the ones
the product's own generator makes.

Box [0,lx]x[0,ly]x[0,lz] cut into nx x ny x nz hexes, each hex into 6 tets around its
(0,0,0)-(1,1,1) diagonal (Kuhn split, the split the reference's BamG unit-test meshes use,
unit_tests/PlatoTestHelpers.hpp:31-84): tet t = [v000, P_t, P_t+1, v111] over the ring
P = (1,1,0),(0,1,0),(0,1,1),(0,0,1),(1,0,1),(1,0,0); nodes and hexes lexicographic, z fastest.
"""
from __future__ import annotations

import numpy as np

RING = np.array([[1, 1, 0], [0, 1, 0], [0, 1, 1], [0, 0, 1], [1, 0, 1], [1, 0, 0]], dtype=np.int64)


def tet_offsets() -> np.ndarray:
    """(6, 4, 3) hex-local offsets of the 4 nodes of each of the 6 tets."""
    off = np.zeros((6, 4, 3), dtype=np.int64)
    for t in range(6):
        off[t, 1] = RING[t]
        off[t, 2] = RING[(t + 1) % 6]
        off[t, 3] = (1, 1, 1)
    return off


def box_mesh(nx: int, ny: int, nz: int, lx: float = 1.0, ly: float = 1.0, lz: float = 1.0):
    """(coords (N,3) float64, connectivity (C,4) int32) of the Kuhn-split box."""
    i, j, k = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    coords = np.stack([lx * i.reshape(-1) / nx, ly * j.reshape(-1) / ny, lz * k.reshape(-1) / nz], axis=1)
    hi, hj, hk = (a.reshape(-1) for a in np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"))
    off = tet_offsets()  # (6, 4, 3)
    I = hi[:, None, None] + off[None, :, :, 0]
    J = hj[:, None, None] + off[None, :, :, 1]
    K = hk[:, None, None] + off[None, :, :, 2]
    conn = (K + (nz + 1) * (J + (ny + 1) * I)).reshape(-1, 4).astype(np.int32)
    return coords.astype(np.float64), conn


def nodeset(nx: int, ny: int, nz: int, axis: int, side: int) -> np.ndarray:
    """Nodes on a box face (axis 0/1/2, side 0: minimum, 1: maximum), increasing ids."""
    ids = np.arange((nx + 1) * (ny + 1) * (nz + 1)).reshape(nx + 1, ny + 1, nz + 1)
    n = (nx, ny, nz)[axis]
    return np.take(ids, n if side else 0, axis=axis).reshape(-1).astype(np.int32)


def sideset(nx: int, ny: int, nz: int, axis: int, side: int):
    """Tet faces on a box face as (cells, (F,3) cell-local node ordinals in increasing order),
    in cell order (the GetSideSetElements / GetSideSetLocalNodes layout)."""
    n = (nx, ny, nz)[axis]
    off = tet_offsets()
    hex_ijk = np.stack([a.reshape(-1) for a in np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz),
                                                             indexing="ij")], axis=1)
    on = hex_ijk[:, axis] == (n - 1 if side else 0)
    cells, local = [], []
    for h in np.nonzero(on)[0]:
        for t in range(6):
            loc = [a for a in range(4) if off[t, a, axis] == side]
            if len(loc) == 3:
                cells.append(6 * h + t)
                local.append(loc)
    return np.asarray(cells, dtype=np.int32), np.asarray(local, dtype=np.int32).reshape(-1, 3)


def splitmix_uniform(n: int, seed: int, lo: float = 0.01, hi: float = 1.0) -> np.ndarray:
    """n i.i.d. U[lo, hi) doubles from a SplitMix64 stream (value k uses state seed + k*golden)."""
    idx = np.arange(1, n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = np.uint64(seed) + idx * np.uint64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        x = x ^ (x >> np.uint64(31))
    u = (x >> np.uint64(11)).astype(np.float64) * (1.0 / float(1 << 53))
    return lo + (hi - lo) * u


def cantilever_oracle(nx: int, ny: int, nz: int, traction=(0.0, -1.0, 0.0), E=1.0, nu=0.3, p=3.0, rho_min=1e-9):
    """The oracle of the benchmark cantilever on [0,2]x[0,1]x[0,1]: clamped on x = 0, uniform
    traction on x = 2."""
    from oracle import Oracle

    coords, conn = box_mesh(nx, ny, nz, 2.0, 1.0, 1.0)
    fixed = nodeset(nx, ny, nz, 0, 0)
    dofs = (3 * fixed[:, None].astype(np.int64) + np.arange(3)[None, :]).reshape(-1).astype(np.int32)
    cells, local = sideset(nx, ny, nz, 0, 1)
    return Oracle(coords, conn, E, nu, p, rho_min, (cells, local), traction, dofs, np.zeros(dofs.size))
