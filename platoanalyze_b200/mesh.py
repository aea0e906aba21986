"""Structured tet box meshes (host arrays) through the library's generator."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from .capi import check, lib

X_MINUS, X_PLUS, Y_MINUS, Y_PLUS, Z_MINUS, Z_PLUS = range(6)


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


@dataclass
class BoxMesh:
    nx: int
    ny: int
    nz: int
    lx: float
    ly: float
    lz: float
    coords: np.ndarray        # (N, 3) float64
    connectivity: np.ndarray  # (C, 4) int32

    @property
    def num_nodes(self) -> int:
        return self.coords.shape[0]

    @property
    def num_cells(self) -> int:
        return self.connectivity.shape[0]

    def nodeset(self, face: int) -> np.ndarray:
        cnt = C.c_int32(0)
        check(lib.plato_box_nodeset(self.nx, self.ny, self.nz, face, None, C.byref(cnt)))
        out = np.empty(cnt.value, dtype=np.int32)
        check(lib.plato_box_nodeset(self.nx, self.ny, self.nz, face, _ptr(out), C.byref(cnt)))
        return out

    def sideset(self, face: int) -> tuple[np.ndarray, np.ndarray]:
        cnt = C.c_int32(0)
        check(lib.plato_box_sideset(self.nx, self.ny, self.nz, face, None, None, C.byref(cnt)))
        cells = np.empty(cnt.value, dtype=np.int32)
        local = np.empty((cnt.value, 3), dtype=np.int32)
        check(lib.plato_box_sideset(self.nx, self.ny, self.nz, face, _ptr(cells), _ptr(local), C.byref(cnt)))
        return cells, local


    def sides(self, faces) -> tuple[np.ndarray, np.ndarray]:
        """The faces of several box sides, concatenated: (owning cells, 3 local node ordinals)."""
        parts = [self.sideset(f) for f in faces]
        if not parts:
            return np.zeros(0, np.int32), np.zeros((0, 3), np.int32)
        return np.concatenate([p[0] for p in parts]), np.concatenate([p[1] for p in parts])


# cell-local node ordinals of the four faces of a tet
TET_FACES = np.array([[0, 1, 3], [1, 2, 3], [0, 3, 2], [0, 2, 1]], dtype=np.int32)


def exterior_faces(connectivity: np.ndarray, exclude_nodes: np.ndarray | None = None):
    """Faces that belong to exactly one cell, as (owning cells, 3 local node ordinals), in cell
    order.  With `exclude_nodes`, faces whose three nodes all lie in that node set are left
    out (the complement of a side set given by its nodes, as the Helmholtz filter's surface
    term takes it)."""
    conn = np.ascontiguousarray(connectivity, dtype=np.int64)
    nc = conn.shape[0]
    tri = conn[:, TET_FACES]                      # (nc, 4, 3) global nodes
    key = np.sort(tri.reshape(-1, 3), axis=1)
    _, inv, cnt = np.unique(key, axis=0, return_inverse=True, return_counts=True)
    once = cnt[inv.reshape(-1)] == 1
    if exclude_nodes is not None and len(exclude_nodes):
        mark = np.zeros(int(conn.max()) + 1, dtype=bool)
        mark[np.asarray(exclude_nodes, dtype=np.int64)] = True
        once &= ~mark[key].all(axis=1)
    idx = np.nonzero(once)[0]
    cells = (idx // 4).astype(np.int32)
    local = TET_FACES[idx % 4].astype(np.int32)
    return cells, local


@dataclass
class MeshFile:
    coords: np.ndarray        # (N, 3) float64
    connectivity: np.ndarray  # (C, 4) int32
    node_sets: dict           # name -> 0-based nodes
    side_sets: dict           # name -> (cells, (F, 3) local node ordinals)

    @property
    def num_nodes(self) -> int:
        return self.coords.shape[0]


def read_exodus(path: str) -> MeshFile:
    """An Exodus II tetrahedral mesh in a netCDF classic encoding (CDF-1, -2 or -5)."""
    from .capi import PlatoError

    h = C.c_void_p()
    rc = lib.plato_mesh_file_open(str(path).encode(), C.byref(h))
    if rc != 0:
        raise PlatoError(rc, (lib.plato_mesh_file_last_error() or b"").decode())
    try:
        nn, nc, nns, nss = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        check(lib.plato_mesh_file_info(h, C.byref(nn), C.byref(nc), C.byref(nns), C.byref(nss)))
        coords = np.empty((nn.value, 3), np.float64)
        conn = np.empty((nc.value, 4), np.int32)
        check(lib.plato_mesh_file_mesh(h, _ptr(coords), _ptr(conn)))
        name = C.create_string_buffer(256)
        node_sets, side_sets = {}, {}
        for k in range(nns.value):
            cnt = C.c_int32()
            check(lib.plato_mesh_file_node_set(h, k, name, 256, None, C.byref(cnt)))
            nodes = np.empty(cnt.value, np.int32)
            check(lib.plato_mesh_file_node_set(h, k, name, 256, _ptr(nodes), C.byref(cnt)))
            node_sets[name.value.decode()] = nodes
        for k in range(nss.value):
            cnt = C.c_int32()
            check(lib.plato_mesh_file_side_set(h, k, name, 256, None, None, C.byref(cnt)))
            cells = np.empty(cnt.value, np.int32)
            local = np.empty((cnt.value, 3), np.int32)
            check(lib.plato_mesh_file_side_set(h, k, name, 256, _ptr(cells), _ptr(local), C.byref(cnt)))
            side_sets[name.value.decode()] = (cells, local)
        return MeshFile(coords, conn, node_sets, side_sets)
    finally:
        lib.plato_mesh_file_close(h)


def box_mesh(nx: int, ny: int, nz: int, lx: float = 1.0, ly: float = 1.0, lz: float = 1.0) -> BoxMesh:
    nn, nc = C.c_int32(0), C.c_int32(0)
    check(lib.plato_box_mesh_sizes(nx, ny, nz, C.byref(nn), C.byref(nc)))
    coords = np.empty((nn.value, 3), dtype=np.float64)
    conn = np.empty((nc.value, 4), dtype=np.int32)
    check(lib.plato_box_mesh_tet4(nx, ny, nz, lx, ly, lz, _ptr(coords), _ptr(conn)))
    return BoxMesh(nx, ny, nz, lx, ly, lz, coords, conn)
