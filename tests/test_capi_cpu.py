"""Host-side checks that need no GPU: the C ABI library loads and exports every symbol its
header declares, and the box-mesh generator produces the expected topology."""
import ctypes as C
import re
from pathlib import Path

import numpy as np

from platoanalyze_b200 import capi
from platoanalyze_b200.mesh import X_MINUS, X_PLUS, Y_MINUS, Z_PLUS, box_mesh

ROOT = Path(__file__).resolve().parents[1]


def header_symbols():
    txt = (ROOT / "include" / "plato_b200.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\*?\s+\*?(plato_[a-z0-9_]+)\s*\(", txt, re.M)))


def test_library_exports_every_declared_symbol():
    syms = header_symbols()
    assert len(syms) >= 25, syms
    lib = C.CDLL(str(capi.LIB_PATH))
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_create_rejects_bad_input_without_touching_device():
    # null description -> BAD_INPUT before any CUDA call
    h = C.c_void_p()
    rc = capi.lib.plato_create(None, C.byref(h))
    assert rc == capi.BAD_INPUT
    assert b"null" in capi.lib.plato_last_error(None)


def test_box_mesh_topology():
    m = box_mesh(3, 2, 4, 2.0, 1.0, 1.0)
    assert m.num_nodes == 4 * 3 * 5 and m.num_cells == 6 * 3 * 2 * 4
    assert m.connectivity.min() == 0 and m.connectivity.max() == m.num_nodes - 1
    # every tet has positive volume of h^3/6
    X = m.coords[m.connectivity]
    J = X[:, :3, :] - X[:, 3:4, :]
    vol = np.abs(np.linalg.det(J)) / 6.0
    np.testing.assert_allclose(vol, (2.0 / 3) * (1.0 / 2) * (1.0 / 4) / 6.0, rtol=1e-12)
    # side sets: 2 triangles per boundary quad
    for face, nq in ((X_MINUS, 2 * 4), (X_PLUS, 2 * 4), (Y_MINUS, 3 * 4), (Z_PLUS, 3 * 2)):
        cells, local = m.sideset(face)
        assert cells.size == 2 * nq
        axis, side = face // 2, face % 2
        coord = m.coords[m.connectivity[cells[:, None], local], axis]
        target = [2.0, 1.0, 1.0][axis] if side else 0.0
        np.testing.assert_allclose(coord, target)
    ns = m.nodeset(X_MINUS)
    assert ns.size == 3 * 5 and np.all(m.coords[ns, 0] == 0.0)


def test_box_mesh_rejects_bad_sizes():
    nn, nc = C.c_int32(), C.c_int32()
    assert capi.lib.plato_box_mesh_sizes(0, 1, 1, C.byref(nn), C.byref(nc)) == capi.BAD_INPUT
    assert capi.lib.plato_box_mesh_sizes(5000, 5000, 5000, C.byref(nn), C.byref(nc)) == capi.BAD_INPUT
