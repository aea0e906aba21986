"""Two-level preconditioner: the Galerkin coarse operator the library assembles equals
(PZ)^T K (PZ) formed here from the assembled Jacobian and the trilinear coarse basis, and the
inverse it applies is E^-1 (Cholesky, diagonal-tile inverses, inverse by doubling)."""
import ctypes as C

import numpy as np
import pytest
import torch

from platoanalyze_b200 import capi
from platoanalyze_b200.capi import check, lib
from platoanalyze_b200.mesh import box_mesh
from platoanalyze_b200.problem import EllipticProblem, SolverOptions, cantilever_spec
from platoanalyze_b200.workloads import splitmix_uniform

pytestmark = pytest.mark.gpu


def coarse_basis(coords, nc):
    lo, hi = coords.min(0), coords.max(0)
    h = (hi - lo) / np.array(nc)
    N = coords.shape[0]
    nn = [n + 1 for n in nc]
    Z = np.zeros((3 * N, 3 * nn[0] * nn[1] * nn[2]))
    for p in range(N):
        t = (coords[p] - lo) / h
        cell = np.clip(np.floor(t).astype(int), 0, np.array(nc) - 1)
        u = t - cell
        for b in range(8):
            off = np.array([(b >> 2) & 1, (b >> 1) & 1, b & 1])
            w = np.prod(np.where(off == 1, u, 1.0 - u))
            J = ((cell[0] + off[0]) * nn[1] + cell[1] + off[1]) * nn[2] + cell[2] + off[2]
            for d in range(3):
                Z[3 * p + d, 3 * J + d] += w
    return Z


@pytest.mark.parametrize("cells,nc", [((8, 4, 4), (4, 2, 2)), ((10, 5, 5), (5, 5, 5))])
def test_galerkin_operator_and_inverse(cells, nc):
    m = box_mesh(*cells, 2.0, 1.0, 1.0)
    opts = SolverOptions(precision=capi.PRECISION_MIXED_FP32, chebyshev_degree=4, coarse_cells=nc)
    spec = cantilever_spec(m, solver=opts)
    prob = EllipticProblem(spec)
    z = splitmix_uniform(m.num_nodes, 61)
    zd = prob.to_dev(z)
    nd = C.c_int32()
    check(lib.plato_coarse_operator(prob.h, C.c_void_p(zd.data_ptr()), C.byref(nd), None, None), prob.h)
    E = np.empty((nd.value, nd.value))
    Einv = np.empty_like(E)
    check(lib.plato_coarse_operator(prob.h, C.c_void_p(zd.data_ptr()), C.byref(nd), E.ctypes.data_as(C.c_void_p),
                                    Einv.ctypes.data_as(C.c_void_p)), prob.h)
    # reference: dense K from the block CRS, masked trilinear basis
    n = 3 * m.num_nodes
    K = np.zeros((n, n))
    rm, cols = (t.cpu().numpy() for t in prob.pattern())
    vals = prob.vf_gradient_u(torch.zeros(n, dtype=torch.float64, device="cuda"), zd).cpu().numpy().reshape(-1, 3, 3)
    for r in range(m.num_nodes):
        for k in range(rm[r], rm[r + 1]):
            K[3 * r:3 * r + 3, 3 * cols[k]:3 * cols[k] + 3] = vals[k]
    Z = coarse_basis(m.coords, nc)
    Z[np.asarray(spec.bc_dofs), :] = 0.0
    Er = Z.T @ K @ Z
    dz = np.diag(Er) <= 0.0
    Er[dz, dz] = 1.0
    assert np.abs(E - Er).max() <= 1e-12 * np.abs(Er).max()
    assert np.abs(E - E.T).max() <= 1e-13 * np.abs(E).max()
    assert np.abs(Einv @ E - np.eye(nd.value)).max() <= 1e-9
    prob.close()


def test_coarse_inverse_bench_grid():
    """The bench's coarse grid (16x8x8 cells, 4131 coarse dofs: 65 tiles of 64, the last one
    35 rows) on a small fine mesh: every step of the look-ahead chain and the ragged last tile.
    Checked by the normwise residual of x = E^-1 b for random b, ||E x - b|| / (||E||_F ||x||): a
    wrong tile gives O(1), rounding gives about n^1.5 eps whatever E's conditioning."""
    m = box_mesh(48, 24, 24, 2.0, 1.0, 1.0)
    opts = SolverOptions(precision=capi.PRECISION_MIXED_FP16, chebyshev_degree=10, coarse_cells=(16, 8, 8))
    prob = EllipticProblem(cantilever_spec(m, solver=opts))
    zd = prob.to_dev(splitmix_uniform(m.num_nodes, 62))
    nd = C.c_int32()
    check(lib.plato_coarse_operator(prob.h, C.c_void_p(zd.data_ptr()), C.byref(nd), None, None), prob.h)
    assert nd.value == 4131
    E = np.empty((nd.value, nd.value))
    Einv = np.empty_like(E)
    check(lib.plato_coarse_operator(prob.h, C.c_void_p(zd.data_ptr()), C.byref(nd), E.ctypes.data_as(C.c_void_p),
                                    Einv.ctypes.data_as(C.c_void_p)), prob.h)
    assert np.abs(E - E.T).max() <= 1e-13 * np.abs(E).max()
    rng = np.random.default_rng(7)
    B = rng.standard_normal((nd.value, 4))
    X = Einv @ B
    backward = np.linalg.norm(E @ X - B, axis=0) / (np.linalg.norm(E) * np.linalg.norm(X, axis=0))
    assert backward.max() <= 1e-10, backward
    prob.close()
