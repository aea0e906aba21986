"""Pins the CPU oracle to the reference's own gold vectors (unit_tests/DerivativeTests.cpp).

Mesh: 2x2x2 TET4 unit cube from the library's box generator (the BamG numbering the golds
imply); E = 1e6, nu = 0.3, SIMP p = 1, rho_min = 0, z = 1, u_i = 1e-4 (i + 1).
Tolerances are the reference test's own.
"""
import numpy as np
import pytest

from helpers import assert_floating_equality, derivative_test_state, load_golden
from oracle import Oracle
from platoanalyze_b200.mesh import box_mesh

G = load_golden()


@pytest.fixture(scope="module")
def cube():
    mesh = box_mesh(2, 2, 2)
    orc = Oracle(mesh.coords, mesh.connectivity, E=1.0e6, nu=0.3, p=1.0, rho_min=0.0)
    u = derivative_test_state(mesh.num_nodes)
    z = np.ones(mesh.num_nodes)
    return mesh, orc, u, z


def test_mesh_sizes(cube):
    mesh, *_ = cube
    assert mesh.num_nodes == 27 and mesh.num_cells == 48


def test_cell_gradients_strain_stress_residual(cube):
    """DerivativeTests.3D (DerivativeTests.cpp:155-237)."""
    _, orc, u, _ = cube
    g, vol, eps, sig, res = orc.cell_fields(u)
    assert_floating_equality(g[:6], np.reshape(G["cell_gradients"], (6, 4, 3)), 1e-13, zero_abs=1e-12)
    assert_floating_equality(eps[:6], np.reshape(G["cell_strain"], (6, 6)), 1e-13, zero_abs=1e-12)
    assert_floating_equality(sig[:6], np.reshape(G["cell_stress"], (6, 6)), 1e-13, zero_abs=1e-12)
    assert_floating_equality(res[:2], np.reshape(G["cell_residual"], (2, 12)), 1e-13, zero_abs=1e-12)
    np.testing.assert_allclose(vol, 0.5 ** 3 / 6.0, rtol=1e-15)


def test_residual(cube):
    """ElastostaticResidual3D value (DerivativeTests.cpp:339-367)."""
    _, orc, u, z = cube
    assert_floating_equality(orc.vf_value(u, z), G["residual"], 1e-13, zero_abs=1e-11)


def test_jacobian_first_entries(cube):
    """ElastostaticResidual3D gradient_u (DerivativeTests.cpp:386-395), tol 1e-15."""
    _, orc, u, z = cube
    K = orc.vf_gradient_u(u, z)
    assert_floating_equality(K[:36], G["jacobian_entries"], 1e-15)


def test_gradient_z_first_entries(cube):
    """ElastostaticResidual3D gradient_z (DerivativeTests.cpp:411-416), tol 2e-14."""
    _, orc, u, z = cube
    assert_floating_equality(orc.vf_gradient_z(u, z)[:12], G["gradient_z_entries"], 2e-14)


def test_energy_value_and_gradients(cube):
    """InternalElasticEnergy3D (DerivativeTests.cpp:547-596)."""
    _, orc, u, z = cube
    assert_floating_equality([orc.sf_value(u, z)], [G["energy_value"]], 1e-13)
    assert_floating_equality(orc.sf_gradient_u(u, z)[:21], G["energy_gradient_u"], 1e-13, zero_abs=1e-12)
    assert_floating_equality(orc.sf_gradient_z(u, z), G["energy_gradient_z"], 1e-13)


def test_graph_matches_sorted_star(cube):
    """CreateBlockMatrix rows = sorted {nodes sharing a cell} U {self}."""
    mesh, orc, *_ = cube
    rm, cols = orc.graph()
    star = [set() for _ in range(mesh.num_nodes)]
    for c in mesh.connectivity:
        for a in c:
            star[a].update(int(b) for b in c)
    for i in range(mesh.num_nodes):
        assert list(cols[rm[i]:rm[i + 1]]) == sorted(star[i] | {i})


def test_transpose_jacobian_is_transpose(cube):
    _, orc, u, z = cube
    rm, cols = orc.graph()
    K = orc.vf_gradient_u(u, z).reshape(-1, 3, 3)
    KT = orc.vf_gradient_u(u, z, transpose=True).reshape(-1, 3, 3)
    # dense check
    n = rm.size - 1
    D = np.zeros((3 * n, 3 * n))
    DT = np.zeros((3 * n, 3 * n))
    for r in range(n):
        for k in range(rm[r], rm[r + 1]):
            D[3 * r:3 * r + 3, 3 * cols[k]:3 * cols[k] + 3] = K[k]
            DT[3 * r:3 * r + 3, 3 * cols[k]:3 * cols[k] + 3] = KT[k]
    np.testing.assert_allclose(DT, D.T, rtol=0, atol=1e-9 * np.abs(D).max())
