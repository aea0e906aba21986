"""CPU oracle of the Helmholtz density filter (src/helmholtz): the reference's known answer (a
uniform density is left unchanged, unit_tests/PlatoHelmholtzFilterTests.cpp
Helmholtz2DUniformFieldTest, here on the 3D tet mesh), the residual's linearity and
symmetry, the mass total, and the chain rule against finite differences."""
import numpy as np

from oracle import Oracle
from platoanalyze_b200.mesh import box_mesh
from platoanalyze_b200.workloads import splitmix_uniform

L = 0.1


def setup(n=4):
    m = box_mesh(n, max(1, n // 2), max(1, n // 2), 2.0, 1.0, 1.0)
    return m, Oracle(m.coords, m.connectivity)


def test_uniform_density_is_a_fixed_point():
    m, orc = setup(6)
    one = np.ones(m.num_nodes)
    R = orc.helmholtz_value(L, one, one)
    assert np.abs(R).max() <= 1e-15
    f, st = orc.helmholtz_solution(L, one, tol=1e-14)
    assert st["converged"] == 1
    assert np.abs(f - 1.0).max() <= 1e-12


def test_residual_is_K_filtered_minus_M_control():
    m, orc = setup(4)
    rng = np.random.default_rng(3)
    f, c = rng.standard_normal(m.num_nodes), rng.standard_normal(m.num_nodes)
    K, D = orc.helmholtz_gradient_u(L), orc.helmholtz_gradient_z()
    y = np.zeros(m.num_nodes)
    orc.matvec_plus(1, 1, K, f, y)
    orc.matvec_plus(1, 1, D, c, y)
    R = orc.helmholtz_value(L, f, c)
    assert np.abs(R - y).max() <= 1e-13 * np.abs(R).max()
    # the Jacobian and the mass term are symmetric on the pattern; the mass total is -volume
    rm, cols = orc.graph()
    rows = np.repeat(np.arange(m.num_nodes), np.diff(rm))
    A = dict(zip(zip(rows, cols), K))
    assert all(abs(A[(j, i)] - v) <= 1e-15 * abs(v) + 1e-18 for (i, j), v in A.items())
    assert abs(D.sum() + 2.0) <= 1e-12


def test_chain_rule_matches_finite_differences():
    m, orc = setup(4)
    control = splitmix_uniform(m.num_nodes, 17)
    w = np.cos(np.arange(m.num_nodes) * 0.37)  # F(filtered) = w . filtered
    g, st = orc.helmholtz_criterion_gradient(L, w, tol=1e-14)
    assert st["converged"] == 1
    for i in (0, m.num_nodes // 3, m.num_nodes - 1):
        cp, cm = control.copy(), control.copy()
        cp[i] += 1e-3
        cm[i] -= 1e-3
        fp, _ = orc.helmholtz_solution(L, cp, tol=1e-14)
        fm, _ = orc.helmholtz_solution(L, cm, tol=1e-14)
        fd = (w @ fp - w @ fm) / 2e-3
        assert abs(fd - g[i]) <= 1e-9 * max(1.0, abs(fd)), (i, fd, g[i])


def surface(m, alpha, symmetry_sides=()):
    from platoanalyze_b200.mesh import X_MINUS, X_PLUS, Y_MINUS, Y_PLUS, Z_MINUS, Z_PLUS

    sides = [s for s in (X_MINUS, X_PLUS, Y_MINUS, Y_PLUS, Z_MINUS, Z_PLUS) if s not in symmetry_sides]
    cells, local = m.sides(sides)
    return alpha, cells, local


def test_surface_term_total_and_symmetry():
    """With filtered = control = 1 only the surface term is left: sum R = alpha L (area of the
    faces that carry it); with every side a symmetry plane the term vanishes; K stays
    symmetric and R = K filtered + D control still holds."""
    from platoanalyze_b200.mesh import X_MINUS, Y_MINUS, Z_MINUS, exterior_faces

    m, orc = setup(4)
    one = np.ones(m.num_nodes)
    R = orc.helmholtz_value(L, one, one, surface=surface(m, 0.7))
    assert abs(R.sum() - 0.7 * L * 10.0) <= 1e-13  # box 2 x 1 x 1: surface area 10
    R = orc.helmholtz_value(L, one, one, surface=surface(m, 0.7, (X_MINUS, Y_MINUS, Z_MINUS)))
    assert abs(R.sum() - 0.7 * L * 5.0) <= 1e-13  # x = 2, y = 1, z = 1 sides: 1 + 2 + 2
    cells, local = exterior_faces(m.connectivity)
    R2 = orc.helmholtz_value(L, one, one, surface=(0.7, cells, local))
    R1 = orc.helmholtz_value(L, one, one, surface=surface(m, 0.7))
    assert np.abs(R2 - R1).max() <= 1e-15
    rng = np.random.default_rng(8)
    f, c = rng.standard_normal(m.num_nodes), rng.standard_normal(m.num_nodes)
    S = surface(m, 0.4, (X_MINUS,))
    K, D = orc.helmholtz_gradient_u(L, surface=S), orc.helmholtz_gradient_z()
    y = np.zeros(m.num_nodes)
    orc.matvec_plus(1, 1, K, f, y)
    orc.matvec_plus(1, 1, D, c, y)
    R = orc.helmholtz_value(L, f, c, surface=S)
    assert np.abs(R - y).max() <= 1e-13 * np.abs(R).max()
    rm, cols = orc.graph()
    rows = np.repeat(np.arange(m.num_nodes), np.diff(rm))
    A = dict(zip(zip(rows, cols), K))
    assert all(abs(A[(j, i)] - v) <= 1e-15 * abs(v) + 1e-18 for (i, j), v in A.items())
    K0 = orc.helmholtz_gradient_u(L)
    assert np.abs(K - K0).max() > 1e-6 and np.abs(K - K0).sum() > 0


def test_surface_term_balance_and_chain_rule():
    m, orc = setup(4)
    S = surface(m, 1.0)
    one = np.ones(m.num_nodes)
    f, st = orc.helmholtz_solution(L, one, tol=1e-14, surface=S)
    assert st["converged"] == 1
    on_boundary = np.zeros(m.num_nodes, bool)
    on_boundary[np.unique(m.connectivity[S[1][:, None], S[2]])] = True
    assert np.abs(f[on_boundary] - 1.0).max() > 1e-3  # the uniform field is no longer a fixed point
    # balance: 1^T K f = 1^T M 1 with 1^T (stiffness) = 0, so volume - 1^T M f = the surface term
    D = orc.helmholtz_gradient_z()
    Mf = np.zeros(m.num_nodes)
    orc.matvec_plus(1, 1, D, -f, Mf)
    assert abs((2.0 - Mf.sum()) - orc.helmholtz_value(L, f, f, surface=S).sum()) <= 1e-12
    control = splitmix_uniform(m.num_nodes, 19)
    w = np.sin(np.arange(m.num_nodes) * 0.23)
    g, _ = orc.helmholtz_criterion_gradient(L, w, tol=1e-14, surface=S)
    for i in (1, m.num_nodes // 2):
        cp, cm = control.copy(), control.copy()
        cp[i] += 1e-3
        cm[i] -= 1e-3
        fp, _ = orc.helmholtz_solution(L, cp, tol=1e-14, surface=S)
        fm, _ = orc.helmholtz_solution(L, cm, tol=1e-14, surface=S)
        fd = (w @ fp - w @ fm) / 2e-3
        assert abs(fd - g[i]) <= 1e-9 * max(1.0, abs(fd)), (i, fd, g[i])
