"""Oracle checks beyond the reference golds: finite differences of every derivative, the
linear patch test, the solve against a direct sparse factorisation, the volume criterion."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from helpers import rel_l2
from oracle import Oracle
from platoanalyze_b200.mesh import box_mesh
from platoanalyze_b200.workloads import cantilever, splitmix_uniform


def bsr_to_scipy(rm, cols, vals, n_nodes):
    blocks = vals.reshape(-1, 3, 3)
    return sp.bsr_matrix((blocks, cols, rm), shape=(3 * n_nodes, 3 * n_nodes)).tocsr()


@pytest.fixture(scope="module")
def small():
    spec = cantilever(4, 2, 2)
    orc = Oracle.from_spec(spec)
    z = splitmix_uniform(orc.N, 21, 0.2, 0.9)
    u = np.sin(np.arange(3 * orc.N) * 0.3) * 1e-2
    return spec, orc, z, u


def test_residual_derivatives_by_finite_differences(small):
    spec, orc, z, u = small
    rm, cols = orc.graph()
    K = bsr_to_scipy(rm, cols, orc.vf_gradient_u(u, z), orc.N)
    du = np.cos(np.arange(3 * orc.N))
    eps = 1e-6
    fd = (orc.vf_value(u + eps * du, z) - orc.vf_value(u - eps * du, z)) / (2 * eps)
    assert rel_l2(K @ du, fd) < 1e-8
    G = sp.bsr_matrix((orc.vf_gradient_z(u, z).reshape(-1, 1, 3), cols, rm), shape=(orc.N, 3 * orc.N)).tocsr()
    dz = np.sin(np.arange(orc.N) * 1.7) * 0.05
    # R is cubic in z (SIMP p = 3), so a central difference with a larger step stays exact to
    # rounding, and the step keeps the threaded oracle's summation noise out of the quotient
    eps_z = 1e-4
    fdz = (orc.vf_value(u, z + eps_z * dz) - orc.vf_value(u, z - eps_z * dz)) / (2 * eps_z)
    assert rel_l2(G.T @ dz, fdz) < 1e-7


def test_energy_derivatives_by_finite_differences(small):
    spec, orc, z, u = small
    eps = 1e-6
    du = np.cos(np.arange(3 * orc.N) * 0.9)
    fd = (orc.sf_value(u + eps * du, z) - orc.sf_value(u - eps * du, z)) / (2 * eps)
    assert abs(orc.sf_gradient_u(u, z) @ du - fd) < 1e-8 * abs(fd)
    dz = np.sin(np.arange(orc.N) * 0.4) * 0.05
    fdz = (orc.sf_value(u, z + eps * dz) - orc.sf_value(u, z - eps * dz)) / (2 * eps)
    assert abs(orc.sf_gradient_z(u, z) @ dz - fdz) < 1e-7 * abs(fdz)


def test_compliance_sensitivity_by_finite_differences(small):
    """d/dz of f(u(z), z) with u solved: the self-adjoint and the adjoint-solve gradients."""
    spec, orc, z, _ = small
    dz = np.sin(np.arange(orc.N) * 0.7) * 0.05

    def compliance(zz):
        uu, _, _ = orc.solution_refined(zz, tol=1e-13)
        return orc.sf_value(uu, zz)

    eps = 1e-5
    fd = (compliance(z + eps * dz) - compliance(z - eps * dz)) / (2 * eps)
    u, _, _ = orc.solution_refined(z, tol=1e-13)
    for self_adjoint in (True, False):
        g = orc.criterion_gradient(z, u, self_adjoint=self_adjoint, tol=1e-13)
        assert abs(g @ dz - fd) < 1e-6 * abs(fd), (self_adjoint, g @ dz, fd)


def test_linear_patch():
    """A linear displacement field has constant strain: the internal force vanishes at every
    interior node of a jittered mesh, and the energy equals 1/2 eps.C.eps * volume."""
    m = box_mesh(4, 3, 3, 1.0, 1.0, 1.0)
    rng = np.random.default_rng(3)
    coords = m.coords.copy()
    inner = np.all((coords > 1e-9) & (coords < 1 - 1e-9), axis=1)
    coords[inner] += rng.uniform(-0.05, 0.05, (inner.sum(), 3))
    A = np.array([[1e-3, 2e-4, -3e-4], [5e-4, -2e-3, 1e-4], [0.0, 7e-4, 1.5e-3]])
    u = (coords @ A.T).ravel()
    orc = Oracle(coords, m.connectivity, E=210.0, nu=0.25, p=3.0, rho_min=0.0)
    z = np.ones(m.num_nodes)
    f = orc.sf_gradient_u(u, z).reshape(-1, 3)
    assert np.abs(f[inner]).max() < 1e-12 * np.abs(f).max()
    e = np.array([A[0, 0], A[1, 1], A[2, 2], A[1, 2] + A[2, 1], A[0, 2] + A[2, 0], A[0, 1] + A[1, 0]])
    lam, mu = 210.0 * 0.25 / (1.25 * 0.5), 210.0 / (2 * 1.25)
    C = np.zeros((6, 6))
    C[:3, :3] = lam
    C[np.arange(3), np.arange(3)] += 2 * mu
    C[np.arange(3, 6), np.arange(3, 6)] = mu
    assert orc.sf_value(u, z) == pytest.approx(0.5 * e @ C @ e, rel=1e-12)


def test_solution_matches_direct_factorisation():
    """Config-1 cantilever (z = 0.5): the FP64 PCG at 1e-10 and the refined solve at 1e-13 both
    equal scipy's sparse direct solve; the PCG's stop test is the recomputed FP64 residual."""
    spec = cantilever(20, 10, 10)
    orc = Oracle.from_spec(spec)
    z = np.full(orc.N, 0.5)
    u, st = orc.solution(z, tol=1e-10)
    rm, cols = orc.graph()
    K = orc.vf_gradient_u(np.zeros(3 * orc.N), z)
    b = -orc.vf_value(np.zeros(3 * orc.N), z)
    orc.apply_constraints(K, b, 1.0)
    ud = spla.spsolve(bsr_to_scipy(rm, cols, K, orc.N).tocsc(), b)
    assert st["converged"] == 1 and st["relative_residual"] <= 1e-10
    r = b - orc.matvec_plus(3, 3, K, u, np.zeros(3 * orc.N))
    assert np.linalg.norm(r) <= 1e-10 * np.linalg.norm(b)
    assert rel_l2(u, ud) < 1e-7
    ur, uld, st2 = orc.solution_refined(z, tol=1e-13)
    assert st2["converged"] == 1 and st2["relative_residual"] <= 1e-13
    assert rel_l2(ur, ud) < 1e-10


def test_refinement_reaches_the_extended_precision_tolerance():
    """The long double refinement lowers the residual floor of an FP64 iterate: from a 1e-10
    solve it reaches <= 1e-13 (long double residual), and the refined iterate is closer to the
    direct solution than the FP64 one."""
    spec = cantilever(12, 6, 6)
    orc = Oracle.from_spec(spec)
    z = np.linspace(0.05, 1.0, orc.N)
    n = 3 * orc.N
    K = orc.vf_gradient_u(np.zeros(n), z)
    b = -orc.vf_value(np.zeros(n), z)
    orc.apply_constraints(K, b, 1.0)
    u0, st0 = orc.pcg(K, b, tol=1e-10)
    uld, st = orc.refine(K, b, u0, tol=1e-13, inner_tol=1e-4)
    assert uld.dtype == np.longdouble and st["converged"] == 1 and st["relative_residual"] <= 1e-13
    rm, cols = orc.graph()
    Ks = bsr_to_scipy(rm, cols, K, orc.N).tocsc()
    ud = spla.spsolve(Ks, b)
    # the FP64 direct solution is itself only good to ~1e-12 here: one refinement step with a
    # long double residual makes it the reference the two iterates are measured against
    Kl = Ks.toarray().astype(np.longdouble)
    r = b.astype(np.longdouble) - Kl @ ud.astype(np.longdouble)
    ref = ud.astype(np.longdouble) + spla.spsolve(Ks, r.astype(np.float64)).astype(np.longdouble)
    ref = ref.astype(np.float64)
    assert rel_l2(uld.astype(np.float64), ref) <= rel_l2(u0, ref)


def test_volume_criterion():
    m = box_mesh(3, 2, 2, 1.0, 1.0, 1.0)
    orc = Oracle(m.coords, m.connectivity)
    assert orc.volume_value(np.ones(m.num_nodes), 1.0, 0.0) == pytest.approx(1.0, rel=1e-14)
    z = splitmix_uniform(m.num_nodes, 8, 0.1, 0.9)
    dz = np.cos(np.arange(m.num_nodes))
    eps = 1e-6
    for p, mn in ((1.0, 0.0), (3.0, 1e-3)):
        fd = (orc.volume_value(z + eps * dz, p, mn) - orc.volume_value(z - eps * dz, p, mn)) / (2 * eps)
        g = orc.volume_gradient_z(z, p, mn)
        assert abs(g @ dz - fd) < 1e-8 * np.linalg.norm(g) * np.linalg.norm(dz)
    # linear in z for p = 1: sum of the gradient is the total volume
    assert orc.volume_gradient_z(z, 1.0, 0.0).sum() == pytest.approx(1.0, rel=1e-13)


def test_element_control_derivatives_by_finite_differences(small):
    """Element control (one density per cell): the energy's and the compliance's control
    derivatives per cell against central differences; a uniform field gives the nodal result."""
    spec, _, _, u = small
    orc = Oracle.from_spec(spec, cell_control=True)
    zc = splitmix_uniform(orc.C, 23, 0.2, 0.9)
    eps = 1e-6
    dz = np.sin(np.arange(orc.C) * 0.4) * 0.05
    fdz = (orc.sf_value(u, zc + eps * dz) - orc.sf_value(u, zc - eps * dz)) / (2 * eps)
    g = orc.sf_gradient_z(u, zc)
    assert g.shape == (orc.C,) and abs(g @ dz - fdz) < 1e-7 * abs(fdz)

    def compliance(zz):
        uu, _, _ = orc.solution_refined(zz, tol=1e-13)
        return orc.sf_value(uu, zz)

    fd = (compliance(zc + eps * dz) - compliance(zc - eps * dz)) / (2 * eps)
    us, _, _ = orc.solution_refined(zc, tol=1e-13)
    for self_adjoint in (True, False):
        gc = orc.criterion_gradient(zc, us, self_adjoint=self_adjoint, tol=1e-13)
        assert abs(gc @ dz - fd) < 1e-6 * abs(fd), (self_adjoint, gc @ dz, fd)
    nodal = Oracle.from_spec(spec)
    z_uniform = np.full(orc.N, 0.6)
    assert abs(orc.sf_value(u, np.full(orc.C, 0.6)) - nodal.sf_value(u, z_uniform)) < 1e-14 * nodal.sf_value(u, z_uniform)
