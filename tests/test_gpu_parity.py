"""Parity of the CUDA path (through the C ABI) with the CPU oracle and the reference golds.

Bars: block pattern bit-exact; residual, Jacobian entries, (dR/dz)^T entries, energy and its
gradients within 1e-11 relative of the oracle (norm-wise, and entry-wise against the
largest entry); solves to the requested FP64 tolerance with the solution within 1e-8 of a
tight oracle solve.
"""
import numpy as np
import pytest

from helpers import assert_floating_equality, derivative_test_state, load_golden, rel_l2
from oracle import Oracle
from platoanalyze_b200 import capi
from platoanalyze_b200.mesh import box_mesh
from platoanalyze_b200.problem import EllipticProblem, ProblemSpec, SolverOptions
from platoanalyze_b200.workloads import cantilever, splitmix_uniform

pytestmark = pytest.mark.gpu
G = load_golden()
TOL = 1e-11


def close(gpu, ref, tol=TOL):
    gpu = np.asarray(gpu, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    scale = np.abs(ref).max() if ref.size else 1.0
    assert rel_l2(gpu, ref) <= tol, rel_l2(gpu, ref)
    assert np.abs(gpu - ref).max() <= tol * max(scale, 1e-300), np.abs(gpu - ref).max() / scale


def host(t):
    return t.detach().cpu().numpy()


@pytest.fixture(scope="module")
def cube():
    mesh = box_mesh(2, 2, 2)
    spec = ProblemSpec(mesh.coords, mesh.connectivity, 1.0e6, 0.3, 1.0, 0.0)
    prob = EllipticProblem(spec)
    u = derivative_test_state(mesh.num_nodes)
    z = np.ones(mesh.num_nodes)
    return mesh, prob, Oracle.from_spec(spec), u, z


@pytest.fixture(scope="module")
def small():
    """20x10x10 cantilever with seeded nodal densities (seed 0x5EED0003)."""
    spec = cantilever(20, 10, 10, SolverOptions(tolerance=1e-10))
    z = splitmix_uniform(spec.coords.shape[0], 0x5EED0003)
    prob = EllipticProblem(spec)
    return spec, prob, Oracle.from_spec(spec), z


def perturbed_mesh(nx, ny, nz, seed):
    """Box mesh with jittered interior coordinates and randomly relabelled nodes."""
    m = box_mesh(nx, ny, nz, 1.3, 0.7, 0.9)
    rng = np.random.default_rng(seed)
    coords = m.coords.copy()
    h = np.array([1.3 / nx, 0.7 / ny, 0.9 / nz])
    interior = np.all((coords > 1e-12) & (coords < np.array([1.3, 0.7, 0.9]) - 1e-12), axis=1)
    coords[interior] += rng.uniform(-0.15, 0.15, (interior.sum(), 3)) * h
    perm = rng.permutation(m.num_nodes).astype(np.int32)
    new_coords = np.empty_like(coords)
    new_coords[perm] = coords
    conn = perm[m.connectivity]
    return new_coords, conn.astype(np.int32)


# ---- reference golds on the 2x2x2 cube ---------------------------------------------------

def test_golden_residual_jacobian_gradz(cube):
    mesh, prob, orc, u, z = cube
    ud, zd = prob.to_dev(u), prob.to_dev(z)
    assert_floating_equality(host(prob.vf_value(ud, zd)), G["residual"], 1e-13, zero_abs=1e-11)
    # closed-form K_e vs the reference's AD: 1e-13 (reference tolerance 1e-15 is for AD order)
    assert_floating_equality(host(prob.vf_gradient_u(ud, zd))[:36], G["jacobian_entries"], 1e-13, zero_abs=1e-9)
    assert_floating_equality(host(prob.vf_gradient_z(ud, zd))[:12], G["gradient_z_entries"], 2e-14)


def test_golden_energy(cube):
    mesh, prob, orc, u, z = cube
    ud, zd = prob.to_dev(u), prob.to_dev(z)
    assert_floating_equality([prob.sf_value(ud, zd)], [G["energy_value"]], 1e-13)
    assert_floating_equality(host(prob.sf_gradient_u(ud, zd))[:21], G["energy_gradient_u"], 1e-13, zero_abs=1e-11)
    assert_floating_equality(host(prob.sf_gradient_z(ud, zd)), G["energy_gradient_z"], 1e-13)


# ---- pattern ---------------------------------------------------------------------------------

@pytest.mark.parametrize("which", ["cube", "small", "perturbed"])
def test_pattern_bit_exact(which, cube, small):
    if which == "cube":
        prob, orc = cube[1], cube[2]
    elif which == "small":
        prob, orc = small[1], small[2]
    else:
        coords, conn = perturbed_mesh(5, 4, 3, 7)
        spec = ProblemSpec(coords, conn)
        prob, orc = EllipticProblem(spec), Oracle.from_spec(ProblemSpec(coords, conn))
    rm, cols = prob.pattern()
    orm, ocols = orc.graph()
    assert np.array_equal(host(rm), orm)
    assert np.array_equal(host(cols), ocols)


# ---- element kernels on a seeded problem -----------------------------------------------------

def test_residual_and_jacobian(small):
    spec, prob, orc, z = small
    u = np.sin(np.arange(3 * orc.N) * 0.37) * 1e-2
    ud, zd = prob.to_dev(u), prob.to_dev(z)
    close(host(prob.vf_value(ud, zd)), orc.vf_value(u, z))
    close(host(prob.vf_gradient_u(ud, zd)), orc.vf_gradient_u(u, z))
    close(host(prob.vf_gradient_u_T(ud, zd)), orc.vf_gradient_u(u, z, transpose=True))
    close(host(prob.vf_gradient_z(ud, zd)), orc.vf_gradient_z(u, z))


def test_energy_and_gradients(small):
    spec, prob, orc, z = small
    u = np.cos(np.arange(3 * orc.N) * 0.11) * 1e-2
    ud, zd = prob.to_dev(u), prob.to_dev(z)
    assert abs(prob.sf_value(ud, zd) - orc.sf_value(u, z)) <= TOL * abs(orc.sf_value(u, z))
    close(host(prob.sf_gradient_u(ud, zd)), orc.sf_gradient_u(u, z))
    close(host(prob.sf_gradient_z(ud, zd)), orc.sf_gradient_z(u, z))


def test_gradient_z_apply_matches_matrix(small):
    spec, prob, orc, z = small
    u = np.cos(np.arange(3 * orc.N) * 0.21) * 1e-2
    lam = np.sin(np.arange(3 * orc.N) * 0.05)
    ud, zd, ld = prob.to_dev(u), prob.to_dev(z), prob.to_dev(lam)
    out = prob.zeros(orc.N)
    prob.vf_gradient_z_apply(ud, zd, ld, out)
    ref = orc.matvec_plus(1, 3, orc.vf_gradient_z(u, z), lam, np.zeros(orc.N))
    close(host(out), ref)


def test_perturbed_mesh_kernels():
    coords, conn = perturbed_mesh(6, 5, 4, 11)
    spec = ProblemSpec(coords, conn, 2.5, 0.27, 3.0, 1e-9)
    prob, orc = EllipticProblem(spec), Oracle.from_spec(spec)
    z = splitmix_uniform(coords.shape[0], 99)
    u = np.sin(np.arange(3 * coords.shape[0]) * 0.3)
    ud, zd = prob.to_dev(u), prob.to_dev(z)
    close(host(prob.vf_value(ud, zd)), orc.vf_value(u, z))
    close(host(prob.vf_gradient_u(ud, zd)), orc.vf_gradient_u(u, z))
    close(host(prob.vf_gradient_z(ud, zd)), orc.vf_gradient_z(u, z))
    close(host(prob.sf_gradient_z(ud, zd)), orc.sf_gradient_z(u, z))


def test_constraints_and_matvec(small):
    spec, prob, orc, z = small
    u = np.zeros(3 * orc.N)
    ud, zd = prob.to_dev(u), prob.to_dev(z)
    K = prob.vf_gradient_u(ud, zd)
    rhs = prob.to_dev(np.linspace(-1, 1, 3 * orc.N))
    prob.apply_constraints(K, rhs, 1.0)
    Ko = orc.vf_gradient_u(u, z)
    rhso = np.linspace(-1, 1, 3 * orc.N)
    orc.apply_constraints(Ko, rhso, 1.0)
    close(host(K), Ko)
    close(host(rhs), rhso)
    x = np.cos(np.arange(3 * orc.N))
    y = prob.matvec_plus(3, 3, K, prob.to_dev(x), prob.to_dev(np.ones(3 * orc.N)))
    close(host(y), orc.matvec_plus(3, 3, Ko, x, np.ones(3 * orc.N)))


# ---- solve, compliance, sensitivity -------------------------------------------------------

def test_solution_compliance_gradient(small):
    spec, prob, orc, z = small
    zd = prob.to_dev(z)
    u, st = prob.solution(zd)
    assert st["converged"] == 1 and st["relative_residual"] <= 1e-10, st
    uo, _, sto = orc.solution_refined(z, tol=1e-13)
    assert rel_l2(host(u), uo) <= 1e-8, rel_l2(host(u), uo)
    # criterion and sensitivity are functions of (u, z): compare on the GPU state at 1e-11
    uh = host(u)
    f = prob.criterion_value(zd, u)
    assert abs(f - orc.sf_value(uh, z)) <= TOL * abs(f)
    g, _ = prob.criterion_gradient(zd, u)
    close(host(g), orc.criterion_gradient(z, uh, self_adjoint=True))


def test_explicit_adjoint_matches_self_adjoint(small):
    spec, prob, orc, z = small
    zd = prob.to_dev(z)
    u, _ = prob.solution(zd)
    g_sa, _ = prob.criterion_gradient(zd, u)
    prob.set_solver(SolverOptions(tolerance=1e-12, self_adjoint=False))
    try:
        g_adj, st = prob.criterion_gradient(zd, u)
    finally:
        prob.set_solver(SolverOptions(tolerance=1e-10))
    assert st["converged"] == 1 and st["iterations"] > 0
    assert rel_l2(host(g_adj), host(g_sa)) <= 1e-8
    ref = orc.criterion_gradient(z, host(u), self_adjoint=False, tol=1e-12)
    assert rel_l2(host(g_adj), ref) <= 1e-8


def test_host_entry_point_matches_device_path(small):
    spec, prob, orc, z = small
    u_h, f_h, g_h, st = prob.solve_and_gradient_host(z)
    zd = prob.to_dev(z)
    u, _ = prob.solution(zd)
    g, _ = prob.criterion_gradient(zd, u)
    assert rel_l2(u_h, host(u)) <= 1e-13
    assert rel_l2(g_h, host(g)) <= 1e-13
    assert abs(f_h - prob.criterion_value(zd, u)) <= 1e-13 * abs(f_h)


def test_warm_start_takes_fewer_iterations(small):
    spec, prob, orc, z = small
    zd = prob.to_dev(z)
    u, st0 = prob.solution(zd)
    u1, st1 = prob.solution(zd, u0=u)
    assert st1["iterations"] <= 2 and st1["converged"] == 1


# ---- edge cases --------------------------------------------------------------------------------

def test_zero_load_gives_zero_state():
    spec = cantilever(4, 2, 2)
    spec.tractions = []
    prob = EllipticProblem(spec)
    z = np.full(spec.coords.shape[0], 0.7)
    u, st = prob.solution(prob.to_dev(z))
    assert st["converged"] == 1 and st["iterations"] == 0
    assert float(u.abs().max()) == 0.0


def test_nonfinite_control_reports_status():
    spec = cantilever(4, 2, 2)
    prob = EllipticProblem(spec)
    z = np.full(spec.coords.shape[0], 0.5)
    z[3] = np.nan
    u, st = prob.solution(prob.to_dev(z), raise_on_error=False)
    assert st["rc"] == capi.NONFINITE


def test_iteration_limit_reports_not_converged():
    spec = cantilever(8, 4, 4, SolverOptions(tolerance=1e-12, max_iterations=3))
    prob = EllipticProblem(spec)
    u, st = prob.solution(prob.to_dev(np.full(spec.coords.shape[0], 0.5)), raise_on_error=False)
    assert st["rc"] == capi.NOT_CONVERGED and st["iterations"] == 3


def fan_mesh(k):
    """Tets (0, pole, ring_j, ring_j+1) around a vertical axis through node 0, above and below
    the ring: node 0 has 2k cells and k + 3 blocks, each pole k cells."""
    t = 2 * np.pi * np.arange(k) / k
    ring = np.stack([np.cos(t), np.sin(t), 0.1 * np.sin(3 * t)], axis=1)
    coords = np.vstack([[0.0, 0.0, 0.0], [0.1, 0.0, 1.0], [0.0, 0.1, -1.0], ring])
    cells = []
    for j in range(k):
        a, b = 3 + j, 3 + (j + 1) % k
        cells.append([0, 1, a, b])
        cells.append([0, 2, b, a])
    return coords, np.asarray(cells, dtype=np.int32)


@pytest.mark.parametrize("k", [12, 14, 20, 40])
def test_high_valence_rows(k):
    """Node 0 has k + 2 upper blocks: up to 15 (k = 12) the thread-per-row kernel assembles it,
    beyond that it is a wide row of the warp-per-row kernel, which also writes the transposes
    of its upper blocks into the narrow ring rows -- in registers while the row has at most
    32 incident cells and blocks (k = 14), with global atomics beyond (k = 20, 40).  All must
    match the oracle."""
    coords, conn = fan_mesh(k)
    spec = ProblemSpec(coords, conn, 1.7, 0.31, 3.0, 1e-9)
    prob, orc = EllipticProblem(spec), Oracle.from_spec(spec)
    z = splitmix_uniform(coords.shape[0], 7 + k)
    u = np.cos(np.arange(3 * coords.shape[0]) * 0.7)
    ud, zd = prob.to_dev(u), prob.to_dev(z)
    rm, cols = orc.graph()
    rmg, colsg = (host(t) for t in prob.pattern())
    assert np.array_equal(rmg, rm) and np.array_equal(colsg, cols)
    close(host(prob.vf_gradient_u(ud, zd)), orc.vf_gradient_u(u, z))
    close(host(prob.vf_gradient_z(ud, zd)), orc.vf_gradient_z(u, z))
    close(host(prob.vf_value(ud, zd)), orc.vf_value(u, z))


def test_bad_connectivity_rejected():
    m = box_mesh(2, 2, 2)
    conn = m.connectivity.copy()
    conn[5, 2] = conn[5, 1]  # repeated node in a cell
    with pytest.raises(capi.PlatoError) as e:
        EllipticProblem(ProblemSpec(m.coords, conn))
    assert e.value.status == capi.BAD_INPUT
    conn = m.connectivity.copy()
    conn[0, 0] = m.num_nodes  # out of range
    with pytest.raises(capi.PlatoError):
        EllipticProblem(ProblemSpec(m.coords, conn))


def test_volume_criterion(small):
    spec, prob, orc, z = small
    zd = prob.to_dev(z)
    for p, m in ((1.0, 0.0), (3.0, 1e-3)):
        v = prob.volume_value(zd, p, m)
        assert abs(v - orc.volume_value(z, p, m)) <= TOL * abs(v)
        close(host(prob.volume_gradient_z(zd, p, m)), orc.volume_gradient_z(z, p, m))
    assert prob.volume_value(prob.to_dev(np.ones(orc.N)), 1.0, 0.0) == pytest.approx(2.0, rel=1e-13)


def test_fused_criterion_value_and_gradient(small):
    """plato_problem_criterion_value_and_gradient (one pass) gives exactly what the two calls
    give: the same energy sum order and the same per-cell sensitivities."""
    spec, prob, orc, z = small
    u = np.cos(np.arange(3 * orc.N) * 0.11) * 1e-2
    ud, zd = prob.to_dev(u), prob.to_dev(z)
    f, g, st = prob.criterion_value_and_gradient(zd, ud)
    assert f == prob.criterion_value(zd, ud)
    g2, _ = prob.criterion_gradient(zd, ud)
    assert np.array_equal(host(g), host(g2))
    assert abs(f - orc.sf_value(u, z)) <= TOL * abs(f)
    close(host(g), orc.criterion_gradient(z, u, self_adjoint=True))
