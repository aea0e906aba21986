"""Matrix-free operator and the polynomial-preconditioned / mixed-precision solvers.

The FP64 plain method is the oracle-checked reference (tests/test_gpu_parity.py).  Every
other solver configuration must reach the same FP64 tolerance (the stop test is always the
FP64 residual) and land within 1e-8 of the CPU oracle's solution; reduced precision may
only change the iteration count.
"""
import numpy as np
import pytest

from helpers import rel_l2
from oracle import Oracle
from platoanalyze_b200 import capi
from platoanalyze_b200.problem import EllipticProblem, ProblemSpec, SolverOptions
from platoanalyze_b200.workloads import cantilever, splitmix_uniform

pytestmark = pytest.mark.gpu

CONFIGS = {
    "fp64_cheb8": SolverOptions(precision=capi.PRECISION_FP64, chebyshev_degree=8),
    "fp32_cheb8": SolverOptions(precision=capi.PRECISION_MIXED_FP32, chebyshev_degree=8),
    "bf16_cheb8": SolverOptions(precision=capi.PRECISION_MIXED_BF16, chebyshev_degree=8),
    "mf_fp64_jacobi": SolverOptions(operator_kind=capi.OPERATOR_MATRIX_FREE, precision=capi.PRECISION_FP64,
                                    chebyshev_degree=1),
    "mf_fp32_cheb8": SolverOptions(operator_kind=capi.OPERATOR_MATRIX_FREE, precision=capi.PRECISION_MIXED_FP32,
                                   chebyshev_degree=8),
    "fp32_cheb4_coarse": SolverOptions(precision=capi.PRECISION_MIXED_FP32, chebyshev_degree=4,
                                       coarse_cells=(5, 5, 5)),
    "bf16_cheb4_coarse": SolverOptions(precision=capi.PRECISION_MIXED_BF16, chebyshev_degree=4,
                                       coarse_cells=(10, 5, 5)),
    "fp16s_cheb8": SolverOptions(precision=capi.PRECISION_MIXED_FP16, chebyshev_degree=8),
    "fp16s_cheb8_coarse": SolverOptions(precision=capi.PRECISION_MIXED_FP16, chebyshev_degree=8,
                                        coarse_cells=(10, 5, 5)),
    "mf_fp32asm_cheb8": SolverOptions(operator_kind=capi.OPERATOR_MATRIX_FREE,
                                      precision=capi.PRECISION_MIXED_FP32_ASSEMBLED, chebyshev_degree=8),
    "mf_fp32asm_cheb4_coarse": SolverOptions(operator_kind=capi.OPERATOR_MATRIX_FREE,
                                             precision=capi.PRECISION_MIXED_FP32_ASSEMBLED, chebyshev_degree=4,
                                             coarse_cells=(10, 5, 5)),
    "mf_fp32_cheb4_coarse": SolverOptions(operator_kind=capi.OPERATOR_MATRIX_FREE,
                                          precision=capi.PRECISION_MIXED_FP32, chebyshev_degree=4,
                                          coarse_cells=(4, 2, 2)),
}


def host(t):
    return t.detach().cpu().numpy()


@pytest.fixture(scope="module")
def setup():
    spec = cantilever(20, 10, 10, SolverOptions(tolerance=1e-10))
    z = splitmix_uniform(spec.coords.shape[0], 0x5EED0003)
    prob = EllipticProblem(spec)
    orc = Oracle.from_spec(spec)
    uo, _, _ = orc.solution_refined(z, tol=1e-13)
    go = orc.criterion_gradient(z, uo)
    return spec, z, prob, orc, uo, go


def constrained_matvec(orc, z, x):
    K = orc.vf_gradient_u(np.zeros(3 * orc.N), z)
    rhs = np.zeros(3 * orc.N)
    orc.apply_constraints(K, rhs, 0.0)
    return orc.matvec_plus(3, 3, K, x, np.zeros(3 * orc.N))


@pytest.mark.parametrize("kind", [capi.OPERATOR_ASSEMBLED, capi.OPERATOR_MATRIX_FREE])
def test_operator_apply_matches_oracle(setup, kind):
    spec, z, prob, orc, *_ = setup
    x = np.sin(np.arange(3 * orc.N) * 0.7)
    y = host(prob.apply_operator(prob.to_dev(z), prob.to_dev(x), kind))
    ref = constrained_matvec(orc, z, x)
    assert rel_l2(y, ref) <= 1e-12, rel_l2(y, ref)


def test_matrix_free_on_perturbed_mesh():
    from test_gpu_parity import perturbed_mesh
    coords, conn = perturbed_mesh(5, 4, 4, 3)
    fixed = np.where(coords[:, 0] < 1e-12)[0]
    dofs = (3 * fixed[:, None] + np.arange(3)).ravel().astype(np.int32)
    spec = ProblemSpec(coords, conn, 1.7, 0.21, 3.0, 1e-9, [], dofs, np.linspace(0, 1e-3, dofs.size))
    prob, orc = EllipticProblem(spec), Oracle.from_spec(spec)
    z = splitmix_uniform(coords.shape[0], 5)
    x = np.cos(np.arange(3 * coords.shape[0]))
    y = host(prob.apply_operator(prob.to_dev(z), prob.to_dev(x), capi.OPERATOR_MATRIX_FREE))
    assert rel_l2(y, constrained_matvec(orc, z, x)) <= 1e-12


@pytest.mark.parametrize("name", list(CONFIGS))
def test_solver_configuration_reaches_fp64_answer(setup, name):
    spec, z, prob, orc, uo, go = setup
    opts = CONFIGS[name]
    opts.tolerance = 1e-10
    prob.set_solver(opts)
    try:
        zd = prob.to_dev(z)
        u, st = prob.solution(zd)
        g, _ = prob.criterion_gradient(zd, u)
    finally:
        prob.set_solver(SolverOptions(tolerance=1e-10))
    assert st["converged"] == 1 and st["relative_residual"] <= 1e-10, st
    assert rel_l2(host(u), uo) <= 1e-8, rel_l2(host(u), uo)
    assert rel_l2(host(g), go) <= 1e-8, rel_l2(host(g), go)


def test_chebyshev_reduces_outer_iterations(setup):
    spec, z, prob, *_ = setup
    zd = prob.to_dev(z)
    _, plain = prob.solution(zd)
    prob.set_solver(SolverOptions(tolerance=1e-10, precision=capi.PRECISION_MIXED_FP32, chebyshev_degree=8))
    try:
        _, poly = prob.solution(zd)
    finally:
        prob.set_solver(SolverOptions(tolerance=1e-10))
    assert poly["iterations"] * 3 < plain["iterations"], (poly, plain)


def test_coarse_space_cuts_iterations(setup):
    spec, z, prob, *_ = setup
    zd = prob.to_dev(z)
    prob.set_solver(SolverOptions(tolerance=1e-10, precision=capi.PRECISION_MIXED_FP32, chebyshev_degree=4))
    try:
        _, one = prob.solution(zd)
        prob.set_solver(SolverOptions(tolerance=1e-10, precision=capi.PRECISION_MIXED_FP32, chebyshev_degree=4,
                                      coarse_cells=(10, 5, 5)))
        _, two = prob.solution(zd)
    finally:
        prob.set_solver(SolverOptions(tolerance=1e-10))
    assert two["converged"] == 1 and two["iterations"] * 2 < one["iterations"], (one, two)


def test_coarse_grid_must_align():
    spec = cantilever(6, 3, 3, SolverOptions(tolerance=1e-10, precision=capi.PRECISION_MIXED_FP32,
                                             chebyshev_degree=4, coarse_cells=(4, 2, 2)))
    prob = EllipticProblem(spec)
    with pytest.raises(capi.PlatoError) as e:
        prob.solution(prob.to_dev(np.full(spec.coords.shape[0], 0.5)))
    assert e.value.status == capi.BAD_INPUT and "straddles" in str(e.value)


def test_inhomogeneous_dirichlet_matrix_free_matches_assembled():
    spec = cantilever(6, 3, 3, SolverOptions(tolerance=1e-11))
    spec.bc_values = np.linspace(-1e-3, 2e-3, spec.bc_dofs.size)
    z = splitmix_uniform(spec.coords.shape[0], 17)
    orc = Oracle.from_spec(spec)
    uo, _, _ = orc.solution_refined(z, tol=1e-13)
    for opts in (SolverOptions(tolerance=1e-11),
                 SolverOptions(tolerance=1e-11, operator_kind=capi.OPERATOR_MATRIX_FREE,
                               precision=capi.PRECISION_MIXED_FP32, chebyshev_degree=6)):
        spec.solver = opts
        prob = EllipticProblem(spec)
        u, st = prob.solution(prob.to_dev(z))
        assert st["converged"] == 1
        assert rel_l2(host(u), uo) <= 1e-8


@pytest.mark.parametrize("kind", [capi.OPERATOR_ASSEMBLED, capi.OPERATOR_MATRIX_FREE])
def test_failed_flexible_cg_falls_back_to_plain_fp64(setup, kind):
    """A flexible-CG method that cannot meet the tolerance within its iteration cap hands the
    solve to the plain FP64 Jacobi-PCG (from a zero guess, with its own cap); the answer is the
    FP64 one.  With the fallback switched off the status is PLATO_NOT_CONVERGED."""
    spec, z, prob, orc, uo, go = setup
    zd = prob.to_dev(z)
    opts = SolverOptions(tolerance=1e-10, max_iterations=2, operator_kind=kind,
                         precision=capi.PRECISION_MIXED_FP32, chebyshev_degree=4, fallback_max_iterations=100000)
    prob.set_solver(opts)
    try:
        u, st = prob.solution(zd)
        assert st["converged"] == 1 and st["fallback"] == 2 and st["relative_residual"] <= 1e-10, st
        assert rel_l2(host(u), uo) <= 1e-8
        opts.fallback_max_iterations = -1
        prob.set_solver(opts)
        u, st = prob.solution(zd, raise_on_error=False)
        assert st["rc"] == capi.NOT_CONVERGED and st["fallback"] == 0 and st["converged"] == 0
    finally:
        prob.set_solver(SolverOptions(tolerance=1e-10))


def test_fallback_after_a_subspace_guess(setup):
    """With a subspace (learned) guess the method is first retried from a zero guess; when that
    fails too the plain FP64 method finishes the solve."""
    spec, z, prob, orc, uo, go = setup
    zd = prob.to_dev(z)
    prob.set_solver(SolverOptions(tolerance=1e-10, max_iterations=2, precision=capi.PRECISION_MIXED_FP32,
                                  chebyshev_degree=4, fallback_max_iterations=100000))
    try:
        W = np.stack([np.sin(np.arange(3 * orc.N) * 0.01 * (k + 1)) for k in range(3)])
        u, st, _ = prob.solution_subspace(zd, prob.to_dev(W))
        assert st["converged"] == 1 and st["fallback"] == 2, st
        assert rel_l2(host(u), uo) <= 1e-8
    finally:
        prob.set_solver(SolverOptions(tolerance=1e-10))


def test_fp32_element_assembly_matches_the_fp64_matrix(setup):
    """The FP32 element assembly of the preconditioner matrix: the solve with it reaches the
    FP64 answer (the outer operator is the FP64 matrix-free apply), and its inverse diagonal
    (the preconditioner's Jacobi scaling) agrees with the FP64 matrix's to FP32 accuracy."""
    spec, z, prob, orc, uo, go = setup
    zd = prob.to_dev(z)
    prob.set_solver(SolverOptions(tolerance=1e-10, operator_kind=capi.OPERATOR_MATRIX_FREE,
                                  precision=capi.PRECISION_MIXED_FP32_ASSEMBLED, chebyshev_degree=8))
    try:
        u, st = prob.solution(zd)
        assert st["converged"] == 1 and st["fallback"] == 0 and rel_l2(host(u), uo) <= 1e-8
    finally:
        prob.set_solver(SolverOptions(tolerance=1e-10))
    with pytest.raises(capi.PlatoError):  # only with the matrix-free FP64 operator
        prob.set_solver(SolverOptions(precision=capi.PRECISION_MIXED_FP32_ASSEMBLED, chebyshev_degree=8))
    prob.set_solver(SolverOptions(tolerance=1e-10))


def test_fp16_sweep_column_offsets_and_their_fallback():
    """The FP16 sweep reads 16-bit column offsets when the numbering keeps every column within
    32767 of its slice and 32-bit columns otherwise (a randomly relabelled 70,785-node mesh).
    Both layouts solve the same problem to the same answer."""
    from platoanalyze_b200.workloads import coarse_grid, method_options
    cells = (64, 32, 32)
    opts = method_options("two-level-fp16", 1e-11, coarse_grid(*cells))
    spec = cantilever(*cells, opts)
    N = spec.coords.shape[0]
    rng = np.random.default_rng(11)
    perm = rng.permutation(N).astype(np.int32)
    coords = np.empty_like(spec.coords)
    coords[perm] = spec.coords
    bc = 3 * perm[spec.bc_dofs // 3] + spec.bc_dofs % 3
    spec_p = ProblemSpec(coords, perm[spec.connectivity].astype(np.int32), spec.youngs_modulus,
                         spec.poissons_ratio, spec.penalty_exponent, spec.penalty_minimum, spec.tractions,
                         bc.astype(np.int32), spec.bc_values, opts)
    a, b = EllipticProblem(spec), EllipticProblem(spec_p)
    assert a.sell_info()["column_bytes"] == 2
    assert b.sell_info()["column_bytes"] == 4
    z = splitmix_uniform(N, 0x5EED0002)
    zp = np.empty_like(z)
    zp[perm] = z
    ua, sa = a.solution(a.to_dev(z))
    ub, sb = b.solution(b.to_dev(zp))
    assert sa["converged"] == 1 and sb["converged"] == 1
    assert sa["relative_residual"] <= 1e-11 and sb["relative_residual"] <= 1e-11
    uah = host(ua).reshape(-1, 3)
    ubh = host(ub).reshape(-1, 3)[perm]
    assert rel_l2(ubh, uah) <= 1e-8, rel_l2(ubh, uah)
    a.close()
    b.close()


@pytest.mark.parametrize("cells", [(20, 10, 10), (40, 20, 20)])
def test_multistep_sweep_matches_one_launch_per_step(cells):
    """The multi-step FP16 sweep (several Chebyshev steps per launch, each step waiting only
    for its neighbouring tiles of the step before) does the same arithmetic per row as one
    launch per step: the same iterations and the same solution, for launch lengths that do and
    do not divide the degree and for a one-tile lag."""
    spec = cantilever(*cells, SolverOptions(tolerance=1e-10))
    z = splitmix_uniform(spec.coords.shape[0], 0x5EED0003)
    prob = EllipticProblem(spec)
    orc = Oracle.from_spec(spec)
    uo, _, _ = orc.solution_refined(z, tol=1e-13)
    zd = prob.to_dev(z)
    coarse = (cells[0] // 10, cells[1] // 10, cells[2] // 10)
    results = {}
    for steps, lag in ((1, 0), (2, 0), (3, 0), (4, 0), (7, 1), (16, 0), (0, 0), (5, 300)):
        prob.set_solver(SolverOptions(tolerance=1e-10, precision=capi.PRECISION_MIXED_FP16, chebyshev_degree=9,
                                      chebyshev_ratio=100.0, coarse_cells=coarse, sweep_steps=steps,
                                      sweep_lag=lag))
        u, st = prob.solution(zd)
        info = prob.sweep_info()
        assert st["converged"] == 1 and st["fallback"] == 0, (steps, st)
        assert info["steps_per_launch"] == max(1, steps)
        assert rel_l2(host(u), uo) <= 1e-8
        results[(steps, lag)] = (st["iterations"], host(u))
    it1, u1 = results[(1, 0)]
    for key, (it, u) in results.items():
        assert it == it1, (key, it, it1)
        assert rel_l2(u, u1) <= 1e-14, key
    prob.close()


def test_multistep_sweep_wait_runs_out_and_falls_back(setup):
    """A multi-step sweep launch whose dependency wait can never be met (the test hook makes it
    wait for a stamp no task writes) gives up after its bounded wait, the host reads the
    timeout, the solve is finished by the plain FP64 fallback with the oracle's answer, later
    solves on the handle run one launch per step, and the device stays usable."""
    from platoanalyze_b200.problem import lib

    spec, z, _, orc, uo, _ = setup
    prob = EllipticProblem(spec)
    zd = prob.to_dev(z)
    prob.set_solver(SolverOptions(tolerance=1e-10, precision=capi.PRECISION_MIXED_FP16, chebyshev_degree=8,
                                  coarse_cells=(10, 5, 5), sweep_steps=4))
    u, st = prob.solution(zd)
    assert st["converged"] == 1 and st["fallback"] == 0 and prob.sweep_info()["steps_per_launch"] == 4
    assert lib.plato_test_stall_next_sweep(prob.h) == 0
    u, st = prob.solution(zd)
    assert st["converged"] == 1 and st["fallback"] == 2, st
    assert rel_l2(host(u), uo) <= 1e-8
    u, st = prob.solution(zd)
    assert st["converged"] == 1 and st["fallback"] == 0 and prob.sweep_info()["steps_per_launch"] == 1
    assert rel_l2(host(u), uo) <= 1e-8
    prob.close()
