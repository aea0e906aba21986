"""Batched solves: one handle over the disjoint union of independent problems.

Every member of a batch must give what its own handle gives: the same block pattern (offset),
residual and Jacobian entries, a solution converged to its own tolerance, its compliance and
dC/dz; members converge independently (their own iteration counts and stop tests).
"""
import numpy as np
import torch
import pytest

from helpers import rel_l2
from oracle import Oracle
from platoanalyze_b200 import capi
from platoanalyze_b200.mesh import box_mesh
from platoanalyze_b200.problem import EllipticProblem, SolverOptions, cantilever_spec
from platoanalyze_b200.workloads import batch_workload, grf_density

pytestmark = pytest.mark.gpu

OPTS = SolverOptions(tolerance=1e-11, max_iterations=20000, precision=capi.PRECISION_MIXED_FP32,
                     chebyshev_degree=6)


def host(t):
    return t.detach().cpu().numpy()


def members(sizes, seed, opts=OPTS, zero_load=()):
    rng = np.random.default_rng(seed)
    specs, zs = [], []
    for k, n in enumerate(sizes):
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        if k in zero_load:
            d = np.zeros(3)
        m = box_mesh(n, max(1, n // 2), max(1, n // 2), 2.0, 1.0, 1.0)
        specs.append(cantilever_spec(m, traction=tuple(d), solver=opts))
        zs.append(grf_density(n, max(1, n // 2), max(1, n // 2), rng=rng))
    return specs, zs


@pytest.fixture(scope="module")
def batch5():
    specs, zs = members([6, 4, 8, 4, 10], 5)
    bp = EllipticProblem.batch(specs)
    singles = [EllipticProblem(s) for s in specs]
    return specs, zs, bp, singles


def test_offsets_and_pattern(batch5):
    specs, zs, bp, singles = batch5
    assert bp.count == len(specs)
    assert np.array_equal(np.diff(bp.node_offsets), [s.coords.shape[0] for s in specs])
    assert np.array_equal(np.diff(bp.cell_offsets), [s.connectivity.shape[0] for s in specs])
    rm, cols = (host(t) for t in bp.pattern())
    for s, p in enumerate(singles):
        rms, colss = (host(t) for t in p.pattern())
        a, b = bp.node_offsets[s], bp.node_offsets[s + 1]
        assert np.array_equal(rm[a:b + 1] - rm[a], rms)
        assert np.array_equal(cols[rm[a]:rm[b]] - a, colss)


def test_residual_and_jacobian_match_members(batch5):
    specs, zs, bp, singles = batch5
    z = np.concatenate(zs)
    u = np.sin(np.arange(bp.num_dofs) * 0.37)
    ud, zd = bp.to_dev(u), bp.to_dev(z)
    R = host(bp.vf_value(ud, zd))
    K = host(bp.vf_gradient_u(ud, zd))
    rm = host(bp.pattern()[0])
    for s, (p, sl) in enumerate(zip(singles, bp.member_slices())):
        Rs = host(p.vf_value(p.to_dev(u[sl]), p.to_dev(zs[s])))
        assert rel_l2(R[sl], Rs) <= 1e-14
        Ks = host(p.vf_gradient_u(p.to_dev(u[sl]), p.to_dev(zs[s])))
        a, b = bp.node_offsets[s], bp.node_offsets[s + 1]
        assert rel_l2(K[9 * rm[a]:9 * rm[b]], Ks) <= 1e-14


def test_batched_solve_matches_member_solves(batch5):
    specs, zs, bp, singles = batch5
    z = np.concatenate(zs)
    zd = bp.to_dev(z)
    u, st = bp.solution(zd)
    assert st["converged"] == 1
    per = bp.batch_last_stats()
    assert all(m["converged"] == 1 and m["relative_residual"] <= 1e-10 for m in per)
    iters = [m["iterations"] for m in per]
    assert st["iterations"] == max(iters)
    assert len(set(iters)) > 1  # members stop on their own tests
    uh = host(u)
    f = bp.batch_criterion_values(zd, u)
    g = host(bp.criterion_gradient(zd, u)[0])
    for s, (p, sl) in enumerate(zip(singles, bp.member_slices())):
        zs_d = p.to_dev(zs[s])
        us, sts = p.solution(zs_d)
        assert sts["converged"] == 1
        assert rel_l2(uh[sl], host(us)) <= 1e-8, s
        fs = p.criterion_value(zs_d, us)
        assert abs(f[s] - fs) <= 1e-8 * abs(fs), s
        gs = host(p.criterion_gradient(zs_d, us)[0])
        a, b = bp.node_offsets[s], bp.node_offsets[s + 1]
        assert rel_l2(g[a:b], gs) <= 1e-8, s
    # the union's energy is the sum of the members'
    assert abs(bp.criterion_value(zd, u) - f.sum()) <= 1e-12 * abs(f.sum())


def test_batched_solution_matches_oracle():
    specs, zs = members([4, 6, 4], 11)
    bp = EllipticProblem.batch(specs)
    u, st = bp.solution(bp.to_dev(np.concatenate(zs)))
    assert st["converged"] == 1
    uh = host(u)
    for s, sl in enumerate(bp.member_slices()):
        orc = Oracle.from_spec(specs[s])
        uo, _, _ = orc.solution_refined(zs[s], tol=1e-13)
        assert rel_l2(uh[sl], uo) <= 1e-8, s


def test_zero_load_member_converges_at_once():
    specs, zs = members([6, 4, 6], 3, zero_load=(1,))
    bp = EllipticProblem.batch(specs)
    u, st = bp.solution(bp.to_dev(np.concatenate(zs)))
    per = bp.batch_last_stats()
    assert st["converged"] == 1
    assert per[1]["iterations"] == 0
    assert np.all(host(u)[bp.member_slices()[1]] == 0.0)
    assert per[0]["iterations"] > 0 and per[2]["iterations"] > 0


def test_explicit_adjoint_matches_self_adjoint_in_batch():
    opts = SolverOptions(tolerance=1e-11, max_iterations=20000, precision=capi.PRECISION_MIXED_FP32,
                         chebyshev_degree=6, self_adjoint=False)
    specs, zs = members([4, 6], 8, opts=opts)
    bp = EllipticProblem.batch(specs)
    zd = bp.to_dev(np.concatenate(zs))
    u, _ = bp.solution(zd)
    g_adj, st = bp.criterion_gradient(zd, u)
    assert st["converged"] == 1
    bp.set_solver(SolverOptions(tolerance=1e-11, max_iterations=20000, precision=capi.PRECISION_MIXED_FP32,
                                chebyshev_degree=6, self_adjoint=True))
    g_sa, _ = bp.criterion_gradient(zd, u)
    assert rel_l2(host(g_adj), host(g_sa)) <= 1e-8


def test_jacobi_and_bf16_batches_converge():
    for opts in (SolverOptions(tolerance=1e-10, max_iterations=20000),
                 SolverOptions(tolerance=1e-10, max_iterations=20000, precision=capi.PRECISION_MIXED_BF16,
                               chebyshev_degree=8)):
        specs, zs = members([4, 6, 5], 21, opts=opts)
        bp = EllipticProblem.batch(specs)
        u, st = bp.solution(bp.to_dev(np.concatenate(zs)))
        assert st["converged"] == 1 and st["relative_residual"] <= 1e-9


def test_unsupported_batch_options():
    specs, _ = members([4, 4], 1, opts=SolverOptions(coarse_cells=(2, 1, 1), precision=capi.PRECISION_MIXED_FP32,
                                                     chebyshev_degree=4))
    with pytest.raises(capi.PlatoError) as e:
        EllipticProblem.batch(specs)
    assert e.value.status == capi.NOT_SUPPORTED
    specs, _ = members([4, 4], 1)
    bp = EllipticProblem.batch(specs)
    with pytest.raises(capi.PlatoError) as e:
        bp.set_solver(SolverOptions(operator_kind=capi.OPERATOR_MATRIX_FREE))
    assert e.value.status == capi.NOT_SUPPORTED


def test_mixed_material_rejected():
    specs, _ = members([4, 4], 1)
    specs[1].youngs_modulus = 2.0
    with pytest.raises(capi.PlatoError) as e:
        EllipticProblem.batch(specs)
    assert e.value.status == capi.BAD_INPUT


def test_batch_workload_small_draw():
    specs, zs, ns = batch_workload(count=6, sizes=(4, 6, 8), solver=OPTS)
    bp = EllipticProblem.batch(specs)
    u, st = bp.solution(bp.to_dev(np.concatenate(zs)))
    assert st["converged"] == 1
    assert len(bp.batch_last_stats()) == 6


def test_autotuned_persistent_batch_with_graphs_matches_members():
    """The autotuner times every (tile rows, CTAs per SM) pair and keeps the fastest; a batch
    on a non-default stream (chunks captured as CUDA graphs) with the chosen tiling gives every
    member the answer of its own handle."""
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        specs, zs = members([6, 10, 4, 8, 12, 6], 21)
        bp = EllipticProblem.batch(specs, stream=stream)
        zd = bp.to_dev(np.concatenate(zs))
        tuning = bp.batch_autotune(zd)
        assert tuning["tile_rows"] in (128, 256, 512) and tuning["ctas_per_sm"] in (2, 4, 8, 16)
        assert len(tuning["tried"]) == 12 and all(t["ms"] > 0 for t in tuning["tried"])
        assert min(t["ms"] for t in tuning["tried"]) == pytest.approx(
            [t["ms"] for t in tuning["tried"] if t["tile_rows"] == tuning["tile_rows"]
             and t["ctas_per_sm"] == tuning["ctas_per_sm"]][0])
        u, st = bp.solution(zd)
        assert st["converged"] == 1
        uh = host(u)
        for s, sl in enumerate(bp.member_slices()):
            single = EllipticProblem(specs[s], stream=stream)
            us, sts = single.solution(single.to_dev(zs[s]))
            assert sts["converged"] == 1
            assert rel_l2(uh[sl], host(us)) <= 1e-8, s
            single.close()
        bp.close()
    torch.cuda.synchronize()
