"""Learned warm start: the network's BF16 tensor-core kernels against the CPU oracle, Adam,
the subspace (Ritz) initial guess, and what a trained network changes against a zero guess."""
import numpy as np
import pytest
import torch

from helpers import rel_l2
from unet_oracle import LAYERS, UNetOracle, num_params
from platoanalyze_b200.learned import (UNet, design_density, energy_captured, evaluate, generate_training_set,
                                       init_params, subspace_solution, train, unit_load_problems)
from platoanalyze_b200.mesh import box_mesh
from platoanalyze_b200.problem import EllipticProblem, SolverOptions, cantilever_spec

pytestmark = pytest.mark.gpu


def layer_slices():
    out, off = [], 0
    for ci, co, t, _ in LAYERS:
        out.append((slice(off, off + t * co * ci), slice(off + t * co * ci, off + t * co * ci + co)))
        off += t * co * ci + co
    return out


@pytest.mark.parametrize("conv_kernel", [UNet.CONV_TCGEN05, UNet.CONV_MMA_SYNC])
@pytest.mark.parametrize("nodes,batch", [((9, 5, 5), 2), ((6, 7, 5), 1)])
def test_network_matches_oracle(nodes, batch, conv_kernel):
    """Forward output, loss and every layer's weight and bias gradient within BF16-level
    tolerance of the oracle, which rounds to BF16 where the GPU stores BF16, with the tcgen05
    (TMEM accumulator) and the mma.sync convolutions."""
    net = UNet(nodes, batch, conv_kernel=conv_kernel)
    assert net.num_params == num_params()
    rng = np.random.default_rng(4)
    p = init_params(net.num_params, 3) + (0.05 * rng.standard_normal(net.num_params)).astype(np.float32)
    net.set_params(p)
    nn = int(np.prod(nodes))
    inp = rng.uniform(-1, 1, (batch, nn, 8)).astype(np.float32)
    tgt = rng.standard_normal((batch, nn, 9)).astype(np.float32)
    orc = UNetOracle(nodes, bf16=True)
    out = net.forward(torch.tensor(inp).cuda()).cpu().numpy()
    out_o = orc.forward(p.astype(np.float64), inp.reshape((batch,) + nodes + (8,))).reshape(batch, nn, 9)
    assert rel_l2(out, out_o) <= 1e-2, rel_l2(out, out_o)
    loss, g = net.loss_and_gradients(torch.tensor(inp).cuda(), torch.tensor(tgt).cuda(), want_grads=True)
    loss_o, g_o = orc.loss_and_gradients(p.astype(np.float64), inp.reshape((batch,) + nodes + (8,)),
                                         tgt.reshape((batch,) + nodes + (9,)))
    assert abs(loss - loss_o) <= 1e-2 * loss_o
    g = g.cpu().numpy()
    assert rel_l2(g, g_o) <= 2e-2, rel_l2(g, g_o)
    for k, (ws, bs) in enumerate(layer_slices()):
        assert rel_l2(g[ws], g_o[ws]) <= 5e-2, (k, rel_l2(g[ws], g_o[ws]))
        assert rel_l2(g[bs], g_o[bs]) <= 5e-2, (k, rel_l2(g[bs], g_o[bs]))


@pytest.mark.parametrize("nodes,batch", [((13, 7, 9), 3), ((65, 33, 33), 8)])
def test_tcgen05_and_mma_sync_convolutions_agree(nodes, batch):
    """The two convolution kernel families on one network: forward outputs and parameter
    gradients agree to FP32 summation order (BF16 activations rounded alike), and no
    tensor-core wait ran out.  The small grid's position count is not a multiple of the
    128-position tile at any level; on the 65x33x33 grid at batch 8 (the training size) the
    persistent tcgen05 CTAs run several tiles each on the two finer levels, through every
    pipeline depth their shared-memory plans choose."""
    rng = np.random.default_rng(8)
    nn = int(np.prod(nodes))
    inp = torch.tensor(rng.uniform(-1, 1, (batch, nn, 8)).astype(np.float32)).cuda()
    tgt = torch.tensor(rng.standard_normal((batch, nn, 9)).astype(np.float32)).cuda()
    outs, grads, p = [], [], None
    for kind in (UNet.CONV_TCGEN05, UNet.CONV_MMA_SYNC):
        net = UNet(nodes, batch, conv_kernel=kind)
        if p is None:
            p = init_params(net.num_params, 5) + (0.05 * rng.standard_normal(net.num_params)).astype(np.float32)
        net.set_params(p)
        outs.append(net.forward(inp).cpu().numpy())
        _, g = net.loss_and_gradients(inp, tgt, want_grads=True)
        net.check()
        grads.append(g.cpu().numpy())
        net.close()
    assert np.all(np.isfinite(outs[0])) and np.abs(outs[0]).max() > 0
    assert rel_l2(outs[0], outs[1]) <= 5e-3, rel_l2(outs[0], outs[1])
    assert rel_l2(grads[0], grads[1]) <= 1e-2, rel_l2(grads[0], grads[1])


def test_adam_first_step():
    net = UNet((5, 5, 5), 1)
    p = init_params(net.num_params, 5)
    net.set_params(p)
    rng = np.random.default_rng(1)
    inp = torch.tensor(rng.uniform(-1, 1, (1, 125, 8)).astype(np.float32)).cuda()
    tgt = torch.tensor(rng.standard_normal((1, 125, 9)).astype(np.float32)).cuda()
    _, g = net.loss_and_gradients(inp, tgt, want_grads=True)
    g = g.cpu().numpy()
    net.adam_step(1e-3, 1)
    p1 = net.get_params()
    expect = p - 1e-3 * g / (np.abs(g) + 1e-8)  # step 1: m_hat = g, v_hat = g^2
    assert np.allclose(p1, expect, rtol=1e-5, atol=1e-7)


@pytest.fixture(scope="module")
def small_cantilever():
    n = 16
    rng = np.random.default_rng(9)
    z = design_density(n, 0.4, rng)
    opts = SolverOptions(tolerance=1e-10, max_iterations=20000)
    probs = unit_load_problems(n, opts)
    zd = probs[0].to_dev(z)
    W = torch.stack([p.solution(zd)[0] for p in probs])
    tr = np.array([0.3, -0.8, 0.5])
    tr /= np.linalg.norm(tr)
    spec = cantilever_spec(box_mesh(n, n // 2, n // 2, 2.0, 1.0, 1.0), traction=tuple(tr), solver=opts)
    return EllipticProblem(spec), spec, zd, W, tr


def test_exact_subspace_solves_at_once(small_cantilever):
    prob, spec, zd, W, tr = small_cantilever
    u_ref, st_ref = prob.solution(zd)
    u, st, ratio = subspace_solution(prob, zd, W)
    assert ratio < 1e-6
    assert st["converged"] == 1 and st["iterations"] <= st_ref["iterations"] // 10
    assert rel_l2(u.cpu().numpy(), u_ref.cpu().numpy()) <= 1e-8
    # the combination the Ritz step finds is the traction itself, and holds all the energy
    assert rel_l2((tr[0] * W[0] + tr[1] * W[1] + tr[2] * W[2]).cpu().numpy(), u_ref.cpu().numpy()) <= 1e-8
    assert abs(energy_captured(prob, zd, W, u_ref, spec.bc_dofs) - 1.0) <= 1e-8


def test_random_and_degenerate_subspaces(small_cantilever):
    prob, spec, zd, W, _ = small_cantilever
    u_ref, st_ref = prob.solution(zd)
    Wr = torch.randn((4, prob.num_dofs), dtype=torch.float64, device="cuda")
    u, st, ratio = subspace_solution(prob, zd, Wr)
    assert st["converged"] == 1 and ratio <= 10.0
    assert rel_l2(u.cpu().numpy(), u_ref.cpu().numpy()) <= 1e-7
    Wz = torch.zeros((2, prob.num_dofs), dtype=torch.float64, device="cuda")
    u, st, ratio = subspace_solution(prob, zd, Wz)  # singular Gram matrix: zero guess kept
    assert ratio == 1.0 and st["iterations"] == st_ref["iterations"]


def test_trained_network_end_to_end():
    """Generate data with the solver, train on 16x8x8 cantilever designs for a few seconds,
    and run the learned guess on held-out designs: the loss falls, the answer is unchanged
    (both solves stop at ||r|| <= 1e-8 ||b||), and the measured change in iterations and the
    energy fraction the learned subspace captures are printed."""
    n = 16
    designs, X, Y, info = generate_training_set(96, n=n, seed=11, method="plain", log=None)
    assert info["solves"] == 288
    net = UNet((n + 1, n // 2 + 1, n // 2 + 1), 8)
    net.set_params(init_params(net.num_params, 2))
    hist = train(net, X, Y, epochs=40, batch=8, lr=2e-3, log=None)
    assert hist[-1] < 0.7 * hist[0]
    rng = np.random.default_rng(123)
    test = [design_density(n, rng.uniform(0.2, 0.6), rng) for _ in range(6)]
    trs = [v / np.linalg.norm(v) for v in rng.standard_normal((6, 3))]
    rows = evaluate(net, n, test, trs, "plain")
    assert all(r["u_rel_diff"] <= 1e-4 and r["u_rel_diff_deflated"] <= 1e-4 for r in rows)
    assert all(0.0 <= r["energy_captured"] <= 1.0 + 1e-9 for r in rows)
    it0 = np.mean([r["iterations"] for r in rows])
    it1 = np.mean([r["iterations_learned"] for r in rows])
    it2 = np.mean([r["iterations_deflated"] for r in rows])
    gain = {"iterations_zero_guess": it0, "iterations_learned_guess": it1, "iterations_learned_deflation": it2,
            "energy_captured": float(np.mean([r["energy_captured"] for r in rows]))}
    print(f"learned gain on held-out 16x8x8 designs (plain Jacobi-PCG to 1e-8): {gain}")
    # what the network gains is measured, not assumed: the deflated solve reaches the same
    # answer, and neither the guess nor the deflation may cost more than a few iterations
    assert it1 <= it0 + 5 and it2 <= it0 + 5, gain


def test_deflation_by_responses_of_a_nearby_design(small_cantilever):
    """Deflated CG with the unit-load responses of a different (uniform) design: smooth global
    bending modes.  The deflated solve reaches the plain solve's answer in fewer iterations
    than both the zero guess and the Galerkin guess alone."""
    prob, spec, zd, W, tr = small_cantilever
    n = 16
    opts = SolverOptions(tolerance=1e-10, max_iterations=20000)
    probs = unit_load_problems(n, opts)
    zu = probs[0].to_dev(np.full(prob.num_nodes, 0.5))
    Wn = torch.stack([p.solution(zu)[0] for p in probs])
    u_ref, st_ref = prob.solution(zd)
    u_g, st_g, _ = subspace_solution(prob, zd, Wn)
    u_d, st_d, _ = prob.solution_deflated(zd, Wn)
    assert st_d["converged"] == 1 and rel_l2(u_d.cpu().numpy(), u_ref.cpu().numpy()) <= 1e-8
    print(f"iterations: zero guess {st_ref['iterations']}, Galerkin guess {st_g['iterations']}, "
          f"deflated {st_d['iterations']}")
    assert st_d["iterations"] < st_ref["iterations"] and st_d["iterations"] <= st_g["iterations"]
    # with the exact responses the deflated solve, like the guess, is done at once
    u_e, st_e, _ = prob.solution_deflated(zd, W)
    assert st_e["iterations"] <= st_ref["iterations"] // 10
    assert rel_l2(u_e.cpu().numpy(), u_ref.cpu().numpy()) <= 1e-8
