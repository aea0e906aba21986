"""Learned warm start for elliptic SIMP solves on box cantilevers (no reference counterpart).

A 3-level 3D U-Net (16-32-64 channels, BF16 tensor-core kernels in csrc/unet.cu) maps a
design - nodal density on the node grid of a 64 x 32 x 32 hex mesh (65 x 33 x 33 nodes) plus
load-face / clamp-face masks, coordinates and the SIMP stiffness scale - to 9 fields per
node: the displacement responses to unit tractions along x, y and z on the loaded face.  Any
end-face traction's response lies in their span, so the three predicted fields form a
subspace W; the solve then starts from the Galerkin (Ritz) guess on span(W)
(plato_problem_solution_subspace), which falls back to the plain guess when it would blow up
the residual, and runs to the same FP64 tolerance, so the network changes the iteration count
only.  Finer box meshes of the same shape (e.g. 160 x 80 x 80) get their density resampled to
the network grid and W interpolated back trilinearly.

Training data: FP64 solves (tolerance 1e-8) of the solver itself on Gaussian-random-field
designs with volume fractions in [0.2, 0.6], three unit-load solves per design, each
response scaled to unit RMS (the Ritz step makes the guess independent of scale).

    python -m platoanalyze_b200.learned --designs 667 --epochs 40 --out weights.npz
"""
from __future__ import annotations

import ctypes as C
import time
from pathlib import Path

import numpy as np

from . import capi
from .capi import check, lib
from .mesh import box_mesh
from .problem import EllipticProblem, SolverOptions, cantilever_spec
from .workloads import grf_field

NET_NODES = (65, 33, 33)
WEIGHTS = Path(__file__).resolve().parent / "data" / "unet_cantilever_64x32x32.npz"


def _ucheck(rc: int):
    if rc != capi.OK:
        msg = lib.plato_unet_last_error()
        raise capi.PlatoError(rc, msg.decode() if msg else "")


def _i3(v):
    return (C.c_int32 * 3)(*[int(x) for x in v])


class UNet:
    """The warm-start network on a fixed node grid (device parameters, FP32 + BF16 copies)."""

    CONV_TCGEN05, CONV_MMA_SYNC = 0, 1

    def __init__(self, nodes=NET_NODES, max_batch: int = 8, stream=None, conv_kernel: int = 0):
        import torch

        self.torch = torch
        self.nodes = tuple(int(v) for v in nodes)
        self.max_batch = max_batch
        self.h = C.c_void_p()
        _ucheck(lib.plato_unet_create(_i3(self.nodes), max_batch, C.byref(self.h)))
        self.stream = stream if stream is not None else torch.cuda.current_stream()
        _ucheck(lib.plato_unet_set_stream(self.h, C.c_void_p(self.stream.cuda_stream)))
        _ucheck(lib.plato_unet_set_conv_kernel(self.h, conv_kernel))
        n = C.c_int64()
        _ucheck(lib.plato_unet_num_params(self.h, C.byref(n)))
        self.num_params = n.value
        self.num_nodes = int(np.prod(self.nodes))

    def check(self):
        """Waits for the network's stream; raises when a tensor-core convolution timed out."""
        _ucheck(lib.plato_unet_check(self.h))

    def close(self):
        if getattr(self, "h", None):
            lib.plato_unet_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ptr(self, t):
        return C.c_void_p(t.data_ptr())

    def set_params(self, params):
        t = self.torch.as_tensor(np.asarray(params, np.float32)).cuda()
        _ucheck(lib.plato_unet_set_params(self.h, self._ptr(t)))
        self.torch.cuda.synchronize()

    def get_params(self) -> np.ndarray:
        t = self.torch.empty(self.num_params, dtype=self.torch.float32, device="cuda")
        _ucheck(lib.plato_unet_get_params(self.h, self._ptr(t)))
        return t.cpu().numpy()

    def forward(self, inp):
        B = inp.shape[0]
        out = self.torch.empty((B, self.num_nodes, 9), dtype=self.torch.float32, device="cuda")
        _ucheck(lib.plato_unet_forward(self.h, B, self._ptr(inp), self._ptr(out)))
        return out

    def loss_and_gradients(self, inp, tgt, want_grads: bool = False):
        B = inp.shape[0]
        loss = C.c_double()
        g = self.torch.empty(self.num_params, dtype=self.torch.float32, device="cuda") if want_grads else None
        _ucheck(lib.plato_unet_loss_and_gradients(self.h, B, self._ptr(inp), self._ptr(tgt), C.byref(loss),
                                                  self._ptr(g) if g is not None else None))
        return loss.value, g

    def adam_step(self, lr: float, step: int):
        _ucheck(lib.plato_unet_adam_step(self.h, C.c_float(lr), int(step)))

    def features(self, z, src_nodes):
        """Network input [1][nodes][8] for nodal density z (FP64 device) on the src_nodes grid."""
        f = self.torch.empty((1, self.num_nodes, 8), dtype=self.torch.float32, device="cuda")
        _ucheck(lib.plato_unet_features(_i3(src_nodes), self._ptr(z), _i3(self.nodes), self._ptr(f),
                                        C.c_void_p(self.stream.cuda_stream)))
        return f

    def subspace(self, out, dst_nodes):
        """The 3 subspace columns [3][3 * prod(dst_nodes)] (FP64) from one network output."""
        n = int(np.prod(dst_nodes))
        W = self.torch.empty((3, 3 * n), dtype=self.torch.float64, device="cuda")
        _ucheck(lib.plato_unet_subspace(_i3(self.nodes), self._ptr(out), _i3(dst_nodes), self._ptr(W),
                                        C.c_void_p(self.stream.cuda_stream)))
        return W

    def save(self, path, **meta):
        path = Path(path)
        path.parent.mkdir(parents=True, exist_ok=True)
        np.savez_compressed(path, params=self.get_params(), nodes=np.asarray(self.nodes),
                            **{k: np.asarray(v) for k, v in meta.items()})

    @classmethod
    def load(cls, path=WEIGHTS, max_batch: int = 1, stream=None) -> "UNet":
        d = np.load(path)
        net = cls(tuple(int(v) for v in d["nodes"]), max_batch, stream)
        net.set_params(d["params"])
        return net


def init_params(num_params: int, seed: int = 0) -> np.ndarray:
    """He-normal weights, zero biases (the layer table of csrc/unet.cu)."""
    layers = [(16, 16, 27, 1), (16, 16, 27, 1), (16, 32, 27, 1), (32, 32, 27, 1), (32, 64, 27, 1), (64, 64, 27, 1),
              (96, 32, 27, 1), (32, 32, 27, 1), (48, 16, 27, 1), (16, 16, 27, 1), (16, 9, 1, 0)]
    rng = np.random.default_rng(seed)
    parts = []
    for ci, co, t, relu in layers:
        std = np.sqrt((2.0 if relu else 1.0) / (t * ci))
        parts += [rng.standard_normal(t * co * ci) * std, np.zeros(co)]
    p = np.concatenate(parts).astype(np.float32)
    assert p.size == num_params
    return p


# ---- designs and training data ------------------------------------------------------------

def design_density(n: int, vf: float, rng: np.random.Generator, sharpness: float = 0.25) -> np.ndarray:
    """A GRF design on the (n+1)(n/2+1)^2 nodes with mean density vf: the standardised field g
    (correlation length 0.1) mapped through logistic((g - t) / sharpness), t by bisection,
    clipped to [0.01, 1]."""
    g = grf_field(n, n // 2, n // 2, rng=rng)
    lo, hi = -6.0, 6.0
    for _ in range(60):
        t = 0.5 * (lo + hi)
        z = np.clip(1.0 / (1.0 + np.exp(-(g - t) / sharpness)), 0.01, 1.0)
        if z.mean() > vf:
            lo = t
        else:
            hi = t
    return z


def solver_for(n: int, method: str = "two-level", tol: float = 1e-8) -> SolverOptions:
    """Plain FP64 Jacobi-PCG, or the two-level mixed-precision method with a coarse box grid
    that aligns with the n x n/2 x n/2 mesh and keeps the dense coarse solve small."""
    if method == "plain":
        return SolverOptions(tolerance=tol, max_iterations=200000)
    coarse = (0, 0, 0)
    if n % 16 == 0 and 3 * (n // 8 + 1) * (n // 16 + 1) ** 2 <= 6144:
        coarse = (n // 8, n // 16, n // 16)
    elif n % 10 == 0:
        coarse = (10, 5, 5)
    return SolverOptions(tolerance=tol, max_iterations=200000, precision=capi.PRECISION_MIXED_FP32,
                         chebyshev_degree=8, coarse_cells=coarse)


def unit_load_problems(n: int, opts: SolverOptions):
    """Three handles on the n x n/2 x n/2 cantilever with unit tractions along x, y, z."""
    mesh = box_mesh(n, n // 2, n // 2, 2.0, 1.0, 1.0)
    return [EllipticProblem(cantilever_spec(mesh, traction=tuple(np.eye(3)[d]), solver=opts)) for d in range(3)]


def generate_training_set(count: int, n: int = 64, seed: int = 0x5EED0005, method: str = "two-level",
                          log=print):
    """Designs, network inputs [count][nodes][8] and targets [count][nodes][9] (each unit-load
    response scaled to unit RMS per design), built from 3 unit-load solves per design to the
    FP64-checked tolerance 1e-8."""
    import torch

    probs = unit_load_problems(n, solver_for(n, method))
    nodes = (n + 1, n // 2 + 1, n // 2 + 1)
    rng = np.random.default_rng(seed)
    net = UNet(nodes, 1)
    X = torch.empty((count, int(np.prod(nodes)), 8), dtype=torch.float32, device="cuda")
    Y = torch.empty((count, int(np.prod(nodes)), 9), dtype=torch.float32, device="cuda")
    designs, iters = [], []
    t0 = time.perf_counter()
    for k in range(count):
        vf = rng.uniform(0.2, 0.6)
        z = design_density(n, vf, rng)
        zd = probs[0].to_dev(z)
        cols = []
        for p in probs:
            u, st = p.solution(zd)
            iters.append(st["iterations"])
            cols.append(u.view(-1, 3))
        # [nodes][9]: channel 3d + c, each load direction's response scaled to unit RMS
        Y[k] = torch.cat([c / torch.sqrt(torch.mean(c * c)) for c in cols], dim=1).float()
        X[k] = net.features(zd, nodes)[0]
        designs.append(z)
        if log and (k + 1) % 100 == 0:
            log(f"  {k + 1}/{count} designs, {3 * (k + 1)} solves, {time.perf_counter() - t0:.1f}s")
    net.close()
    for p in probs:
        p.close()
    return designs, X, Y, {"solves": 3 * count, "mean_iterations": float(np.mean(iters)),
                           "seconds": time.perf_counter() - t0}


def train(net: UNet, X, Y, epochs: int = 40, batch: int = 8, lr: float = 2e-3, seed: int = 0, log=print):
    """Adam with a cosine learning-rate schedule over shuffled minibatches; returns losses."""
    rng = np.random.default_rng(seed)
    count = X.shape[0]
    steps_per_epoch = max(1, count // batch)
    total = epochs * steps_per_epoch
    step, hist = 0, []
    t0 = time.perf_counter()
    for ep in range(epochs):
        perm = rng.permutation(count)
        losses = []
        for b in range(steps_per_epoch):
            idx = net.torch.as_tensor(perm[b * batch:(b + 1) * batch], device="cuda")
            loss, _ = net.loss_and_gradients(X[idx].contiguous(), Y[idx].contiguous())
            step += 1
            net.adam_step(lr * 0.5 * (1.0 + np.cos(np.pi * (step - 1) / total)), step)
            losses.append(loss)
        hist.append(float(np.mean(losses)))
        if log:
            log(f"  epoch {ep + 1}/{epochs}: loss {hist[-1]:.4e} ({time.perf_counter() - t0:.1f}s)")
    return hist


# ---- inference ------------------------------------------------------------------------------

def learned_subspace(net: UNet, zd, src_nodes, smooth_passes: int = 0):
    """The 3 subspace columns for a design on the src_nodes grid; smooth_passes 7-point
    averaging passes on the network grid first damp node-scale noise of the prediction,
    which dominates its energy norm."""
    torch = net.torch
    out = net.forward(net.features(zd, src_nodes))[0].contiguous()
    if smooth_passes > 0:
        scratch = torch.empty_like(out)
        _ucheck(lib.plato_box_smooth(_i3(net.nodes), 9, int(smooth_passes), C.c_void_p(out.data_ptr()),
                                     C.c_void_p(scratch.data_ptr()), C.c_void_p(net.stream.cuda_stream)))
    return net.subspace(out, src_nodes)


def subspace_solution(prob: EllipticProblem, zd, W):
    """plato_problem_solution_subspace from a zero guess; returns (u, stats, residual ratio)."""
    return prob.solution_subspace(zd, W)


def warm_start_solution(prob: EllipticProblem, net: UNet, zd, src_nodes, smooth_passes: int = 0):
    """Problem::solution from the learned Ritz guess; returns (u, stats, residual ratio)."""
    return subspace_solution(prob, zd, learned_subspace(net, zd, src_nodes, smooth_passes))


def energy_captured(prob: EllipticProblem, zd, W, u_star, bc_dofs) -> float:
    """Fraction of the solution's energy norm ||u*||_K^2 held by the Galerkin guess on span(PW)
    (1 = W contains the solution, 0 = K-orthogonal to it); diagnostic, FP64."""
    torch = prob.torch
    Wm = W.clone()
    Wm[:, torch.as_tensor(np.asarray(bc_dofs, np.int64), device="cuda")] = 0.0
    Q = torch.stack([prob.apply_operator(zd, Wm[j].contiguous()) for j in range(Wm.shape[0])])
    b = -prob.vf_value(torch.zeros_like(u_star), zd)  # F (zero on the clamped dofs)
    G = (Wm @ Q.T).cpu().numpy()
    rhs = (Wm @ b).cpu().numpy()
    try:
        c = np.linalg.solve(G, rhs)
    except np.linalg.LinAlgError:
        return 0.0
    return float(c @ G @ c / float(b @ u_star))


def evaluate(net: UNet, n: int, designs, tractions, method: str = "two-level", smooth_passes: int = 0):
    """Iterations and solve time with and without the learned guess on the n x n/2 x n/2 mesh,
    and the energy fraction the learned subspace captures."""
    import torch

    opts = solver_for(n, method)
    mesh = box_mesh(n, n // 2, n // 2, 2.0, 1.0, 1.0)
    nodes = (n + 1, n // 2 + 1, n // 2 + 1)
    rows = []
    for z, tr in zip(designs, tractions):
        spec = cantilever_spec(mesh, traction=tuple(tr), solver=opts)
        prob = EllipticProblem(spec)
        zd = prob.to_dev(z)
        prob.solution(zd)  # warm-up (buffers, coarse buckets)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        u0, st0 = prob.solution(zd)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        u1, st1, ratio = warm_start_solution(prob, net, zd, nodes, smooth_passes)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        W = learned_subspace(net, zd, nodes, smooth_passes)
        torch.cuda.synchronize()
        t3 = time.perf_counter()
        u2, st2, _ = prob.solution_deflated(zd, W)  # the same fields as a deflation subspace
        torch.cuda.synchronize()
        t4 = time.perf_counter()
        rows.append({"iterations": st0["iterations"], "iterations_learned": st1["iterations"],
                     "iterations_deflated": st2["iterations"],
                     "ms": 1e3 * (t1 - t0), "ms_learned": 1e3 * (t2 - t1), "ms_deflated": 1e3 * (t4 - t3),
                     "initial_residual_ratio": ratio,
                     "energy_captured": energy_captured(prob, zd, W, u0, spec.bc_dofs),
                     "u_rel_diff": float(torch.linalg.norm(u1 - u0) / torch.linalg.norm(u0)),
                     "u_rel_diff_deflated": float(torch.linalg.norm(u2 - u0) / torch.linalg.norm(u0))})
        prob.close()
    return rows


def time_kernels(batch: int = 8, steps: int = 10, nodes=NET_NODES) -> int:
    """Forward and training-step (loss, backward) times of the network on random inputs with
    the tcgen05 and the mma.sync convolutions, CUDA events on the network's stream, 3 warm-up
    repetitions; prints one JSON line per kernel family."""
    import json

    import torch

    rng = np.random.default_rng(0)
    nn = int(np.prod(nodes))
    inp = torch.tensor(rng.uniform(-1, 1, (batch, nn, 8)).astype(np.float32)).cuda()
    tgt = torch.tensor(rng.standard_normal((batch, nn, 9)).astype(np.float32)).cuda()
    for kind, name in ((UNet.CONV_TCGEN05, "tcgen05"), (UNet.CONV_MMA_SYNC, "mma.sync")):
        net = UNet(nodes, batch, conv_kernel=kind)
        net.set_params(init_params(net.num_params, 1))
        for _ in range(3):
            net.forward(inp)
            net.loss_and_gradients(inp, tgt)
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        ev[0].record(net.stream)
        for _ in range(steps):
            net.forward(inp)
        ev[1].record(net.stream)
        for _ in range(steps):
            net.loss_and_gradients(inp, tgt)
        ev[2].record(net.stream)
        torch.cuda.synchronize()
        net.check()
        print(json.dumps({"conv_kernel": name, "nodes": list(nodes), "batch": batch,
                          "forward_ms": ev[0].elapsed_time(ev[1]) / steps,
                          "train_step_ms": ev[1].elapsed_time(ev[2]) / steps}), flush=True)
        net.close()
    return 0


def main(argv=None) -> int:
    import argparse

    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("--designs", type=int, default=667)
    ap.add_argument("--test-designs", type=int, default=16)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--out", default=str(WEIGHTS))
    ap.add_argument("--load", default="", help="evaluate saved weights instead of training")
    ap.add_argument("--fine", type=int, default=160, help="also evaluate on the fine x fine/2 x fine/2 mesh (0: skip)")
    ap.add_argument("--smooth", default="0", help="comma-separated smoothing passes to evaluate")
    ap.add_argument("--time-kernels", action="store_true",
                    help="time the network alone (forward and training step on random data, both convolution "
                         "kernel families) and exit")
    ap.add_argument("--steps", type=int, default=10, help="--time-kernels: timed repetitions")
    a = ap.parse_args(argv)
    torch.cuda.set_device(0)
    if a.time_kernels:
        return time_kernels(a.batch, a.steps)
    if a.load:
        net = UNet.load(a.load, a.batch)
    else:
        print(f"generating {a.designs} designs x 3 unit-load solves on 64x32x32")
        designs, X, Y, info = generate_training_set(a.designs)
        print(f"  {info}")
        net = UNet(NET_NODES, a.batch)
        net.set_params(init_params(net.num_params, 1))
        hist = train(net, X, Y, a.epochs, a.batch, a.lr)
        net.save(a.out, losses=np.asarray(hist), designs=a.designs, epochs=a.epochs)
        del X, Y
    rng = np.random.default_rng(0x5EED0006)
    test = [design_density(64, rng.uniform(0.2, 0.6), rng) for _ in range(a.test_designs)]
    trs = [v / np.linalg.norm(v) for v in rng.standard_normal((a.test_designs, 3))]
    fine = [design_density(a.fine, rng.uniform(0.2, 0.6), rng) for _ in range(2)] if a.fine else []
    ftr = [v / np.linalg.norm(v) for v in rng.standard_normal((2, 3))]
    for passes in (int(v) for v in a.smooth.split(",")):
        for method in ("plain", "two-level"):
            rows = evaluate(net, 64, test, trs, method, passes)
            print(f"64x32x32 {method} smooth={passes}: iterations "
                  f"{np.mean([r['iterations'] for r in rows]):.1f} -> {np.mean([r['iterations_learned'] for r in rows]):.1f} "
                  f"(guess), {np.mean([r['iterations_deflated'] for r in rows]):.1f} (deflation); "
                  f"ms {np.mean([r['ms'] for r in rows]):.2f} -> {np.mean([r['ms_learned'] for r in rows]):.2f}, "
                  f"{np.mean([r['ms_deflated'] for r in rows]):.2f}; "
                  f"energy captured {np.mean([r['energy_captured'] for r in rows]):.4f}; initial residual ratio "
                  f"{np.mean([r['initial_residual_ratio'] for r in rows]):.3f}", flush=True)
        if a.fine:
            f = a.fine
            for method in ("plain", "two-level"):
                rows = evaluate(net, f, fine, ftr, method, passes)
                print(f"{f}x{f // 2}x{f // 2} {method} smooth={passes}: " + "; ".join(
                    f"it {r['iterations']} -> {r['iterations_learned']} (guess), {r['iterations_deflated']} (deflation), "
                    f"ms {r['ms']:.1f} -> {r['ms_learned']:.1f}, {r['ms_deflated']:.1f}, "
                    f"energy {r['energy_captured']:.4f}, ratio {r['initial_residual_ratio']:.3f}" for r in rows),
                    flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
