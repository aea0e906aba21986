"""Benchmark: solve+adjoint throughput of SIMP linear-tet elastostatics on B200.

One step = one optimisation unit of the reference's Elliptic::Problem: assemble K(z) and
eliminate the clamped dofs, solve K u = F to the FP64 tolerance, compliance value and dC/dz
(self-adjoint).  Workload (default): 160 x 80 x 80 hexes x 6 tets on [0,2]x[0,1]x[0,1]
(6,144,000 tets, 3,168,963 dofs), clamped at x = 0, traction (0,-1,0) on x = 2, E = 1,
nu = 0.3, SIMP p = 3, rho_min = 1e-9, nodal densities i.i.d. U[0.01, 1] (SplitMix64 seed
0x5EED0002).  Synthetic data; every input and the 1.12 GB block matrix exceed the 126 MB L2.

Methods (--method):
  two-level-fp16  (default) FP64 flexible CG; preconditioner = FP32 Chebyshev-Jacobi smoothing
             on an FP16 copy of the Jacobi-scaled matrix D^-1/2 A D^-1/2 + Galerkin coarse
             correction on a 16x8x8 box grid (A-DEF2 two-level form).
  two-level  the same with an FP32 copy of the unscaled matrix.
  plain      the reference's algorithm: FP64 Jacobi-PCG on the assembled block matrix.
Both stop on the same FP64 residual test (1e-10); the line also carries the plain method's
throughput measured in the same run, and the accuracy of the timed solution against the
CPU oracle's own FP64 solve.

    python bench.py [--gpus N --steps K --warmup W] [--method plain] [--impl reference]
    python bench.py --profile-unit --cells 120,60,60 [--method two-level] [--repeat 1] [--coarse 16,8,8]

--profile-unit runs untimed solve+adjoint units of the same cantilever on other meshes (the
command the profiles' ncu captures run) and prints each unit's solver statistics.

Prints one JSON line (rank 0).  Multi-GPU runs are independent replicas (weak scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "solve+adjoint/s at 3.2M DoF, 1e-8 rel err: learned-MP PCG vs plain FP64 PCG"
UNIT = "solve+adjoint/s"
SIZES = {"large": (160, 80, 80), "medium": (80, 40, 40), "small": (20, 10, 10)}
# coarse box grid of the two-level method: coarse cells of 10^3 hexes (16x8x8 on 160x80x80,
# 4131 coarse dofs), see workloads.coarse_grid
SEED_LARGE = 0x5EED0002  # nodal densities of the workload (SplitMix64 stream)
# DRAM bytes per algorithmic byte of each roofline kernel: ncu's dram__bytes_read.sum +
# dram__bytes_write.sum per launch on the 120x60x60 cantilever (450,241 nodes, 2,592,000 cells,
# 6,606,721 blocks; inputs above L2) divided by that launch's algorithmic bytes.  Every stream
# of these kernels grows with the mesh, so the bench line's traffic is this ratio times the
# algorithmic bytes of its own launch.  Ratios near 1: no re-reads; the dC/dz pair reads the
# cell values and the node -> cell incidence a second time (nodal sums after the cell pass).
TRAFFIC_RATIO = {
    "sweep": (150.34 + 3.67) / 166.35,  # k_sell16s_st<0> (16-bit columns)
    "fp64_spmv": 533.8 / 525.52,    # k_fcg_sell_apply
    "assembly": 595.5 / 559.79,     # k_assemble_rows<SELL>
    "residual": 79.58 / 77.49,      # k_internal_force
    "energy": 67.58 / 66.69,        # k_energy_sum
    "dcdz": 135.35 / 70.29,         # k_cell_quantity<2> + k_node_sum
    "criterion": 135.34 / 70.29,    # k_energy_and_cell_grad + k_node_sum
}
TRAFFIC_NOTE = "ncu DRAM bytes per launch on the 120x60x60 cantilever, scaled by the algorithmic bytes"


METHOD_TEXT = {
    "two-level": ("FP64 flexible CG; preconditioner: FP32 Chebyshev-Jacobi (10 steps on [lmax/200, lmax]) on an FP32 SELL copy + "
                  "FP64 Galerkin coarse correction on a 16x8x8 trilinear box grid"),
    "two-level-fp16": ("FP64 flexible CG; preconditioner: FP32 Chebyshev-Jacobi (14 steps on [lmax/300, lmax]) on an FP16 copy of the "
                       "Jacobi-scaled matrix D^-1/2 A D^-1/2 + FP64 Galerkin coarse correction on a 16x8x8 trilinear "
                       "box grid"),
    "plain": "plain FP64 Jacobi-PCG on the assembled 3x3 block matrix (the reference's algorithm)",
    "chebyshev": "FP64 flexible CG; preconditioner: FP32 Chebyshev-Jacobi (8 steps) on an FP32 SELL copy",
    "bf16": "FP64 flexible CG; preconditioner: Chebyshev-Jacobi (16 steps) on a BF16-stored SELL copy",
    "matrix-free": "FP64 flexible CG on the matrix-free operator; FP32 matrix-free Chebyshev-Jacobi (16 steps)",
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--method", default="two-level-fp16", choices=list(METHOD_TEXT))
    ap.add_argument("--size", default="large", choices=list(SIZES))
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-unit", action="store_true",
                    help="run --repeat untimed solve+adjoint units on the --cells mesh (for profilers)")
    ap.add_argument("--cells", default="80,40,40", help="--profile-unit: hexes along x,y,z (6 tets each)")
    ap.add_argument("--repeat", type=int, default=1, help="--profile-unit: units to run")
    ap.add_argument("--coarse", default=None, help="--profile-unit: coarse box cells x,y,z")
    ap.add_argument("--api-kernels", action="store_true",
                    help="--profile-unit: each unit also evaluates R(u, z) and the block-CRS K(z) of the API")
    ap.add_argument("--workload", default="cantilever", choices=["cantilever", "batch", "helmholtz", "mixed"],
                    help="batch: 64 independent GRF cantilevers n x n/2 x n/2, n in {16,24,32,48,64}, one batched "
                         "solve; helmholtz: the density filter's solution and chain rule on the --size mesh; "
                         "mixed: the error report of every reduced-precision variant on the 20x10x10 mesh")
    return ap.parse_args()


def solver_options(method: str, tol: float, size: str = "large"):
    from platoanalyze_b200.workloads import coarse_grid, method_options

    return method_options(method, tol, coarse_grid(*SIZES[size]))


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d["hbm_gbs"], "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.out = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self):
        if not self.out:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------------------------
# CPU side: the oracle (FP64 restatement of the reference path, plain Jacobi-PCG), built with
# numpy and the oracle library alone (oracle/workload.py) so the reference arm never loads the
# product's CUDA library.

def _oracle_modules():
    sys.path.insert(0, str(ROOT / "oracle"))
    import workload as ow
    from oracle import Oracle
    return ow, Oracle


def oracle_step(orc, z, tol):
    """One full solve+adjoint unit of the reference path on the host: assemble K(z), the
    load, Dirichlet elimination, Jacobi-PCG to tol, compliance, self-adjoint dC/dz."""
    n = 3 * orc.N
    t0 = time.perf_counter()
    K = orc.vf_gradient_u(np.zeros(n), z)
    rhs = -orc.vf_value(np.zeros(n), z)
    orc.apply_constraints(K, rhs, 1.0)
    t1 = time.perf_counter()
    u, st = orc.pcg(K, rhs, tol=tol, max_it=10_000_000)
    t2 = time.perf_counter()
    f = orc.sf_value(u, z)
    g = orc.criterion_gradient(z, u, self_adjoint=True)
    t3 = time.perf_counter()
    return {"K": K, "rhs": rhs, "u": u, "dcdz": g, "compliance": f, "iterations": st["iterations"],
            "relative_residual": st["relative_residual"], "converged": st["converged"], "seconds": t3 - t0,
            "t_assembly": t1 - t0, "t_pcg": t2 - t1, "t_criterion": t3 - t2}


def oracle_reference(size, z, tol):
    """The oracle's full solve+adjoint of the problem on all host threads, timed (the CPU
    baseline), then (untimed) the accuracy reference: that solution refined with a long double
    iterate to a long double relative residual <= 1e-13, its compliance and dC/dz."""
    ow, Oracle = _oracle_modules()
    orc = ow.cantilever_oracle(*size)
    orc.graph()  # pattern build is one-off setup (not part of a step)
    r = oracle_step(orc, z, tol)
    K, rhs = r.pop("K"), r.pop("rhs")
    t0 = time.perf_counter()
    uld, st = orc.refine(K, rhs, r["u"], tol=1e-13, inner_tol=1e-4)
    ustar = uld.astype(np.float64)
    r["refine"] = {"seconds": time.perf_counter() - t0, "inner_iterations": st["iterations"],
                   "relative_residual": st["relative_residual"], "converged": st["converged"]}
    r["u_star"], r["u_star_ld"] = ustar, uld
    r["dcdz_star"] = orc.criterion_gradient(z, ustar, self_adjoint=True)
    r["compliance_star"] = orc.sf_value(ustar, z)
    r["cores"] = Oracle.num_threads()
    return r


def workload_config(args, size, num_cells, num_nodes, method):
    nx, ny, nz = size
    return {"workload": f"SIMP cantilever {nx}x{ny}x{nz} hexes x 6 tets on [0,2]x[0,1]x[0,1]",
            "tets": int(num_cells), "dofs": int(3 * num_nodes),
            "density": "nodal i.i.d. U[0.01,1], SplitMix64 seed 0x5EED0002", "method": METHOD_TEXT[method],
            "tolerance": args.tol, "adjoint": "self-adjoint (lambda = -u)",
            "l2": "inputs larger than L2 (block matrix 1.12 GB, vectors 25 MB each)",
            "parallelism": f"replicas x{args.gpus}"}


REFERENCE_BUDGET_S = 150.0  # timed full solves of the reference arm stop once the next would pass this


def run_reference(args):
    """--impl reference: the reference path's algorithm (the oracle port: FP64 assembly, plain
    Jacobi-PCG to the same tolerance, compliance, self-adjoint dC/dz) on all host threads.
    Every timed step is one complete solve+adjoint of the full workload -- nothing is
    extrapolated.  A step takes tens of seconds, so the arm times as many of the requested
    steps as fit in REFERENCE_BUDGET_S (at least one) and reports that count; its warm-up is
    the pattern build and one assembly (page placement), not whole solves.  A 1-thread pass
    over the phases (assembly, PCG iterations, criteria) is reported beside it."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    ow, Oracle = _oracle_modules()
    size = SIZES[args.size]
    orc = ow.cantilever_oracle(*size)
    z = ow.splitmix_uniform(orc.N, SEED_LARGE)
    orc.graph()
    orc.vf_gradient_u(np.zeros(3 * orc.N), z)  # warm-up: first touch of the matrix pages
    steps, t_total = [], 0.0
    while len(steps) < args.steps:
        r = oracle_step(orc, z, args.tol)
        for k in ("K", "rhs", "u", "dcdz"):
            r.pop(k)
        steps.append(r)
        t_total += r["seconds"]
        if t_total + r["seconds"] > REFERENCE_BUDGET_S:
            break
    v = len(steps) / t_total
    # 1-thread phase sample (not a throughput: a full 1-thread solve would take many minutes)
    threads = Oracle.num_threads()
    Oracle.set_num_threads(1)
    n = 3 * orc.N
    t0 = time.perf_counter()
    K = orc.vf_gradient_u(np.zeros(n), z)
    rhs = -orc.vf_value(np.zeros(n), z)
    orc.apply_constraints(K, rhs, 1.0)
    t1 = time.perf_counter()
    u, st = orc.pcg(K, rhs, tol=1e-300, max_it=10)
    t2 = time.perf_counter()
    orc.sf_value(u, z)
    orc.criterion_gradient(z, u, self_adjoint=True)
    t3 = time.perf_counter()
    Oracle.set_num_threads(threads)
    one_thread = {"assembly_constraints_s": t1 - t0, "pcg_ms_per_iteration": (t2 - t1) * 1e3 / max(1, st["iterations"]),
                  "compliance_dcdz_s": t3 - t2, "iterations_sampled": st["iterations"]}
    last = steps[-1]
    sample = (f"{len(steps)} full oracle solve+adjoint unit(s) of the workload on {threads} host threads "
              f"(assembly+constraints {last['t_assembly']:.2f}s, {last['iterations']} PCG iterations {last['t_pcg']:.2f}s, "
              f"compliance+dC/dz {last['t_criterion']:.2f}s in the last), no extrapolation")
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": len(steps),
            "steps_requested": args.steps, "warmup": args.warmup,
            "warmup_done": "pattern build + one assembly (page placement); each step is a complete solve",
            "ms_per_step": 1e3 * t_total / len(steps), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": workload_config(args, size, orc.C, orc.N, "plain") | {
                "pcg_iterations": [r["iterations"] for r in steps],
                "relative_residual": [r["relative_residual"] for r in steps],
                "converged": [r["converged"] for r in steps]},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
                             "one_thread_phases": one_thread},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------------------------

BATCH_METRIC = "batched solve+adjoint throughput: 64 independent GRF cantilevers, FP64-checked tol 1e-8"


def run_batch(args):
    """64 independent cantilevers as one batch handle; a step = batched solution to 1e-8,
    per-member compliance and dC/dz.  The same members are also solved one handle at a time."""
    import torch

    from platoanalyze_b200.problem import EllipticProblem
    from platoanalyze_b200.workloads import batch_workload, method_options

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    opts = method_options("chebyshev", 1e-8)
    specs, zs, ns = batch_workload(64, solver=opts)
    # a stream of its own, so the solver can capture its iteration chunks in CUDA graphs
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    bp = EllipticProblem.batch(specs, stream=stream)
    z = np.concatenate(zs)
    zd = bp.to_dev(z)
    tuning = bp.batch_autotune(zd)  # untimed: picks tile rows and persistent CTAs per SM

    def step():
        u, st = bp.solution(zd)
        f = bp.batch_criterion_values(zd, u)
        g, _ = bp.criterion_gradient(zd, u)
        return u, f, g, st

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    bp.reset_instrumentation()
    with ClockSampler(0) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            u, f, g, st = step()
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    per = bp.batch_last_stats()
    inst = bp.instrumentation()
    # e2e: host densities in, host displacements / gradients / compliances out
    z_pin = torch.from_numpy(z).pin_memory()
    u_pin = torch.empty(bp.num_dofs, dtype=torch.float64).pin_memory()
    g_pin = torch.empty(bp.num_nodes, dtype=torch.float64).pin_memory()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        zd.copy_(z_pin, non_blocking=True)
        u, f, g, _ = step()
        u_pin.copy_(u, non_blocking=True)
        g_pin.copy_(g, non_blocking=True)
        torch.cuda.synchronize()
    ms_e2e = (time.perf_counter() - t0) * 1e3 / args.steps
    # the same members one handle at a time (same solver)
    singles = [EllipticProblem(sp) for sp in specs]
    zds = [p.to_dev(zz) for p, zz in zip(singles, zs)]
    for p, zzd in zip(singles, zds):
        uu, _ = p.solution(zzd)
    torch.cuda.synchronize()
    e0.record(stream)
    its = []
    for p, zzd in zip(singles, zds):
        uu, st1 = p.solution(zzd)
        p.criterion_value(zzd, uu)
        p.criterion_gradient(zzd, uu)
        its.append(st1["iterations"])
    e1.record(stream)
    torch.cuda.synchronize()
    ms_seq = e0.elapsed_time(e1)
    for p in singles:
        p.close()
    line = {"metric": BATCH_METRIC, "value": 64 / (ms / 1e3), "unit": "problems/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32", "data": "synthetic",
            "config": {"workload": "64 cantilevers n x n/2 x n/2 hexes x 6 tets, n ~ U{16,24,32,48,64} (seed 0x5EED0004); "
                                   "GRF density (corr. length 0.1, logistic, clip [0.01,1]); unit traction, random direction",
                       "sizes": ns, "dofs_total": int(bp.num_dofs), "method": METHOD_TEXT["chebyshev"] + ", batched "
                       "(persistent kernels per stage, iteration chunks replayed as CUDA graphs)",
                       "autotuned": tuning,
                       "member_iterations": [m["iterations"] for m in per],
                       "max_relative_residual": max(m["relative_residual"] for m in per),
                       "one_handle_at_a_time_ms": ms_seq, "one_handle_at_a_time_iterations": its,
                       "speedup_vs_one_at_a_time": ms_seq / ms},
            "e2e": {"value": 64 / (ms_e2e / 1e3), "unit": "problems/s", "h2d_bytes_per_step": 8 * int(bp.num_nodes),
                    "d2h_bytes_per_step": 8 * int(bp.num_dofs + bp.num_nodes) + 8 * 64},
            "gpu_launches": inst["launches"], "clocks": clk.summary()}
    print(json.dumps(line))
    bp.close()
    return 0

# ---------------------------------------------------------------------------------------------

FILTER_METRIC = "Helmholtz filter solution + chain rule per second, 1.06M nodes, tol 1e-12"
FILTER_LENGTH = 0.025  # two element edges of the 160x80x80 mesh


def run_helmholtz(args):
    """The Helmholtz density filter on the 160x80x80 mesh: a step = filtered = K^-1 M control
    (Problem::solution) and dF/dcontrol = M K^-1 dF/dfiltered (Problem::criterionGradient),
    both scalar Jacobi-PCG to 1e-12; the oracle solves the same two systems on the host."""
    import torch

    from platoanalyze_b200.mesh import box_mesh
    from platoanalyze_b200.problem import HelmholtzFilter
    from platoanalyze_b200.workloads import SEED_FILTER, splitmix_uniform

    local = int(os.environ.get("LOCAL_RANK", "0"))
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    torch.cuda.set_device(local)
    nx, ny, nz = SIZES[args.size]
    mesh = box_mesh(nx, ny, nz, 2.0, 1.0, 1.0)
    filt = HelmholtzFilter(mesh.coords, mesh.connectivity, FILTER_LENGTH, tolerance=1e-12)
    N = filt.num_nodes
    control = splitmix_uniform(N, SEED_FILTER)
    dfdf = np.cos(np.arange(N) * 0.37)
    cd, wd = filt.to_dev(control), filt.to_dev(dfdf)
    stream = torch.cuda.current_stream()

    def step():
        f, s1 = filt.solution(cd)
        g, s2 = filt.criterion_gradient(wd)
        return f, g, s1, s2

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    filt.reset_instrumentation()
    filt.set_timing(True)
    with ClockSampler(local) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            f, g, s1, s2 = step()
        e1.record(stream)
        torch.cuda.synchronize()
    filt.set_timing(False)
    ms = e0.elapsed_time(e1) / args.steps
    inst = filt.instrumentation()

    # e2e: control and dF/dfiltered from pinned host memory, filtered and dF/dcontrol back
    c_pin = torch.from_numpy(control).pin_memory()
    w_pin = torch.from_numpy(dfdf).pin_memory()
    f_pin = torch.empty(N, dtype=torch.float64).pin_memory()
    g_pin = torch.empty(N, dtype=torch.float64).pin_memory()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        cd.copy_(c_pin, non_blocking=True)
        wd.copy_(w_pin, non_blocking=True)
        ff, gg, _, _ = step()
        f_pin.copy_(ff, non_blocking=True)
        g_pin.copy_(gg, non_blocking=True)
        torch.cuda.synchronize()
    ms_e2e = (time.perf_counter() - t0) * 1e3 / args.steps

    # roofline of the scalar SELL SpMV (k_sell1_spmv, fused p.Ap): values (8 B) and column
    # index (4 B) per stored entry, slice metadata, x read once and y written once
    rm, cols = filt.pattern()
    nnz = int(cols.numel())
    peak, peak_kind = peaks()
    spmv_bytes = 12 * nnz + 12 * ((N + 31) // 32) + 16 * N
    spmv_ms = inst["op_ms_total"] / max(1, inst["op_timed"])
    roof = {"bound": "hbm", "kernel": "k_sell1_spmv (scalar FP64 SELL-32 SpMV + p.Ap)",
            "achieved": spmv_bytes / (spmv_ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
            "frac": spmv_bytes / (spmv_ms / 1e3) / 1e9 / peak, "peak_source": peak_kind, "traffic": None,
            "algorithmic_bytes": spmv_bytes, "avg_launch_ms": spmv_ms, "launches_timed": inst["op_timed"]}

    cpu, accuracy = None, None
    if not args.no_cpu_baseline:
        sys.path.insert(0, str(ROOT / "oracle"))
        from oracle import Oracle

        orc = Oracle(mesh.coords, mesh.connectivity)
        orc.graph()
        t0 = time.perf_counter()
        fo, so1 = orc.helmholtz_solution(FILTER_LENGTH, control, tol=1e-12)
        go, so2 = orc.helmholtz_criterion_gradient(FILTER_LENGTH, dfdf, tol=1e-12)
        sec = time.perf_counter() - t0
        fh, gh = f.cpu().numpy(), g.cpu().numpy()
        accuracy = {"filtered_rel_err": float(np.linalg.norm(fh - fo) / np.linalg.norm(fo)),
                    "dfdcontrol_rel_err": float(np.linalg.norm(gh - go) / np.linalg.norm(go)),
                    "vs": f"CPU FP64 oracle solves ({so1['iterations']}+{so2['iterations']} PCG iterations)"}
        cpu = {"value": 1.0 / sec, "unit": "filter+chain-rule/s", "cores": Oracle.num_threads(), "kind": "port",
               "sample": f"full oracle filter solve + chain rule on the same mesh: {sec:.2f}s"}

    line = {"metric": FILTER_METRIC, "value": 1e3 / ms, "unit": "filter+chain-rule/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"Helmholtz density filter, {nx}x{ny}x{nz} hexes x 6 tets on [0,2]x[0,1]x[0,1]",
                       "nodes": N, "stored_entries": nnz, "length_scale": FILTER_LENGTH,
                       "control": "nodal i.i.d. U[0.01,1], SplitMix64 seed 0x5EED0005",
                       "method": "scalar FP64 Jacobi-PCG on the assembled K (assembled once per handle)",
                       "tolerance": 1e-12, "pcg_iterations": [s1["iterations"], s2["iterations"]],
                       "l2": "vectors 8.5 MB, matrix 190 MB: the matrix exceeds L2, the vectors do not"},
            "accuracy": accuracy, "roofline": roof, "cpu_baseline": cpu,
            "e2e": {"value": 1e3 / ms_e2e, "unit": "filter+chain-rule/s", "h2d_bytes_per_step": 16 * N,
                    "d2h_bytes_per_step": 16 * N},
            "gpu_launches": inst["launches"], "clocks": clk.summary()}
    print(json.dumps(line))
    filt.close()
    return 0


def run_profile_unit(args):
    """Untimed solve+adjoint units (Problem::solution, compliance, self-adjoint dC/dz) of the
    cantilever on the --cells mesh with nodal densities U[0.01, 1] (seed 0x5EED0002), for
    profilers; prints the solver statistics and compliance of each unit."""
    import torch

    from platoanalyze_b200.problem import EllipticProblem
    from platoanalyze_b200.workloads import SEED_LARGE, cantilever, coarse_grid, method_options, splitmix_uniform

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    nx, ny, nz = (int(v) for v in args.cells.split(","))
    cg = tuple(int(v) for v in args.coarse.split(",")) if args.coarse else coarse_grid(nx, ny, nz)
    spec = cantilever(nx, ny, nz, method_options(args.method, args.tol, cg))
    z = splitmix_uniform(spec.coords.shape[0], SEED_LARGE)
    prob = EllipticProblem(spec)
    zd = prob.to_dev(z)
    for _ in range(args.repeat):
        u, st = prob.solution(zd)
        f = prob.criterion_value(zd, u)
        prob.criterion_gradient(zd, u)
        if args.api_kernels:  # VectorFunction::value and ::gradient_u, the fused criterion pass
            prob.vf_value(u, zd)
            prob.vf_gradient_u(u, zd)
            prob.criterion_value_and_gradient(zd, u)
        torch.cuda.synchronize()
        print({"cells": (nx, ny, nz), "method": args.method, "compliance": f} | st)
    prob.close()
    return 0


MIXED_METRIC = "mixed-precision variants, 20x10x10 seeded cantilever, FP64-checked tol 1e-8: max relative error in u vs the FP64 oracle"


def run_mixed(args):
    """The mixed-precision error report: every reduced-precision variant solves the 20x10x10
    cantilever with nodal densities U[0.01, 1] (seed 0x5EED0003) to the FP64-recomputed
    relative residual 1e-8 (FP64 residuals, dot products and step lengths; the reduced
    precision lives in the preconditioner's matrix, element kernels and sweep), and reports
    its error in u, compliance and dC/dz against the oracle solved to a long double relative
    residual <= 1e-13.  The plain FP64 method at the same tolerance is the first row."""
    import torch

    from platoanalyze_b200 import capi
    from platoanalyze_b200.problem import EllipticProblem, SolverOptions
    from platoanalyze_b200.workloads import cantilever, splitmix_uniform

    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    tol = 1e-8
    spec = cantilever(20, 10, 10)
    z = splitmix_uniform(spec.coords.shape[0], 0x5EED0003)
    ow, Oracle = _oracle_modules()
    orc = ow.cantilever_oracle(20, 10, 10)
    us, _, st_ref = orc.solution_refined(z, tol=1e-13)
    fs = orc.sf_value(us, z)
    gs = orc.criterion_gradient(z, us, self_adjoint=True)
    variants = {
        "fp64: plain Jacobi-PCG (reference algorithm)": SolverOptions(tolerance=tol, max_iterations=200000),
        "fp32: Chebyshev(8)-Jacobi on an FP32 SELL copy, FP32 accumulation": SolverOptions(
            tolerance=tol, max_iterations=200000, precision=capi.PRECISION_MIXED_FP32, chebyshev_degree=8),
        "bf16-stored: Chebyshev(8)-Jacobi on a BF16 SELL copy, FP32 accumulation": SolverOptions(
            tolerance=tol, max_iterations=200000, precision=capi.PRECISION_MIXED_BF16, chebyshev_degree=8),
        "fp16-scaled: Chebyshev(8) on FP16 D^-1/2 A D^-1/2, FP32 accumulation": SolverOptions(
            tolerance=tol, max_iterations=200000, precision=capi.PRECISION_MIXED_FP16, chebyshev_degree=8),
        "fp32 element kernels: matrix-free FP32 element-by-element Chebyshev(8), FP64 matrix-free outer": SolverOptions(
            tolerance=tol, max_iterations=200000, operator_kind=capi.OPERATOR_MATRIX_FREE,
            precision=capi.PRECISION_MIXED_FP32, chebyshev_degree=8),
        "fp32 element assembly: FP32 element kernels assemble the preconditioner's SELL matrix, "
        "Chebyshev(8), FP64 matrix-free outer": SolverOptions(
            tolerance=tol, max_iterations=200000, operator_kind=capi.OPERATOR_MATRIX_FREE,
            precision=capi.PRECISION_MIXED_FP32_ASSEMBLED, chebyshev_degree=8),
        "fp16-scaled two-level: Chebyshev(8) + Galerkin coarse space 10x5x5": SolverOptions(
            tolerance=tol, max_iterations=200000, precision=capi.PRECISION_MIXED_FP16, chebyshev_degree=8,
            coarse_cells=(10, 5, 5)),
    }
    prob = EllipticProblem(spec)
    zd = prob.to_dev(z)
    rows = []
    for name, opts in variants.items():
        prob.set_solver(opts)
        prob.solution(zd)  # warm-up
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        u, st = prob.solution(zd)
        f = prob.criterion_value(zd, u)
        g, _ = prob.criterion_gradient(zd, u)
        e1.record()
        torch.cuda.synchronize()
        uh, gh = u.cpu().numpy(), g.cpu().numpy()
        rows.append({"variant": name, "iterations": st["iterations"], "relative_residual": st["relative_residual"],
                     "fallback": st["fallback"], "ms_solve_adjoint": e0.elapsed_time(e1),
                     "e_u": float(np.linalg.norm(uh - us) / np.linalg.norm(us)),
                     "e_compliance": abs(f - fs) / abs(fs),
                     "e_dcdz": float(np.linalg.norm(gh - gs) / np.linalg.norm(gs))})
    prob.close()
    worst = max(r["e_u"] for r in rows)
    line = {"metric": MIXED_METRIC, "value": worst, "unit": "relative error", "n_gpus": 1, "steps": 1,
            "warmup": 1, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32+bf16+f16",
            "data": "synthetic",
            "config": {"workload": "SIMP cantilever 20x10x10 hexes x 6 tets, nodal densities U[0.01,1] seed 0x5EED0003",
                       "tolerance": tol, "oracle": f"FP64 Jacobi-PCG refined with a long double iterate to relres "
                                                   f"{st_ref['relative_residual']:.2e}",
                       "variants": rows}}
    print(json.dumps(line))
    return 0


def main():
    args = parse()
    if args.profile_unit:
        return run_profile_unit(args)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "helmholtz":
        return run_helmholtz(args)
    if args.workload == "mixed":
        return run_mixed(args)

    import torch
    import torch.distributed as dist

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    from platoanalyze_b200.problem import EllipticProblem
    from platoanalyze_b200.workloads import cantilever, splitmix_uniform

    spec = cantilever(*SIZES[args.size], solver_options(args.method, args.tol, args.size))
    z = splitmix_uniform(spec.coords.shape[0], SEED_LARGE)
    prob = EllipticProblem(spec)
    zd = prob.to_dev(z)
    stream = torch.cuda.current_stream()

    def step():  # Problem::solution, then ComputeCriterion (compliance and dC/dz together)
        u, st = prob.solution(zd)
        f, g, _ = prob.criterion_value_and_gradient(zd, u)
        return u, f, g, st

    def timed_steps(k):
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out, stats = None, []
        for _ in range(k):
            out = step()
            stats.append(out[3])
        e1.record(stream)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item()), out, stats

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    prob.reset_instrumentation()
    prob.set_timing(True)
    with ClockSampler(local) as clk:
        ms_max, (u, f, g, _), stats = timed_steps(args.steps)
    prob.set_timing(False)
    inst = prob.instrumentation()
    value = world * args.steps / (ms_max / 1e3)

    # end to end through the C ABI with host buffers (H2D z, D2H u and dC/dz, compliance)
    u_pin = torch.empty(prob.num_dofs, dtype=torch.float64).pin_memory().numpy()
    g_pin = torch.empty(prob.num_nodes, dtype=torch.float64).pin_memory().numpy()
    z_pin = torch.from_numpy(np.ascontiguousarray(z)).pin_memory().numpy()
    prob.solve_and_gradient_host(z_pin, u_out=u_pin, g_out=g_pin)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record(stream)
    for _ in range(args.steps):
        prob.solve_and_gradient_host(z_pin, u_out=u_pin, g_out=g_pin)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = max(e0.elapsed_time(e1), (time.perf_counter() - t0) * 1e3)
    t = torch.tensor([ms_e2e], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_value = world * args.steps / (float(t.item()) / 1e3)

    # roofline: the FP64 operator apply of the Krylov loop (SELL SpMV) and, for the two-level
    # method, the FP32 Chebyshev step that dominates its step.  Algorithmic bytes per launch:
    # the matrix once (entries + column index per block, row pointers) and each vector stream once.
    N, B = prob.num_nodes, prob.num_blocks
    peak, peak_kind = peaks()
    spmv_bytes = 9 * B * 8 + B * 4 + (N + 1) * 4 + 3 * N * 8 * 2
    spmv_ms = inst["op_ms_total"] / max(1, inst["op_timed"])
    rl_spmv = {"bound": "hbm", "kernel": "k_sell_spmv / k_fcg_sell_apply (FP64 SELL-32 SpMV + p.Ap)",
               "achieved": spmv_bytes / (spmv_ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
               "frac": spmv_bytes / (spmv_ms / 1e3) / 1e9 / peak, "peak_source": peak_kind,
               "traffic": TRAFFIC_RATIO["fp64_spmv"] * spmv_bytes, "traffic_source": TRAFFIC_NOTE,
               "algorithmic_bytes": spmv_bytes, "avg_launch_ms": spmv_ms, "launches_timed": inst["op_timed"]}
    roofline, roofline_other = rl_spmv, None
    if inst["inner_timed"]:
        if args.method == "two-level-fp16":  # FP16 entries, no Jacobi diagonal stream (unit diagonal)
            cb = prob.sell_info()["column_bytes"]  # 16-bit column offsets when the numbering allows
            cheb_bytes = 9 * B * 2 + B * cb + (N + 1) * 4 + 6 * 3 * N * 4
            cheb_name = ("k_sell16s_st<0> (FP16 Jacobi-scaled SELL SpMV fused with one Chebyshev step; entries and "
                         "16-bit column offsets staged through shared memory)" if cb == 2 else
                         "k_sell16s<0> (FP16 Jacobi-scaled SELL SpMV fused with one Chebyshev step, 32-bit column indices)")
        else:
            cheb_bytes = 9 * B * 4 + B * 4 + (N + 1) * 4 + 7 * 3 * N * 4
            cheb_name = "k_cheb_sell<FP32> (FP32 SELL SpMV fused with one Chebyshev step)"
        cheb_ms = inst["inner_ms_total"] / inst["inner_timed"]
        rl_cheb = {"bound": "hbm", "kernel": cheb_name,
                   "achieved": cheb_bytes / (cheb_ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                   "frac": cheb_bytes / (cheb_ms / 1e3) / 1e9 / peak, "peak_source": peak_kind,
                   "traffic": TRAFFIC_RATIO["sweep"] * cheb_bytes if args.method == "two-level-fp16" and cb == 2 else None,
                   "traffic_source": TRAFFIC_NOTE,
                   "algorithmic_bytes": cheb_bytes, "avg_launch_ms": cheb_ms, "launches_timed": inst["inner_timed"]}
        roofline, roofline_other = rl_cheb, rl_spmv

    rl_asm = None
    if inst["assembly_timed"]:
        # connectivity + coordinates + control in; block values + column indices + row map out
        asm_bytes = 16 * prob.num_cells + 24 * N + 8 * N + 72 * B + 4 * B + 4 * (N + 1)
        asm_ms = inst["assembly_ms_total"] / inst["assembly_timed"]
        rl_asm = {"bound": "hbm", "kernel": "k_assemble_rows<SELL> (K(z) straight into the constrained SELL copy: "
                                           "thread per block row, upper blocks and their transposes)",
                  "achieved": asm_bytes / (asm_ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                  "frac": asm_bytes / (asm_ms / 1e3) / 1e9 / peak, "peak_source": peak_kind,
                  "traffic": TRAFFIC_RATIO["assembly"] * asm_bytes, "traffic_source": TRAFFIC_NOTE,
                  "algorithmic_bytes": asm_bytes, "avg_launch_ms": asm_ms, "launches_timed": inst["assembly_timed"]}

    # element kernels: the energy sum and the fused self-adjoint dC/dz are inside every step; the
    # residual R(u, z) = K(z) u - F (not part of the step) is timed on the step's solution.
    # Algorithmic bytes: connectivity 16 C, coordinates 24 N, control 8 N, state 24 N, plus the
    # output (R 24 N; dC/dz 8 N; the energy is a scalar).
    prob.set_timing(True)
    for _ in range(5):
        prob.vf_value(u, zd)
        prob.criterion_value(zd, u)
        prob.criterion_gradient(zd, u)
    torch.cuda.synchronize()
    prob.set_timing(False)
    inst_e = prob.instrumentation()
    elem_in = 16 * prob.num_cells + 24 * N + 8 * N + 24 * N

    def roof_line(kernel, nbytes, ms_total, count, ratio):
        if not count:
            return None
        ms = ms_total / count
        return {"bound": "hbm", "kernel": kernel, "achieved": nbytes / (ms / 1e3) / 1e9, "peak": peak,
                "unit": "GB/s", "frac": nbytes / (ms / 1e3) / 1e9 / peak, "peak_source": peak_kind,
                "traffic": ratio * nbytes, "traffic_source": TRAFFIC_NOTE, "algorithmic_bytes": nbytes,
                "avg_launch_ms": ms, "launches_timed": count}

    rl_elements = {
        "residual": roof_line("k_internal_force (+ the load copy): R = K(z) u - F", elem_in + 24 * N,
                              inst_e["residual_ms_total"], inst_e["residual_timed"], TRAFFIC_RATIO["residual"]),
        "energy": roof_line("k_energy_sum: compliance 1/2 u^T K(z) u", elem_in,
                            inst_e["energy_ms_total"], inst_e["energy_timed"], TRAFFIC_RATIO["energy"]),
        "dcdz": roof_line("k_cell_quantity<2> + k_node_sum: self-adjoint dC/dz", elem_in + 8 * N,
                          inst_e["dcdz_ms_total"], inst_e["dcdz_timed"], TRAFFIC_RATIO["dcdz"]),
        "criterion_in_step": roof_line("k_energy_and_cell_grad + k_node_sum: compliance and dC/dz in one pass "
                                       "(the step's ComputeCriterion)", elem_in + 8 * N,
                                       inst["criterion_ms_total"], inst["criterion_timed"],
                                       TRAFFIC_RATIO["criterion"])}

    # two-level coarse operator, once per solve: the Galerkin product P^T A P, then the banded
    # FP64 Cholesky (the coarse operator couples only corners of a common coarse cell) and the
    # dense L^-1 (FP64 mma.sync tiles).  dense_equivalent_tflops divides the dense-algorithm
    # flops (n^3/3 each) by the time, for comparison with the dense factorization.
    coarse = None
    if inst["coarse_galerkin_timed"]:
        cc = spec.solver.coarse_cells
        nc = 3 * int(np.prod([c + 1 for c in cc]))
        band = 3 * ((cc[1] + 1) * (cc[2] + 1) + (cc[2] + 1) + 1) + 2
        inv_ms = inst["coarse_inverse_ms_total"] / inst["coarse_galerkin_timed"]
        flops = 2.0 * nc ** 3 / 3.0
        coarse = {"coarse_dofs": nc, "band": band,
                  "galerkin_ms": inst["coarse_galerkin_ms_total"] / inst["coarse_galerkin_timed"],
                  "inverse_ms": inv_ms, "dense_equivalent_flops": flops,
                  "dense_equivalent_tflops": flops / (inv_ms / 1e3) / 1e12,
                  "setups_timed": inst["coarse_galerkin_timed"]}

    # the plain FP64 GPU method on the same problem, same run (comparison only)
    plain = None
    if args.method != "plain":
        prob.set_solver(solver_options("plain", args.tol, args.size))
        step()
        ms_plain, _, pstats = timed_steps(2)
        plain = {"value": world * 2 / (ms_plain / 1e3), "ms_per_step": ms_plain / 2,
                 "pcg_iterations": [s["iterations"] for s in pstats]}
        prob.set_solver(solver_options(args.method, args.tol, args.size))

    # secondary figure: Self-Adjoint = false, the adjoint K^T lambda = -df/du solved explicitly
    # by the same method (Problem::criterionGradient, src/elliptic/Problem.hpp:428-448)
    explicit_adjoint = None
    o = solver_options(args.method, args.tol, args.size)
    o.self_adjoint = False
    prob.set_solver(o)
    step()
    ms_ea, (_, _, g_ea, _), _ = timed_steps(2)
    prob.set_solver(solver_options(args.method, args.tol, args.size))
    explicit_adjoint = {"value": world * 2 / (ms_ea / 1e3), "unit": UNIT, "ms_per_step": ms_ea / 2,
                        "dcdz_rel_diff_vs_self_adjoint": float((g_ea - g).norm() / g.norm())}

    # accuracy against the oracle: its full FP64 solve of the problem (timed: the CPU baseline on
    # all host threads), refined with a long double iterate to a relative residual <= 1e-13
    # (untimed; u* and dC/dz* of the error definitions)
    cpu, accuracy = None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ref = oracle_reference(SIZES[args.size], z, args.tol)
        uh, gh = u.cpu().numpy(), g.cpu().numpy()
        us, gs = ref["u_star"], ref["dcdz_star"]
        e_u = float(np.linalg.norm((uh.astype(np.longdouble) - ref["u_star_ld"])) / np.linalg.norm(ref["u_star_ld"]))
        accuracy = {"u_rel_err": e_u,
                    "dcdz_rel_err": float(np.linalg.norm(gh - gs) / np.linalg.norm(gs)),
                    "compliance": f, "compliance_rel_err": abs(f - ref["compliance_star"]) / abs(ref["compliance_star"]),
                    "oracle_fp64_solve_u_rel_err": float(np.linalg.norm(ref["u"] - us) / np.linalg.norm(us)),
                    "vs": (f"CPU oracle: FP64 Jacobi-PCG ({ref['iterations']} iterations, relres "
                           f"{ref['relative_residual']:.2e}) refined with a long double iterate to relres "
                           f"{ref['refine']['relative_residual']:.2e} ({ref['refine']['inner_iterations']} inner "
                           f"iterations, {ref['refine']['seconds']:.1f}s, untimed)")}
        cpu = {"value": 1.0 / ref["seconds"], "unit": UNIT, "cores": ref["cores"], "kind": "port",
               "sample": (f"full oracle solve+adjoint of the same workload on the host (plain FP64 Jacobi-PCG): "
                          f"assembly+constraints {ref['t_assembly']:.2f}s, {ref['iterations']} PCG iterations "
                          f"{ref['t_pcg']:.2f}s, compliance+dC/dz {ref['t_criterion']:.2f}s")}

    cfg = workload_config(args, SIZES[args.size], prob.num_cells, prob.num_nodes, args.method) | {
        "krylov_iterations": [s["iterations"] for s in stats],
        "preconditioner_operator_applies": [s["refinements"] for s in stats],
        "relative_residual": [s["relative_residual"] for s in stats]}
    if plain:
        cfg["plain_fp64_gpu"] = plain
        cfg["speedup_vs_plain_fp64_gpu"] = value / plain["value"]
    cfg["explicit_adjoint"] = explicit_adjoint
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": {"plain": "f64", "bf16": "f64+bf16", "two-level-fp16": "f64+f32+f16"}.get(args.method, "f64+f32"),
            "data": "synthetic", "config": cfg, "accuracy": accuracy, "roofline": roofline,
            "roofline_fp64_spmv": roofline_other, "roofline_assembly": rl_asm, "roofline_elements": rl_elements,
            "coarse_setup": coarse,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 8 * N,
                    "d2h_bytes_per_step": 8 * (3 * N + N) + 8},
            "gpu_launches": inst["launches"], "clocks": clk.summary()}
    if rank == 0:
        print(json.dumps(line))
    prob.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
