"""Benchmark: solve+adjoint throughput of SIMP linear-tet elastostatics on B200.

One step = one optimisation unit of the reference's Elliptic::Problem: assemble K(z),
apply the Dirichlet elimination, Jacobi-PCG to the FP64 tolerance, compliance value and
dC/dz (self-adjoint).  Workload (default): 160 x 80 x 80 hexes x 6 tets on [0,2]x[0,1]x[0,1]
(6,144,000 tets, 3,168,963 dofs), clamped at x = 0, traction (0,-1,0) on x = 2, E = 1,
nu = 0.3, SIMP p = 3, rho_min = 1e-9, nodal densities i.i.d. U[0.01, 1] (SplitMix64 seed
0x5EED0002).  Synthetic data; every input and the 1.12 GB block matrix exceed the 126 MB L2.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

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
# Jacobi-PCG iterations of the plain FP64 method on the large workload at tol 1e-10 (from the
# B200 run of this bench; the GPU arm re-measures and reports its own count).
FP64_ITERATIONS = {"large": 3634, "medium": 1834, "small": None}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", default="large", choices=list(SIZES))
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--cpu-iters", type=int, default=20, help="PCG iterations in the CPU sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


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
# CPU arm: the oracle (FP64 restatement of the reference path) on a bounded sample

def cpu_sample(spec, z, n_iters_full, cpu_iters):
    """Times assembly + constraints + `cpu_iters` PCG iterations + compliance + dC/dz on the
    full mesh with the oracle, and extrapolates the PCG part to `n_iters_full` iterations."""
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle import Oracle

    orc = Oracle.from_spec(spec)
    orc.graph()  # pattern build is one-off setup (not part of a step)
    t0 = time.perf_counter()
    K = orc.vf_gradient_u(np.zeros(3 * orc.N), z)
    rhs = np.zeros(3 * orc.N)
    R = orc.vf_value(np.zeros(3 * orc.N), z)
    rhs[:] = -R
    orc.apply_constraints(K, rhs, 1.0)
    t1 = time.perf_counter()
    x, st = orc.pcg(K, rhs, tol=1e-300, max_it=cpu_iters)
    t2 = time.perf_counter()
    orc.sf_value(x, z)
    orc.criterion_gradient(z, x, self_adjoint=True)
    t3 = time.perf_counter()
    per_iter = (t2 - t1) / max(1, st["iterations"])
    unit_s = (t1 - t0) + per_iter * n_iters_full + (t3 - t2)
    return {"value": 1.0 / unit_s, "unit": UNIT, "cores": Oracle.num_threads(), "kind": "port",
            "sample": (f"oracle on the full mesh: assembly+constraints {t1 - t0:.2f}s, {st['iterations']} PCG "
                       f"iterations at {per_iter * 1e3:.1f} ms each extrapolated to {n_iters_full}, "
                       f"compliance+dC/dz {t3 - t2:.2f}s"),
            "seconds_per_unit": unit_s}


def oracle_reference(spec, z, tol):
    """Full FP64 solve + compliance + dC/dz of the problem with the CPU oracle, timed."""
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle import Oracle

    orc = Oracle.from_spec(spec)
    orc.graph()  # pattern build is one-off setup (not part of a step)
    n = 3 * orc.N
    t0 = time.perf_counter()
    K = orc.vf_gradient_u(np.zeros(n), z)
    rhs = -orc.vf_value(np.zeros(n), z)
    orc.apply_constraints(K, rhs, 1.0)
    t1 = time.perf_counter()
    u, st = orc.pcg(K, rhs, tol=tol, max_it=1000000)
    t2 = time.perf_counter()
    f = orc.sf_value(u, z)
    g = orc.criterion_gradient(z, u, self_adjoint=True)
    t3 = time.perf_counter()
    return {"u": u, "dcdz": g, "compliance": f, "iterations": st["iterations"],
            "relative_residual": st["relative_residual"], "seconds": t3 - t0, "t_assembly": t1 - t0,
            "t_pcg": t2 - t1, "t_criterion": t3 - t2, "cores": Oracle.num_threads()}


def run_reference(args):
    """--impl reference: the oracle port of the reference path on the host cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from platoanalyze_b200.workloads import SEED_LARGE, cantilever, splitmix_uniform

    spec = cantilever(*SIZES[args.size])
    z = splitmix_uniform(spec.coords.shape[0], SEED_LARGE)
    n_it = FP64_ITERATIONS.get(args.size)
    if n_it is None:
        print(json.dumps({"impl": "reference", "unavailable": "plain FP64 iteration count for this size not recorded"}))
        return 0
    vals = []
    for s in range(args.warmup + args.steps):
        r = cpu_sample(spec, z, n_it, args.cpu_iters)
        if s >= args.warmup:
            vals.append(r)
    v = statistics.median([r["value"] for r in vals])
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": workload_config(args, spec),
            "cpu_baseline": {k: vals[-1][k] for k in ("cores", "kind", "sample")} | {"value": v, "unit": UNIT},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def workload_config(args, spec, method="plain FP64 Jacobi-PCG, assembled 3x3 block CRS"):
    nx, ny, nz = SIZES[args.size]
    return {"workload": f"SIMP cantilever {nx}x{ny}x{nz} hexes x 6 tets on [0,2]x[0,1]x[0,1]",
            "tets": int(spec.connectivity.shape[0]), "dofs": int(3 * spec.coords.shape[0]),
            "density": "nodal i.i.d. U[0.01,1], SplitMix64 seed 0x5EED0002", "method": method,
            "tolerance": args.tol, "adjoint": "self-adjoint (lambda = -u)",
            "l2": "inputs larger than L2 (block matrix 1.12 GB, vectors 25 MB x 7)",
            "parallelism": f"replicas x{args.gpus}"}


# ---------------------------------------------------------------------------------------------

def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)

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

    from platoanalyze_b200.problem import EllipticProblem, SolverOptions
    from platoanalyze_b200.workloads import SEED_LARGE, cantilever, splitmix_uniform

    spec = cantilever(*SIZES[args.size], SolverOptions(tolerance=args.tol, max_iterations=200000))
    z = splitmix_uniform(spec.coords.shape[0], SEED_LARGE)
    prob = EllipticProblem(spec)
    zd = prob.to_dev(z)
    stream = torch.cuda.current_stream()

    def step():
        u, st = prob.solution(zd)
        f = prob.criterion_value(zd, u)
        g, _ = prob.criterion_gradient(zd, u)
        return u, f, g, st

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    prob.reset_instrumentation()
    prob.set_timing(True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        iters = []
        for _ in range(args.steps):
            u, f, g, st = step()
            iters.append(st["iterations"])
        e1.record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    prob.set_timing(False)
    ms = e0.elapsed_time(e1)
    inst = prob.instrumentation()
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * args.steps / (ms_max / 1e3)

    # end to end through the C ABI with host buffers (H2D z, D2H u, compliance, dC/dz)
    z_host = np.ascontiguousarray(z)
    u_host = np.empty(prob.num_dofs)
    g_host = np.empty(prob.num_nodes)
    u_pin = torch.empty(prob.num_dofs, dtype=torch.float64).pin_memory().numpy()
    g_pin = torch.empty(prob.num_nodes, dtype=torch.float64).pin_memory().numpy()
    z_pin = torch.from_numpy(z_host).pin_memory().numpy()
    prob.solve_and_gradient_host(z_pin, u_out=u_pin, g_out=g_pin)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0.record(stream)
    for _ in range(args.steps):
        prob.solve_and_gradient_host(z_pin, u_out=u_pin, g_out=g_pin)
    e1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    ms_e2e = max(e0.elapsed_time(e1), wall * 1e3)
    t = torch.tensor([ms_e2e], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_value = world * args.steps / (float(t.item()) / 1e3)
    del u_host, g_host

    # roofline of the dominant kernel (FP64 SELL SpMV inside PCG).  Algorithmic bytes: the
    # constrained block matrix once (9 doubles + 1 column index per block, row pointers),
    # x gathered once and y written once.
    N, B = prob.num_nodes, prob.num_blocks
    spmv_bytes = 9 * B * 8 + B * 4 + (N + 1) * 4 + 3 * N * 8 * 2
    avg_ms = inst["op_ms_total"] / max(1, inst["op_timed"])
    peak, peak_kind = peaks()
    achieved = spmv_bytes / (avg_ms / 1e3) / 1e9
    roofline = {"bound": "hbm", "kernel": "k_sell_spmv (FP64 SELL-32 block SpMV + p.Ap)", "achieved": achieved,
                "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": None, "algorithmic_bytes": spmv_bytes, "avg_launch_ms": avg_ms,
                "launches_timed": inst["op_timed"]}

    # accuracy against the CPU oracle's own FP64 solve of the full problem (untimed), and the
    # CPU baseline from the same oracle run
    cpu, accuracy = None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ref = oracle_reference(spec, z, args.tol)
        uo, go = ref.pop("u"), ref.pop("dcdz")
        uh, gh = u.cpu().numpy(), g.cpu().numpy()
        accuracy = {"u_rel_err": float(np.linalg.norm(uh - uo) / np.linalg.norm(uo)),
                    "dcdz_rel_err": float(np.linalg.norm(gh - go) / np.linalg.norm(go)),
                    "compliance": f, "compliance_rel_err": abs(f - ref["compliance"]) / abs(ref["compliance"]),
                    "vs": f"CPU FP64 oracle solve of the same problem ({ref['iterations']} PCG iterations, "
                          f"relres {ref['relative_residual']:.2e})"}
        cpu = {"value": 1.0 / ref["seconds"], "unit": UNIT, "cores": ref["cores"], "kind": "port",
               "sample": (f"full oracle solve+adjoint of the same workload on the host: assembly+constraints "
                          f"{ref['t_assembly']:.2f}s, {ref['iterations']} PCG iterations {ref['t_pcg']:.2f}s, "
                          f"compliance+dC/dz {ref['t_criterion']:.2f}s")}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args, spec) | {"pcg_iterations": iters},
            "accuracy": accuracy,
            "roofline": roofline, "cpu_baseline": cpu,
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
