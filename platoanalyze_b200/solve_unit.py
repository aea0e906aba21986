"""Run solve+adjoint units of the SIMP cantilever on cuda:0 (for profilers and quick checks).

    python -m platoanalyze_b200.solve_unit --cells 120,60,60 --method two-level [--repeat 1] [--coarse 16,8,8]

One unit = Problem::solution (assembly, constraints, solve), compliance and dC/dz
(self-adjoint), the bench's step.  Densities are nodal i.i.d. U[0.01, 1] from SplitMix64
seed 0x5EED0002.  Prints the solver statistics and the compliance of each unit.
"""
from __future__ import annotations

import argparse


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--cells", default="80,40,40", help="hexes along x,y,z (each cut into 6 tets)")
    ap.add_argument("--method", default="two-level")
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--coarse", default=None, help="coarse box cells x,y,z (default: chosen from --cells)")
    a = ap.parse_args(argv)

    import torch

    from .problem import EllipticProblem
    from .workloads import SEED_LARGE, cantilever, coarse_grid, method_options, splitmix_uniform

    nx, ny, nz = (int(v) for v in a.cells.split(","))
    cg = tuple(int(v) for v in a.coarse.split(",")) if a.coarse else coarse_grid(nx, ny, nz)
    spec = cantilever(nx, ny, nz, method_options(a.method, a.tol, cg))
    z = splitmix_uniform(spec.coords.shape[0], SEED_LARGE)
    prob = EllipticProblem(spec)
    zd = prob.to_dev(z)
    for _ in range(a.repeat):
        u, st = prob.solution(zd)
        f = prob.criterion_value(zd, u)
        prob.criterion_gradient(zd, u)
        torch.cuda.synchronize()
        print({"cells": (nx, ny, nz), "method": a.method, "compliance": f} | st)
    prob.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
