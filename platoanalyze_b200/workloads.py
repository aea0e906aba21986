"""Synthetic workloads of the elliptic SIMP benchmark (box cantilevers, seeded densities).

Box [0,2]x[0,1]x[0,1] cut into nx x ny x nz hexes x 6 tets, clamped on x = 0, uniform
traction (0,-1,0) on x = 2, E = 1, nu = 0.3, SIMP p = 3, rho_min = 1e-9.
  * small:  20 x 10 x 10 hexes (12,000 tets,    7,623 dofs), uniform z = 0.5
  * large: 160 x 80 x 80 hexes (6,144,000 tets, 3,168,963 dofs), nodal z ~ U[0.01, 1]
           from SplitMix64 seed 0x5EED0002
"""
from __future__ import annotations

import numpy as np

from .mesh import box_mesh
from .problem import ProblemSpec, SolverOptions, cantilever_spec

SEED_LARGE = 0x5EED0002
SEED_MIXED = 0x5EED0003


def splitmix_uniform(n: int, seed: int, lo: float = 0.01, hi: float = 1.0) -> np.ndarray:
    """n i.i.d. U[lo, hi) doubles from a SplitMix64 stream (the k-th value uses state seed + k*golden)."""
    idx = np.arange(1, n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = np.uint64(seed) + idx * np.uint64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        x = x ^ (x >> np.uint64(31))
    u = (x >> np.uint64(11)).astype(np.float64) * (1.0 / float(1 << 53))
    return lo + (hi - lo) * u


def cantilever(nx: int, ny: int, nz: int, solver: SolverOptions | None = None) -> ProblemSpec:
    return cantilever_spec(box_mesh(nx, ny, nz, 2.0, 1.0, 1.0), traction=(0.0, -1.0, 0.0), E=1.0, nu=0.3,
                           p=3.0, rho_min=1e-9, solver=solver)


def small_problem(solver: SolverOptions | None = None):
    spec = cantilever(20, 10, 10, solver)
    z = np.full(spec.coords.shape[0], 0.5)
    return spec, z


def large_problem(solver: SolverOptions | None = None, n: tuple[int, int, int] = (160, 80, 80)):
    spec = cantilever(*n, solver)
    z = splitmix_uniform(spec.coords.shape[0], SEED_LARGE)
    return spec, z
