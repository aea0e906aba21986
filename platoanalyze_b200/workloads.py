"""Synthetic workloads of the elliptic SIMP benchmark (box cantilevers, seeded densities).

Box [0,2]x[0,1]x[0,1] cut into nx x ny x nz hexes x 6 tets, clamped on x = 0, uniform
traction (0,-1,0) on x = 2, E = 1, nu = 0.3, SIMP p = 3, rho_min = 1e-9.
  * small:  20 x 10 x 10 hexes (12,000 tets,    7,623 dofs), uniform z = 0.5
  * large: 160 x 80 x 80 hexes (6,144,000 tets, 3,168,963 dofs), nodal z ~ U[0.01, 1]
           from SplitMix64 seed 0x5EED0002
"""
from __future__ import annotations

import numpy as np

from . import capi
from .mesh import box_mesh
from .problem import ProblemSpec, SolverOptions, cantilever_spec

SEED_LARGE = 0x5EED0002
SEED_MIXED = 0x5EED0003
SEED_BATCH = 0x5EED0004
SEED_FILTER = 0x5EED0005
BATCH_SIZES = (16, 24, 32, 48, 64)


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


COARSE_BOX = (10, 5, 5)  # coarse box grid of the two-level method (aligns with 20k x 10k x 10k hex grids)


def coarse_grid(nx: int, ny: int, nz: int, span: int = 10, max_dofs: int = 6144) -> tuple:
    """Coarse box grid for an nx x ny x nz hex mesh: per axis the largest count that divides
    the hex count and gives coarse cells of at least `span` hexes (one cell when none does),
    halved while the dense coarse solve would exceed max_dofs."""
    def axis(n: int) -> int:
        for g in range(max(1, n // span), 0, -1):
            if n % g == 0:
                return g
        return 1

    g = [axis(nx), axis(ny), axis(nz)]
    while 3 * (g[0] + 1) * (g[1] + 1) * (g[2] + 1) > max_dofs and all(v % 2 == 0 for v in g):
        g = [v // 2 for v in g]
    return tuple(g)

METHODS = ("two-level", "two-level-fp16", "plain", "chebyshev", "bf16", "matrix-free")


def method_options(method: str, tol: float = 1e-10, coarse=COARSE_BOX) -> SolverOptions:
    """Solver options of the named method; every method stops on the same FP64 residual test.

    plain        FP64 Jacobi-PCG on the assembled block matrix (the reference's algorithm)
    two-level    FP64 flexible CG; FP32 Chebyshev(10)-Jacobi on [lmax/200, lmax] on an FP32 copy
                 of the matrix plus a Galerkin coarse correction on a trilinear box grid
    two-level-fp16  the same with the Chebyshev sweep on an FP16 copy of the Jacobi-scaled
                 matrix D^-1/2 A D^-1/2, Chebyshev(14) on [lmax/300, lmax]
    chebyshev    the same without the coarse correction
    bf16         BF16-stored matrix, Chebyshev(16)-Jacobi, no coarse correction
    matrix-free  FP32 element-by-element operator, Chebyshev(16)-Jacobi, no coarse correction
    """
    if method == "plain":
        return SolverOptions(tolerance=tol, max_iterations=200000)
    # with the coarse correction taking the low end of the spectrum, the smoother targets
    # [lmax/200, lmax]; degree 10 (measured on 160x80x80: 45 iterations, against 64 at degree
    # 8 on [lmax/30, lmax])
    if method == "two-level":
        return SolverOptions(tolerance=tol, max_iterations=200000, precision=capi.PRECISION_MIXED_FP32,
                             chebyshev_degree=10, chebyshev_ratio=200.0, coarse_cells=tuple(coarse))
    # the FP16 sweep step is cheap against an outer iteration (FP64 apply, coarse solve, vector
    # updates), so a longer polynomial pays: on 160x80x80 degree 14 on [lmax/300, lmax] takes 22
    # iterations, 51.5 ms per solve+adjoint, against 29 and 52.3 ms at degree 10 on [lmax/200, lmax]
    if method == "two-level-fp16":
        return SolverOptions(tolerance=tol, max_iterations=200000, precision=capi.PRECISION_MIXED_FP16,
                             chebyshev_degree=14, chebyshev_ratio=300.0, coarse_cells=tuple(coarse))
    if method == "chebyshev":
        return SolverOptions(tolerance=tol, max_iterations=200000, precision=capi.PRECISION_MIXED_FP32,
                             chebyshev_degree=8, chebyshev_ratio=30.0)
    if method == "bf16":
        return SolverOptions(tolerance=tol, max_iterations=200000, precision=capi.PRECISION_MIXED_BF16,
                             chebyshev_degree=16)
    if method == "matrix-free":
        return SolverOptions(tolerance=tol, max_iterations=200000, operator_kind=capi.OPERATOR_MATRIX_FREE,
                             precision=capi.PRECISION_MIXED_FP32, chebyshev_degree=16)
    raise ValueError(f"unknown method {method!r}; one of {METHODS}")


def grf_field(nx: int, ny: int, nz: int, lengths=(2.0, 1.0, 1.0), corr: float = 0.1,
              rng: np.random.Generator | None = None) -> np.ndarray:
    """A stationary Gaussian random field with covariance exp(-r^2 / (2 corr^2)) on the
    (nx+1)(ny+1)(nz+1) box-mesh nodes (z fastest), sampled by filtering white noise in Fourier
    space (spectral density exp(-|k|^2 corr^2 / 2)) and standardised to zero mean, unit variance."""
    rng = rng or np.random.default_rng(0)
    shape = (nx + 1, ny + 1, nz + 1)
    h = [lengths[0] / nx, lengths[1] / ny, lengths[2] / nz]
    noise = rng.standard_normal(shape)
    k = np.meshgrid(*[2 * np.pi * np.fft.fftfreq(m, d=hh) for m, hh in zip(shape, h)], indexing="ij")
    k2 = k[0] ** 2 + k[1] ** 2 + k[2] ** 2
    field = np.real(np.fft.ifftn(np.fft.fftn(noise) * np.exp(-0.25 * k2 * corr * corr)))
    return ((field - field.mean()) / max(field.std(), 1e-300)).reshape(-1)


def grf_density(nx: int, ny: int, nz: int, lengths=(2.0, 1.0, 1.0), corr: float = 0.1,
                rng: np.random.Generator | None = None) -> np.ndarray:
    """Nodal density: grf_field passed through the logistic function and clipped to [0.01, 1]."""
    g = grf_field(nx, ny, nz, lengths, corr, rng)
    return np.clip(1.0 / (1.0 + np.exp(-g)), 0.01, 1.0)


def batch_workload(count: int = 64, seed: int = SEED_BATCH, sizes=BATCH_SIZES,
                   solver: SolverOptions | None = None):
    """Independent cantilevers n x n/2 x n/2 hexes x 6 tets on [0,2]x[0,1]x[0,1], n drawn
    uniformly from `sizes`; density from grf_density; traction on the x = 2 face with a
    direction uniform on the unit sphere and magnitude 1.  Returns (specs, densities, ns)."""
    rng = np.random.default_rng(seed)
    specs, zs, ns = [], [], []
    for _ in range(count):
        n = int(rng.choice(np.asarray(sizes)))
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        mesh = box_mesh(n, n // 2, n // 2, 2.0, 1.0, 1.0)
        specs.append(cantilever_spec(mesh, traction=tuple(float(v) for v in d), E=1.0, nu=0.3, p=3.0,
                                     rho_min=1e-9, solver=solver))
        zs.append(grf_density(n, n // 2, n // 2, rng=rng))
        ns.append(n)
    return specs, zs, ns
