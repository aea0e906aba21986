"""Python mirror of the reference's elliptic interfaces over the C ABI.

`EllipticProblem` owns one plato_problem handle and exposes the reference's method names:
VectorFunction (`vf_value`, `vf_gradient_u`, `vf_gradient_u_T`, `vf_gradient_z`),
PhysicsScalarFunction "Internal Elastic Energy" (`sf_value`, `sf_gradient_u`,
`sf_gradient_z`) and Problem (`solution`, `criterion_value`, `criterion_gradient`).
Device buffers are torch CUDA tensors (torch is used for memory and streams only; all
arithmetic runs in the library's kernels).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import capi
from .capi import check, lib
from .mesh import BoxMesh


def _np_ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


@dataclass
class SolverOptions:
    tolerance: float = 1e-10
    max_iterations: int = 20000
    operator_kind: int = capi.OPERATOR_ASSEMBLED
    precision: int = capi.PRECISION_FP64
    self_adjoint: bool = True
    chebyshev_ratio: float = 30.0
    chebyshev_degree: int = 0
    coarse_cells: tuple = (0, 0, 0)
    fallback_max_iterations: int = 0  # plain FP64 Jacobi-PCG fallback cap (0: max_iterations, < 0: none)
    chebyshev_kind: int = 1  # 1: first kind on [lmax/ratio, lmax]; 4: fourth kind on (0, lmax]
    sweep_steps: int = 0  # FP16 sweep: Chebyshev steps per launch (0 or 1: one per launch)
    sweep_lag: int = 0  # multi-step sweep: extra tiles between consecutive steps (0: 600 / steps)

    def to_c(self) -> capi.SolverOpts:
        return capi.SolverOpts(self.tolerance, self.max_iterations, self.operator_kind, self.precision,
                               int(self.self_adjoint), self.chebyshev_ratio, self.chebyshev_degree,
                               (C.c_int32 * 3)(*self.coarse_cells), self.fallback_max_iterations,
                               self.chebyshev_kind, self.sweep_steps, self.sweep_lag)


@dataclass
class ProblemSpec:
    coords: np.ndarray
    connectivity: np.ndarray
    youngs_modulus: float = 1.0
    poissons_ratio: float = 0.3
    penalty_exponent: float = 3.0
    penalty_minimum: float = 1e-9
    tractions: list = field(default_factory=list)  # [(face_cells, face_local_nodes, (tx,ty,tz))]
    bc_dofs: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    bc_values: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float64))
    solver: SolverOptions = field(default_factory=SolverOptions)


def cantilever_spec(mesh: BoxMesh, traction=(0.0, -1.0, 0.0), E=1.0, nu=0.3, p=3.0, rho_min=1e-9,
                    solver: SolverOptions | None = None) -> ProblemSpec:
    """Box clamped on x = 0 (all three dofs), uniform traction on the x = Lx face."""
    from .mesh import X_MINUS, X_PLUS
    fixed = mesh.nodeset(X_MINUS)
    dofs = (3 * fixed[:, None] + np.arange(3)[None, :]).reshape(-1).astype(np.int32)
    cells, local = mesh.sideset(X_PLUS)
    return ProblemSpec(mesh.coords, mesh.connectivity, E, nu, p, rho_min,
                       [(cells, local, traction)], dofs, np.zeros(dofs.size), solver or SolverOptions())


def _problem_desc(spec: ProblemSpec, keep: list) -> capi.ProblemDesc:
    """C description of a problem; the arrays it points to are appended to `keep`."""
    coords = np.ascontiguousarray(spec.coords, dtype=np.float64)
    conn = np.ascontiguousarray(spec.connectivity, dtype=np.int32)
    keep += [coords, conn]
    nbcs = (capi.NaturalBC * max(1, len(spec.tractions)))()
    keep.append(nbcs)
    for k, (cells, local, vec) in enumerate(spec.tractions):
        cells = np.ascontiguousarray(cells, dtype=np.int32)
        local = np.ascontiguousarray(local, dtype=np.int32)
        keep += [cells, local]
        nbcs[k].num_faces = cells.size
        nbcs[k].face_cells = cells.ctypes.data_as(capi.i32p)
        nbcs[k].face_local_nodes = local.ctypes.data_as(capi.i32p)
        nbcs[k].vector = (C.c_double * 3)(*vec)
    dofs = np.ascontiguousarray(spec.bc_dofs, dtype=np.int32)
    vals = np.ascontiguousarray(spec.bc_values, dtype=np.float64)
    keep += [dofs, vals]
    desc = capi.ProblemDesc()
    desc.mesh = capi.MeshDesc(coords.shape[0], conn.shape[0], coords.ctypes.data_as(capi.f64p),
                              conn.ctypes.data_as(capi.i32p))
    desc.material = capi.Material(spec.youngs_modulus, spec.poissons_ratio)
    desc.penalty = capi.Penalty(spec.penalty_exponent, spec.penalty_minimum)
    desc.num_natural_bcs = len(spec.tractions)
    desc.natural_bcs = nbcs
    desc.essential_bcs = capi.EssentialBCs(dofs.size, dofs.ctypes.data_as(capi.i32p), vals.ctypes.data_as(capi.f64p))
    desc.solver = spec.solver.to_c()
    return desc


class EllipticProblem:
    """Elliptic::Problem with its VectorFunction and compliance criterion on one GPU.

    EllipticProblem.batch(specs) builds one handle over several independent problems (their
    disjoint union); node_offsets / cell_offsets locate each member in the union's vectors.
    """

    def __init__(self, spec: ProblemSpec, stream=None, _batch: list | None = None):
        import torch  # device memory and streams only

        self.torch = torch
        self.spec = spec
        self._keep = []
        h = C.c_void_p()
        if _batch is None:
            desc = _problem_desc(spec, self._keep)
            check(lib.plato_create(C.byref(desc), C.byref(h)))
        else:
            descs = (capi.ProblemDesc * len(_batch))()
            for k, sp in enumerate(_batch):
                descs[k] = _problem_desc(sp, self._keep)
            check(lib.plato_create_batch(len(_batch), descs, C.byref(h)))
        self.h = h
        self.set_stream(stream if stream is not None else torch.cuda.current_stream())
        nn, nc, nb = C.c_int32(), C.c_int32(), C.c_int64()
        check(lib.plato_get_sizes(h, C.byref(nn), C.byref(nc), C.byref(nb)), h)
        self.num_nodes, self.num_cells, self.num_blocks = nn.value, nc.value, nb.value
        self.num_dofs = 3 * self.num_nodes
        self.nz = self.num_nodes  # control entries (nodal layout)
        cnt = C.c_int32()
        check(lib.plato_batch_info(h, C.byref(cnt), None, None), h)
        self.count = cnt.value
        self.node_offsets = np.zeros(self.count + 1, np.int32)
        self.cell_offsets = np.zeros(self.count + 1, np.int32)
        check(lib.plato_batch_info(h, None, self.node_offsets.ctypes.data_as(capi.i32p),
                                   self.cell_offsets.ctypes.data_as(capi.i32p)), h)

    @classmethod
    def batch(cls, specs: list, stream=None) -> "EllipticProblem":
        """One handle over independent problems (shared material and penalty; solver options of
        specs[0]); solves run every member to its own tolerance in one batched flexible CG."""
        return cls(specs[0], stream, _batch=list(specs))

    def member_slices(self, dofs_per_node: int = 3):
        """Slices of member s in union node vectors with dofs_per_node entries per node."""
        o = self.node_offsets
        return [slice(dofs_per_node * int(o[s]), dofs_per_node * int(o[s + 1])) for s in range(self.count)]

    def batch_autotune(self, z) -> dict:
        """Times the batched solve's (tile rows, CTAs per SM) candidates and keeps the fastest."""
        t = capi.BatchTuning()
        check(lib.plato_batch_autotune(self.h, self._dev(z), C.byref(t)), self.h)
        return t.as_dict()

    def batch_last_stats(self) -> list:
        st = (capi.SolveStats * self.count)()
        check(lib.plato_batch_last_stats(self.h, st), self.h)
        return [x.as_dict() for x in st]

    def batch_criterion_values(self, z, u) -> np.ndarray:
        v = self.zeros(self.count)
        check(lib.plato_batch_criterion_values(self.h, self._dev(z), self._dev(u), self._dev(v)), self.h)
        return v.cpu().numpy()

    # -- plumbing ------------------------------------------------------------------------
    def set_control_layout(self, layout: str) -> None:
        """'nodal' (the reference's: a cell takes the mean of its nodes) or 'element' (one
        density per cell; control vectors and their gradients then have num_cells entries)."""
        code = {"nodal": capi.CONTROL_NODAL, "element": capi.CONTROL_ELEMENT}[layout]
        check(lib.plato_set_control_layout(self.h, code), self.h)
        self.nz = self.num_cells if code == capi.CONTROL_ELEMENT else self.num_nodes

    def set_stream(self, stream) -> None:
        self.stream = stream
        check(lib.plato_set_stream(self.h, C.c_void_p(stream.cuda_stream)), self.h)

    def set_solver(self, opts: SolverOptions) -> None:
        o = opts.to_c()
        check(lib.plato_set_solver_opts(self.h, C.byref(o)), self.h)
        self.spec.solver = opts

    def set_timing(self, enable: bool) -> None:
        check(lib.plato_set_timing(self.h, int(enable)), self.h)

    def instrumentation(self) -> dict:
        n, ms, k = C.c_int64(), C.c_double(), C.c_int64()
        check(lib.plato_get_instrumentation(self.h, C.byref(n), C.byref(ms), C.byref(k)), self.h)
        out = {"launches": n.value, "op_ms_total": ms.value, "op_timed": k.value}
        for kind, name in ((1, "inner"), (2, "assembly"), (3, "coarse_galerkin"), (4, "coarse_inverse"),
                           (5, "residual"), (6, "energy"), (7, "dcdz"), (8, "criterion")):
            t, c = C.c_double(), C.c_int64()
            check(lib.plato_get_kernel_timing(self.h, kind, C.byref(t), C.byref(c)), self.h)
            out[name + "_ms_total"], out[name + "_timed"] = t.value, c.value
        return out

    def sell_info(self) -> dict:
        """The solver's SELL-32 layout: slots (with slice padding) and the bytes per column
        index the FP16 preconditioner sweep reads."""
        slots, cb = C.c_int64(), C.c_int32()
        check(lib.plato_get_sell_info(self.h, C.byref(slots), C.byref(cb)), self.h)
        return {"total_slots": slots.value, "column_bytes": cb.value}

    def sweep_info(self) -> dict:
        """The FP16 sweep of the last flexible-CG solve: Chebyshev steps per launch (1: one
        launch per step) and the column reach in tiles of 512 rows (-1: not measured)."""
        steps, halo = C.c_int32(), C.c_int32()
        check(lib.plato_get_sweep_info(self.h, C.byref(steps), C.byref(halo)), self.h)
        return {"steps_per_launch": steps.value, "halo_tiles": halo.value}

    def reset_instrumentation(self) -> None:
        check(lib.plato_reset_instrumentation(self.h), self.h)

    def close(self) -> None:
        if getattr(self, "h", None):
            lib.plato_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _dev(self, t):
        assert t.is_cuda and t.is_contiguous(), "device tensors must be contiguous CUDA tensors"
        return C.c_void_p(t.data_ptr())

    def zeros(self, n, dtype=None):
        return self.torch.zeros(n, dtype=dtype or self.torch.float64, device="cuda")

    def to_dev(self, a: np.ndarray):
        return self.torch.from_numpy(np.ascontiguousarray(a)).cuda()

    # -- pattern ---------------------------------------------------------------------------
    def pattern(self):
        rm = self.zeros(self.num_nodes + 1, self.torch.int32)
        cols = self.zeros(self.num_blocks, self.torch.int32)
        check(lib.plato_jacobian_pattern(self.h, self._dev(rm), self._dev(cols)), self.h)
        return rm, cols

    # -- VectorFunction ----------------------------------------------------------------------
    def vf_value(self, u, z):
        R = self.zeros(self.num_dofs)
        check(lib.plato_vf_value(self.h, self._dev(u), self._dev(z), self._dev(R)), self.h)
        return R

    def vf_gradient_u(self, u, z):
        K = self.zeros(9 * self.num_blocks)
        check(lib.plato_vf_gradient_u(self.h, self._dev(u), self._dev(z), self._dev(K)), self.h)
        return K

    def vf_gradient_u_T(self, u, z):
        K = self.zeros(9 * self.num_blocks)
        check(lib.plato_vf_gradient_u_T(self.h, self._dev(u), self._dev(z), self._dev(K)), self.h)
        return K

    def vf_gradient_z(self, u, z):
        G = self.zeros(3 * self.num_blocks)
        check(lib.plato_vf_gradient_z(self.h, self._dev(u), self._dev(z), self._dev(G)), self.h)
        return G

    def vf_gradient_z_apply(self, u, z, lam, out):
        check(lib.plato_vf_gradient_z_apply(self.h, self._dev(u), self._dev(z), self._dev(lam), self._dev(out)),
              self.h)
        return out

    # -- ScalarFunction ------------------------------------------------------------------------
    def sf_value(self, u, z) -> float:
        v = C.c_double()
        check(lib.plato_sf_value(self.h, self._dev(u), self._dev(z), C.byref(v)), self.h)
        return v.value

    def sf_gradient_u(self, u, z):
        g = self.zeros(self.num_dofs)
        check(lib.plato_sf_gradient_u(self.h, self._dev(u), self._dev(z), self._dev(g)), self.h)
        return g

    def sf_gradient_z(self, u, z):
        g = self.zeros(self.nz)
        check(lib.plato_sf_gradient_z(self.h, self._dev(u), self._dev(z), self._dev(g)), self.h)
        return g

    # -- helpers ---------------------------------------------------------------------------------
    def apply_constraints(self, entries, rhs, scale=1.0):
        check(lib.plato_apply_constraints(self.h, self._dev(entries), self._dev(rhs) if rhs is not None else None,
                                          scale), self.h)

    def matvec_plus(self, rb, cb, entries, x, y):
        check(lib.plato_matvec_plus(self.h, rb, cb, self._dev(entries), self._dev(x), self._dev(y)), self.h)
        return y

    def volume_value(self, z, exponent=1.0, minimum=0.0) -> float:
        """Geometric Volume criterion sum_e vol_e s_v(rho_e) (penalty exponent 1, minimum 0 by default)."""
        v, pen = C.c_double(), capi.Penalty(exponent, minimum)
        check(lib.plato_volume_value(self.h, self._dev(z), C.byref(pen), C.byref(v)), self.h)
        return v.value

    def volume_gradient_z(self, z, exponent=1.0, minimum=0.0):
        g, pen = self.zeros(self.nz), capi.Penalty(exponent, minimum)
        check(lib.plato_volume_gradient_z(self.h, self._dev(z), C.byref(pen), self._dev(g)), self.h)
        return g

    def apply_operator(self, z, x, operator_kind=capi.OPERATOR_ASSEMBLED):
        """y = K_c(z) x, K_c the Dirichlet-constrained stiffness (assembled or matrix-free)."""
        y = self.zeros(self.num_dofs)
        check(lib.plato_apply_operator(self.h, self._dev(z), operator_kind, self._dev(x), self._dev(y)), self.h)
        return y

    def solver_solve(self, entries, x, b):
        st = capi.SolveStats()
        check(lib.plato_solver_solve(self.h, self._dev(entries), self._dev(x), self._dev(b), C.byref(st)), self.h)
        return st.as_dict()

    # -- Problem -------------------------------------------------------------------------------------
    def solution(self, z, u0=None, raise_on_error=True):
        u = self.zeros(self.num_dofs)
        st = capi.SolveStats()
        rc = lib.plato_problem_solution(self.h, self._dev(z), self._dev(u0) if u0 is not None else None,
                                        self._dev(u), C.byref(st))
        if raise_on_error:
            check(rc, self.h)
        return u, st.as_dict() | {"rc": rc}

    def solution_subspace(self, z, W, u0=None):
        """Problem::solution from the guess u0 (or zero) improved on span(P W), W a (k, 3N)
        device array; returns (u, stats, residual ratio of the subspace correction)."""
        u = self.zeros(self.num_dofs)
        st = capi.SolveStats()
        ratio = C.c_double()
        check(lib.plato_problem_solution_subspace(self.h, self._dev(z), self._dev(u0) if u0 is not None else None,
                                                  self._dev(W), int(W.shape[0]), self._dev(u), C.byref(st),
                                                  C.byref(ratio)), self.h)
        return u, st.as_dict(), ratio.value

    def solution_deflated(self, z, W, u0=None):
        """Problem::solution with the Galerkin guess on span(P W) and deflated Krylov directions
        (W a (k, 3N) device array); returns (u, stats, residual ratio of the guess)."""
        u = self.zeros(self.num_dofs)
        st = capi.SolveStats()
        ratio = C.c_double()
        check(lib.plato_problem_solution_deflated(self.h, self._dev(z), self._dev(u0) if u0 is not None else None,
                                                  self._dev(W), int(W.shape[0]), self._dev(u), C.byref(st),
                                                  C.byref(ratio)), self.h)
        return u, st.as_dict(), ratio.value

    def criterion_value(self, z, u) -> float:
        v = C.c_double()
        check(lib.plato_problem_criterion_value(self.h, self._dev(z), self._dev(u), C.byref(v)), self.h)
        return v.value

    def criterion_value_and_gradient(self, z, u):
        """Compliance and dC/dz together (one pass over the cells with the self-adjoint
        shortcut); returns (value, dC/dz, stats)."""
        g = self.zeros(self.nz)
        v = C.c_double()
        st = capi.SolveStats()
        check(lib.plato_problem_criterion_value_and_gradient(self.h, self._dev(z), self._dev(u), C.byref(v),
                                                             self._dev(g), C.byref(st)), self.h)
        return v.value, g, st.as_dict()

    def criterion_gradient(self, z, u):
        g = self.zeros(self.nz)
        st = capi.SolveStats()
        check(lib.plato_problem_criterion_gradient(self.h, self._dev(z), self._dev(u), self._dev(g), C.byref(st)),
              self.h)
        return g, st.as_dict()

    def solve_and_gradient_host(self, z: np.ndarray, u0: np.ndarray | None = None, u_out=None, g_out=None):
        """One optimisation step on host (numpy) buffers; returns (u, value, dfdz, stats)."""
        z = np.ascontiguousarray(z, dtype=np.float64)
        u = u_out if u_out is not None else np.empty(self.num_dofs)
        g = g_out if g_out is not None else np.empty(self.nz)
        v = C.c_double()
        st = capi.SolveStats()
        rc = lib.plato_problem_solve_and_gradient_host(self.h, _np_ptr(z), _np_ptr(u0) if u0 is not None else None,
                                                       _np_ptr(u), C.byref(v), _np_ptr(g), C.byref(st))
        check(rc, self.h)
        return u, v.value, g, st.as_dict()


class HelmholtzFilter:
    """Helmholtz density filter (src/helmholtz/Problem.hpp) over a tet mesh with length scale L
    and, optionally, the surface term with multiplier alpha on `surface_faces` = (owning cells,
    3 local node ordinals) - the exterior faces outside the symmetry planes, e.g.
    `mesh.exterior_faces(connectivity, symmetry_nodes)`.  One unknown per node; vectors are
    device (torch) arrays of num_nodes values."""

    def __init__(self, coords, connectivity, length_scale: float, surface_length_scale: float = 0.0,
                 surface_faces=None, tolerance: float = 1e-12, max_iterations: int = 100000, stream=None):
        import torch

        self.torch = torch
        coords = np.ascontiguousarray(coords, dtype=np.float64)
        conn = np.ascontiguousarray(connectivity, dtype=np.int32)
        if surface_faces is None:
            fc, fl = np.zeros(0, np.int32), np.zeros((0, 3), np.int32)
        else:
            fc = np.ascontiguousarray(surface_faces[0], dtype=np.int32)
            fl = np.ascontiguousarray(surface_faces[1], dtype=np.int32)
        mesh = capi.MeshDesc(coords.shape[0], conn.shape[0], coords.ctypes.data_as(capi.f64p),
                             conn.ctypes.data_as(capi.i32p))
        opts = SolverOptions(tolerance=tolerance, max_iterations=max_iterations).to_c()
        desc = capi.HelmholtzDesc(mesh, float(length_scale), float(surface_length_scale), fc.size,
                                  fc.ctypes.data_as(capi.i32p), fl.ctypes.data_as(capi.i32p), opts)
        h = C.c_void_p()
        check(lib.plato_create_helmholtz(C.byref(desc), C.byref(h)))
        self.h = h
        self.length_scale = float(length_scale)
        self.surface_length_scale = float(surface_length_scale)
        self.stream = stream if stream is not None else torch.cuda.current_stream()
        check(lib.plato_set_stream(h, C.c_void_p(self.stream.cuda_stream)), h)
        nn, nc, nb = C.c_int32(), C.c_int32(), C.c_int64()
        check(lib.plato_get_sizes(h, C.byref(nn), C.byref(nc), C.byref(nb)), h)
        self.num_nodes, self.num_cells, self.num_blocks = nn.value, nc.value, nb.value

    def close(self) -> None:
        if getattr(self, "h", None):
            lib.plato_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _dev(self, t):
        return C.c_void_p(t.data_ptr())

    def to_dev(self, a):
        return self.torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64)).cuda()

    def zeros(self, n, dtype=None):
        return self.torch.zeros(n, dtype=dtype or self.torch.float64, device="cuda")

    set_timing = EllipticProblem.set_timing
    instrumentation = EllipticProblem.instrumentation
    reset_instrumentation = EllipticProblem.reset_instrumentation

    def pattern(self):
        rm = self.zeros(self.num_nodes + 1, self.torch.int32)
        cols = self.zeros(self.num_blocks, self.torch.int32)
        check(lib.plato_jacobian_pattern(self.h, self._dev(rm), self._dev(cols)), self.h)
        return rm, cols

    def value(self, filtered, control):
        R = self.zeros(self.num_nodes)
        check(lib.plato_helmholtz_value(self.h, self._dev(filtered), self._dev(control), self._dev(R)), self.h)
        return R

    def gradient_u(self):
        K = self.zeros(self.num_blocks)
        check(lib.plato_helmholtz_gradient_u(self.h, self._dev(K)), self.h)
        return K

    def gradient_z(self):
        K = self.zeros(self.num_blocks)
        check(lib.plato_helmholtz_gradient_z(self.h, self._dev(K)), self.h)
        return K

    def solution(self, control):
        f = self.zeros(self.num_nodes)
        st = capi.SolveStats()
        check(lib.plato_helmholtz_solution(self.h, self._dev(control), self._dev(f), C.byref(st)), self.h)
        return f, st.as_dict()

    def criterion_gradient(self, dfdfiltered):
        g = self.zeros(self.num_nodes)
        st = capi.SolveStats()
        check(lib.plato_helmholtz_criterion_gradient(self.h, self._dev(dfdfiltered), self._dev(g), C.byref(st)),
              self.h)
        return g, st.as_dict()
