"""ctypes binding of the CPU FP64 oracle (oracle/plato_oracle.cpp).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the CPU-baseline leg
of bench.py as the checker.  Nothing in the product path imports this module.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libplato_oracle.so"

i32p = C.POINTER(C.c_int32)
f64p = C.POINTER(C.c_double)


class OracleProblem(C.Structure):
    _fields_ = [("num_nodes", C.c_int32), ("num_cells", C.c_int32), ("coords", f64p),
                ("connectivity", i32p), ("youngs_modulus", C.c_double), ("poissons_ratio", C.c_double),
                ("penalty_exponent", C.c_double), ("penalty_minimum", C.c_double),
                ("num_traction_faces", C.c_int32), ("face_cells", i32p), ("face_local_nodes", i32p),
                ("traction", C.c_double * 3), ("num_bc_dofs", C.c_int32), ("bc_dofs", i32p),
                ("bc_values", f64p), ("cell_control", C.c_int32)]


class OracleStats(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("relative_residual", C.c_double), ("converged", C.c_int32)]


class OracleHelmholtz(C.Structure):
    _fields_ = [("length_scale", C.c_double), ("surface_length_scale", C.c_double), ("num_faces", C.c_int32),
                ("face_cells", i32p), ("face_local_nodes", i32p)]


def _build() -> None:
    if not LIB_PATH.exists():
        cxx = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"
        subprocess.run(["make", "-s", "-C", str(HERE), f"ORACLE_CXX={cxx}"], check=True)


def _load() -> C.CDLL:
    _build()
    lib = C.CDLL(str(LIB_PATH))
    P = C.POINTER(OracleProblem)
    H = C.POINTER(OracleHelmholtz)
    vp = C.c_void_p
    sig = {
        "oracle_cell_fields": ([P, vp, vp, vp, vp, vp, vp], None),
        "oracle_graph_nnz": ([P], C.c_int64),
        "oracle_graph": ([P, vp, vp], None),
        "oracle_vf_value": ([P, vp, vp, vp], None),
        "oracle_vf_gradient_u": ([P, vp, vp, vp, vp, vp], None),
        "oracle_vf_gradient_u_T": ([P, vp, vp, vp, vp, vp], None),
        "oracle_vf_gradient_z": ([P, vp, vp, vp, vp, vp], None),
        "oracle_sf_value": ([P, vp, vp], C.c_double),
        "oracle_sf_gradient_u": ([P, vp, vp, vp], None),
        "oracle_sf_gradient_z": ([P, vp, vp, vp], None),
        "oracle_apply_block_constraints": ([C.c_int32, vp, vp, vp, vp, C.c_int32, vp, vp, C.c_double], None),
        "oracle_matvec_plus": ([C.c_int32, C.c_int32, C.c_int32, vp, vp, vp, vp, vp], None),
        "oracle_pcg_jacobi": ([C.c_int32, vp, vp, vp, vp, vp, C.c_double, C.c_int32, C.POINTER(OracleStats)], C.c_int),
        "oracle_refine_solution": ([C.c_int32, vp, vp, vp, vp, vp, C.c_double, C.c_double, C.c_int32, C.c_int32,
                                    C.POINTER(OracleStats)], C.c_int),
        "oracle_problem_solution": ([P, vp, vp, C.c_double, C.c_int32, C.POINTER(OracleStats)], C.c_int),
        "oracle_problem_criterion_gradient": ([P, vp, vp, C.c_int32, C.c_double, C.c_int32, vp,
                                               C.POINTER(OracleStats)], C.c_int),
        "oracle_num_threads": ([], C.c_int),
        "oracle_set_num_threads": ([C.c_int], None),
        "oracle_volume_value": ([P, vp, C.c_double, C.c_double], C.c_double),
        "oracle_volume_gradient_z": ([P, vp, C.c_double, C.c_double, vp], None),
        "oracle_helmholtz_value": ([P, H, vp, vp, vp], None),
        "oracle_helmholtz_gradient_u": ([P, H, vp, vp, vp], None),
        "oracle_helmholtz_gradient_z": ([P, vp, vp, vp], None),
        "oracle_helmholtz_solution": ([P, H, vp, vp, C.c_double, C.c_int32, C.POINTER(OracleStats)], C.c_int),
        "oracle_helmholtz_criterion_gradient": ([P, H, vp, vp, C.c_double, C.c_int32,
                                                 C.POINTER(OracleStats)], C.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return lib


lib = _load()


def _p(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


class Oracle:
    """FP64 CPU restatement of the reference path on one mesh + material + BCs."""

    def __init__(self, coords, connectivity, E=1.0, nu=0.3, p=3.0, rho_min=1e-9,
                 traction_faces=None, traction=(0.0, 0.0, 0.0), bc_dofs=None, bc_values=None, cell_control=False):
        self.coords = np.ascontiguousarray(coords, dtype=np.float64)
        self.conn = np.ascontiguousarray(connectivity, dtype=np.int32)
        if traction_faces is None:
            fc, fl = np.zeros(0, np.int32), np.zeros((0, 3), np.int32)
        else:
            fc, fl = traction_faces
        self.fc = np.ascontiguousarray(fc, dtype=np.int32)
        self.fl = np.ascontiguousarray(fl, dtype=np.int32)
        self.bc_dofs = np.ascontiguousarray(bc_dofs if bc_dofs is not None else np.zeros(0), dtype=np.int32)
        self.bc_values = np.ascontiguousarray(bc_values if bc_values is not None else np.zeros(self.bc_dofs.size),
                                              dtype=np.float64)
        P = OracleProblem()
        P.num_nodes = self.coords.shape[0]
        P.num_cells = self.conn.shape[0]
        P.coords = self.coords.ctypes.data_as(f64p)
        P.connectivity = self.conn.ctypes.data_as(i32p)
        P.youngs_modulus, P.poissons_ratio, P.penalty_exponent, P.penalty_minimum = E, nu, p, rho_min
        P.num_traction_faces = self.fc.size
        P.face_cells = self.fc.ctypes.data_as(i32p)
        P.face_local_nodes = self.fl.ctypes.data_as(i32p)
        P.traction = (C.c_double * 3)(*traction)
        P.num_bc_dofs = self.bc_dofs.size
        P.bc_dofs = self.bc_dofs.ctypes.data_as(i32p)
        P.bc_values = self.bc_values.ctypes.data_as(f64p)
        P.cell_control = int(bool(cell_control))
        self.P = P
        self.N = P.num_nodes
        self.C = P.num_cells
        self.nz = self.C if cell_control else self.N  # control entries
        self._graph = None

    @classmethod
    def from_spec(cls, spec, cell_control=False) -> "Oracle":
        (fc, fl, vec) = spec.tractions[0] if spec.tractions else (None, None, (0.0, 0.0, 0.0))
        return cls(spec.coords, spec.connectivity, spec.youngs_modulus, spec.poissons_ratio,
                   spec.penalty_exponent, spec.penalty_minimum,
                   (fc, fl) if fc is not None else None, vec, spec.bc_dofs, spec.bc_values, cell_control)

    def cell_fields(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        g = np.empty((self.C, 4, 3))
        v = np.empty(self.C)
        e = np.empty((self.C, 6))
        s = np.empty((self.C, 6))
        r = np.empty((self.C, 12))
        lib.oracle_cell_fields(C.byref(self.P), _p(u), _p(g), _p(v), _p(e), _p(s), _p(r))
        return g, v, e, s, r

    def graph(self):
        if self._graph is None:
            nnz = lib.oracle_graph_nnz(C.byref(self.P))
            rm = np.empty(self.N + 1, np.int32)
            cols = np.empty(nnz, np.int32)
            lib.oracle_graph(C.byref(self.P), _p(rm), _p(cols))
            self._graph = (rm, cols)
        return self._graph

    def vf_value(self, u, z):
        R = np.empty(3 * self.N)
        lib.oracle_vf_value(C.byref(self.P), _p(np.ascontiguousarray(u, np.float64)),
                            _p(np.ascontiguousarray(z, np.float64)), _p(R))
        return R

    def vf_gradient_u(self, u, z, transpose=False):
        rm, cols = self.graph()
        K = np.empty(9 * cols.size)
        fn = lib.oracle_vf_gradient_u_T if transpose else lib.oracle_vf_gradient_u
        fn(C.byref(self.P), _p(np.ascontiguousarray(u, np.float64)), _p(np.ascontiguousarray(z, np.float64)),
           _p(rm), _p(cols), _p(K))
        return K

    def vf_gradient_z(self, u, z):
        rm, cols = self.graph()
        G = np.empty(3 * cols.size)
        lib.oracle_vf_gradient_z(C.byref(self.P), _p(np.ascontiguousarray(u, np.float64)),
                                 _p(np.ascontiguousarray(z, np.float64)), _p(rm), _p(cols), _p(G))
        return G

    def sf_value(self, u, z) -> float:
        return lib.oracle_sf_value(C.byref(self.P), _p(np.ascontiguousarray(u, np.float64)),
                                   _p(np.ascontiguousarray(z, np.float64)))

    def sf_gradient_u(self, u, z):
        g = np.empty(3 * self.N)
        lib.oracle_sf_gradient_u(C.byref(self.P), _p(np.ascontiguousarray(u, np.float64)),
                                 _p(np.ascontiguousarray(z, np.float64)), _p(g))
        return g

    def sf_gradient_z(self, u, z):
        g = np.empty(self.nz)
        lib.oracle_sf_gradient_z(C.byref(self.P), _p(np.ascontiguousarray(u, np.float64)),
                                 _p(np.ascontiguousarray(z, np.float64)), _p(g))
        return g

    def apply_constraints(self, K, rhs, scale=1.0):
        rm, cols = self.graph()
        lib.oracle_apply_block_constraints(self.N, _p(rm), _p(cols), _p(K), _p(rhs), self.bc_dofs.size,
                                           _p(self.bc_dofs), _p(self.bc_values), scale)

    def matvec_plus(self, rb, cb, A, x, y):
        rm, cols = self.graph()
        lib.oracle_matvec_plus(self.N, rb, cb, _p(rm), _p(cols), _p(A), _p(np.ascontiguousarray(x, np.float64)),
                               _p(y))
        return y

    def pcg(self, A, b, x=None, tol=1e-10, max_it=100000):
        rm, cols = self.graph()
        x = np.zeros(3 * self.N) if x is None else np.array(x, dtype=np.float64)
        st = OracleStats()
        lib.oracle_pcg_jacobi(self.N, _p(rm), _p(cols), _p(A), _p(np.ascontiguousarray(b, np.float64)), _p(x),
                              tol, max_it, C.byref(st))
        return x, {"iterations": st.iterations, "relative_residual": st.relative_residual,
                   "converged": st.converged}

    def refine(self, A, b, u, tol=1e-13, inner_tol=1e-5, max_rounds=6, max_it=1000000):
        """Iterative refinement of A u = b from u (any float array) with a long double iterate
        and long double residuals; returns (u as np.longdouble, stats)."""
        rm, cols = self.graph()
        x = np.array(u, dtype=np.longdouble)
        st = OracleStats()
        lib.oracle_refine_solution(self.N, _p(rm), _p(cols), _p(A), _p(np.ascontiguousarray(b, np.float64)), _p(x),
                                   tol, inner_tol, max_rounds, max_it, C.byref(st))
        return x, {"iterations": st.iterations, "relative_residual": st.relative_residual,
                   "converged": st.converged}

    def solution_refined(self, z, tol=1e-13, tol0=1e-10, max_it=1000000):
        """Problem::solution to a long double relative residual <= tol: FP64 Jacobi-PCG to
        tol0, then iterative refinement.  Returns (u as float64, u as np.longdouble, stats)."""
        n = 3 * self.N
        K = self.vf_gradient_u(np.zeros(n), z)
        rhs = -self.vf_value(np.zeros(n), z)
        self.apply_constraints(K, rhs, 1.0)
        u0, st0 = self.pcg(K, rhs, tol=tol0, max_it=max_it)
        uld, st = self.refine(K, rhs, u0, tol=tol, max_it=max_it)
        st["iterations"] += st0["iterations"]
        return uld.astype(np.float64), uld, st

    def solution(self, z, tol=1e-10, max_it=100000):
        u = np.empty(3 * self.N)
        st = OracleStats()
        lib.oracle_problem_solution(C.byref(self.P), _p(np.ascontiguousarray(z, np.float64)), _p(u), tol, max_it,
                                    C.byref(st))
        return u, {"iterations": st.iterations, "relative_residual": st.relative_residual,
                   "converged": st.converged}

    def criterion_gradient(self, z, u, self_adjoint=True, tol=1e-10, max_it=100000):
        g = np.empty(self.nz)
        st = OracleStats()
        lib.oracle_problem_criterion_gradient(C.byref(self.P), _p(np.ascontiguousarray(z, np.float64)),
                                              _p(np.ascontiguousarray(u, np.float64)), int(self_adjoint), tol,
                                              max_it, _p(g), C.byref(st))
        return g

    def volume_value(self, z, p=1.0, m=0.0) -> float:
        return lib.oracle_volume_value(C.byref(self.P), _p(np.ascontiguousarray(z, np.float64)), p, m)

    def volume_gradient_z(self, z, p=1.0, m=0.0):
        g = np.empty(self.nz)
        lib.oracle_volume_gradient_z(C.byref(self.P), _p(np.ascontiguousarray(z, np.float64)), p, m, _p(g))
        return g

    # -- Helmholtz density filter (scalar, one value per node) ------------------------------
    # `surface` = (alpha, face_cells, face_local_nodes): "Surface Length Scale" and its faces
    def _helm(self, L, surface):
        if surface is None:
            return OracleHelmholtz(L, 0.0, 0, None, None)
        alpha, cells, local = surface
        cells = np.ascontiguousarray(cells, np.int32)
        local = np.ascontiguousarray(local, np.int32)
        self._helm_keep = (cells, local)
        return OracleHelmholtz(L, alpha, cells.size, cells.ctypes.data_as(i32p), local.ctypes.data_as(i32p))

    def helmholtz_value(self, L, filtered, control, surface=None):
        R = np.empty(self.N)
        H = self._helm(L, surface)
        lib.oracle_helmholtz_value(C.byref(self.P), C.byref(H), _p(np.ascontiguousarray(filtered, np.float64)),
                                   _p(np.ascontiguousarray(control, np.float64)), _p(R))
        return R

    def helmholtz_gradient_u(self, L, surface=None):
        rm, cols = self.graph()
        K = np.empty(cols.size)
        H = self._helm(L, surface)
        lib.oracle_helmholtz_gradient_u(C.byref(self.P), C.byref(H), _p(rm), _p(cols), _p(K))
        return K

    def helmholtz_gradient_z(self):
        rm, cols = self.graph()
        K = np.empty(cols.size)
        lib.oracle_helmholtz_gradient_z(C.byref(self.P), _p(rm), _p(cols), _p(K))
        return K

    def helmholtz_solution(self, L, control, tol=1e-12, max_it=100000, surface=None):
        f = np.empty(self.N)
        st = OracleStats()
        H = self._helm(L, surface)
        lib.oracle_helmholtz_solution(C.byref(self.P), C.byref(H), _p(np.ascontiguousarray(control, np.float64)),
                                      _p(f), tol, max_it, C.byref(st))
        return f, {"iterations": st.iterations, "relative_residual": st.relative_residual,
                   "converged": st.converged}

    def helmholtz_criterion_gradient(self, L, dfdfiltered, tol=1e-12, max_it=100000, surface=None):
        g = np.empty(self.N)
        st = OracleStats()
        H = self._helm(L, surface)
        lib.oracle_helmholtz_criterion_gradient(C.byref(self.P), C.byref(H),
                                                _p(np.ascontiguousarray(dfdfiltered, np.float64)), _p(g), tol, max_it,
                                                C.byref(st))
        return g, {"iterations": st.iterations, "relative_residual": st.relative_residual,
                   "converged": st.converged}

    @staticmethod
    def num_threads() -> int:
        return lib.oracle_num_threads()

    @staticmethod
    def set_num_threads(n: int) -> None:
        lib.oracle_set_num_threads(int(n))
