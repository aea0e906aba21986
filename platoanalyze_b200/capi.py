"""ctypes binding of the C ABI in include/plato_b200.h.

The CUDA library is required: importing this module raises if
platoanalyze_b200/lib/libplato_b200.so is missing.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libplato_b200.so"

CONTROL_NODAL, CONTROL_ELEMENT = 0, 1
OK, BAD_INPUT, NOT_CONVERGED, NONFINITE, DEVICE_TIMEOUT, CUDA_ERROR, OUT_OF_MEMORY, NOT_SUPPORTED = range(8)
LAYOUT_SCALAR_FIELD, LAYOUT_SCALAR_VALUE, LAYOUT_SCALAR_PARAMETER = range(3)
STATUS_NAMES = ["OK", "BAD_INPUT", "NOT_CONVERGED", "NONFINITE", "DEVICE_TIMEOUT", "CUDA_ERROR",
                "OUT_OF_MEMORY", "NOT_SUPPORTED"]

OPERATOR_ASSEMBLED, OPERATOR_MATRIX_FREE = 0, 1
PRECISION_FP64, PRECISION_MIXED_FP32, PRECISION_MIXED_BF16, PRECISION_MIXED_FP16 = 0, 1, 2, 3
PRECISION_MIXED_FP32_ASSEMBLED = 4  # FP32 element assembly of the preconditioner matrix (matrix-free outer)

i32p = C.POINTER(C.c_int32)
f64p = C.POINTER(C.c_double)


class MeshDesc(C.Structure):
    _fields_ = [("num_nodes", C.c_int32), ("num_cells", C.c_int32),
                ("coords", f64p), ("connectivity", i32p)]


class Material(C.Structure):
    _fields_ = [("youngs_modulus", C.c_double), ("poissons_ratio", C.c_double)]


class Penalty(C.Structure):
    _fields_ = [("exponent", C.c_double), ("minimum_value", C.c_double)]


class NaturalBC(C.Structure):
    _fields_ = [("num_faces", C.c_int32), ("face_cells", i32p), ("face_local_nodes", i32p),
                ("vector", C.c_double * 3)]


class EssentialBCs(C.Structure):
    _fields_ = [("num_dofs", C.c_int32), ("dofs", i32p), ("values", f64p)]


class SolverOpts(C.Structure):
    _fields_ = [("tolerance", C.c_double), ("max_iterations", C.c_int32), ("operator_kind", C.c_int32),
                ("precision", C.c_int32), ("self_adjoint", C.c_int32), ("chebyshev_ratio", C.c_double),
                ("chebyshev_degree", C.c_int32), ("coarse_cells", C.c_int32 * 3),
                ("fallback_max_iterations", C.c_int32), ("chebyshev_kind", C.c_int32),
                ("sweep_steps", C.c_int32), ("sweep_lag", C.c_int32)]


class ProblemDesc(C.Structure):
    _fields_ = [("mesh", MeshDesc), ("material", Material), ("penalty", Penalty),
                ("num_natural_bcs", C.c_int32), ("natural_bcs", C.POINTER(NaturalBC)),
                ("essential_bcs", EssentialBCs), ("solver", SolverOpts)]


class HelmholtzDesc(C.Structure):
    _fields_ = [("mesh", MeshDesc), ("length_scale", C.c_double), ("surface_length_scale", C.c_double),
                ("num_surface_faces", C.c_int32), ("surface_face_cells", i32p),
                ("surface_face_local_nodes", i32p), ("solver", SolverOpts)]


class SolveStats(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("refinements", C.c_int32), ("relative_residual", C.c_double),
                ("converged", C.c_int32), ("status", C.c_int32), ("fallback", C.c_int32)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class BatchTuning(C.Structure):
    _fields_ = [("tile_rows", C.c_int32), ("ctas_per_sm", C.c_int32), ("candidates", C.c_int32),
                ("iterations", C.c_int32), ("tile_rows_tried", C.c_int32 * 16), ("ctas_per_sm_tried", C.c_int32 * 16),
                ("ms_tried", C.c_double * 16)]

    def as_dict(self) -> dict:
        k = self.candidates
        return {"tile_rows": self.tile_rows, "ctas_per_sm": self.ctas_per_sm, "iterations": self.iterations,
                "tried": [{"tile_rows": self.tile_rows_tried[i], "ctas_per_sm": self.ctas_per_sm_tried[i],
                           "ms": self.ms_tried[i]} for i in range(k)]}


class PlatoError(RuntimeError):
    def __init__(self, status: int, msg: str):
        name = STATUS_NAMES[status] if 0 <= status < len(STATUS_NAMES) else str(status)
        super().__init__(f"{name}: {msg}")
        self.status = status


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(f"CUDA library not built: {LIB_PATH} (run python -m platoanalyze_b200.build)")
    lib = C.CDLL(str(LIB_PATH))
    vp = C.c_void_p
    sig = {
        "plato_create": ([C.POINTER(ProblemDesc), C.POINTER(vp)], C.c_int),
        "plato_destroy": ([vp], C.c_int),
        "plato_last_error": ([vp], C.c_char_p),
        "plato_set_stream": ([vp, vp], C.c_int),
        "plato_set_solver_opts": ([vp, C.POINTER(SolverOpts)], C.c_int),
        "plato_set_control_layout": ([vp, C.c_int32], C.c_int),
        "plato_batch_autotune": ([vp, vp, C.POINTER(BatchTuning)], C.c_int),
        "plato_set_timing": ([vp, C.c_int32], C.c_int),
        "plato_get_instrumentation": ([vp, C.POINTER(C.c_int64), f64p, C.POINTER(C.c_int64)], C.c_int),
        "plato_reset_instrumentation": ([vp], C.c_int),
        "plato_get_kernel_timing": ([vp, C.c_int32, f64p, C.POINTER(C.c_int64)], C.c_int),
        "plato_get_sell_info": ([vp, C.POINTER(C.c_int64), C.POINTER(C.c_int32)], C.c_int),
        "plato_get_sweep_info": ([vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32)], C.c_int),
        "plato_test_stall_next_sweep": ([vp], C.c_int),
        "plato_get_sizes": ([vp, i32p, i32p, C.POINTER(C.c_int64)], C.c_int),
        "plato_jacobian_pattern": ([vp, vp, vp], C.c_int),
        "plato_vf_value": ([vp, vp, vp, vp], C.c_int),
        "plato_vf_gradient_u": ([vp, vp, vp, vp], C.c_int),
        "plato_vf_gradient_u_T": ([vp, vp, vp, vp], C.c_int),
        "plato_vf_gradient_z": ([vp, vp, vp, vp], C.c_int),
        "plato_vf_gradient_z_apply": ([vp, vp, vp, vp, vp], C.c_int),
        "plato_sf_value": ([vp, vp, vp, f64p], C.c_int),
        "plato_sf_gradient_u": ([vp, vp, vp, vp], C.c_int),
        "plato_sf_gradient_z": ([vp, vp, vp, vp], C.c_int),
        "plato_apply_constraints": ([vp, vp, vp, C.c_double], C.c_int),
        "plato_matvec_plus": ([vp, C.c_int32, C.c_int32, vp, vp, vp], C.c_int),
        "plato_apply_operator": ([vp, vp, C.c_int32, vp, vp], C.c_int),
        "plato_volume_value": ([vp, vp, C.POINTER(Penalty), f64p], C.c_int),
        "plato_volume_gradient_z": ([vp, vp, C.POINTER(Penalty), vp], C.c_int),
        "plato_solver_solve": ([vp, vp, vp, vp, C.POINTER(SolveStats)], C.c_int),
        "plato_problem_solution": ([vp, vp, vp, vp, C.POINTER(SolveStats)], C.c_int),
        "plato_problem_criterion_value": ([vp, vp, vp, f64p], C.c_int),
        "plato_problem_criterion_gradient": ([vp, vp, vp, vp, C.POINTER(SolveStats)], C.c_int),
        "plato_problem_criterion_value_and_gradient": ([vp, vp, vp, f64p, vp, C.POINTER(SolveStats)], C.c_int),
        "plato_problem_solve_and_gradient_host": ([vp, vp, vp, vp, f64p, vp, C.POINTER(SolveStats)], C.c_int),
        "plato_sf_value_noalloc": ([C.c_int32, C.c_int32, vp, vp, vp, vp, C.POINTER(Material), C.POINTER(Penalty),
                                    vp, vp], C.c_int),
        "plato_create_batch": ([C.c_int32, C.POINTER(ProblemDesc), C.POINTER(vp)], C.c_int),
        "plato_batch_info": ([vp, i32p, i32p, i32p], C.c_int),
        "plato_batch_last_stats": ([vp, C.POINTER(SolveStats)], C.c_int),
        "plato_batch_criterion_values": ([vp, vp, vp, vp], C.c_int),
        "plato_problem_solution_subspace": ([vp, vp, vp, vp, C.c_int32, vp, C.POINTER(SolveStats), f64p], C.c_int),
        "plato_problem_solution_deflated": ([vp, vp, vp, vp, C.c_int32, vp, C.POINTER(SolveStats), f64p], C.c_int),
        "plato_unet_create": ([i32p, C.c_int32, C.POINTER(vp)], C.c_int),
        "plato_unet_destroy": ([vp], C.c_int),
        "plato_unet_set_stream": ([vp, vp], C.c_int),
        "plato_unet_set_conv_kernel": ([vp, C.c_int32], C.c_int),
        "plato_unet_check": ([vp], C.c_int),
        "plato_unet_last_error": ([], C.c_char_p),
        "plato_unet_num_params": ([vp, C.POINTER(C.c_int64)], C.c_int),
        "plato_unet_set_params": ([vp, vp], C.c_int),
        "plato_unet_get_params": ([vp, vp], C.c_int),
        "plato_unet_forward": ([vp, C.c_int32, vp, vp], C.c_int),
        "plato_unet_loss_and_gradients": ([vp, C.c_int32, vp, vp, f64p, vp], C.c_int),
        "plato_unet_adam_step": ([vp, C.c_float, C.c_int32], C.c_int),
        "plato_unet_features": ([i32p, vp, i32p, vp, vp], C.c_int),
        "plato_unet_subspace": ([i32p, vp, i32p, vp, vp], C.c_int),
        "plato_box_smooth": ([i32p, C.c_int32, C.c_int32, vp, vp, vp], C.c_int),
        "plato_box_resample": ([i32p, i32p, C.c_int32, vp, vp, vp], C.c_int),
        "plato_create_helmholtz": ([C.POINTER(HelmholtzDesc), C.POINTER(vp)], C.c_int),
        "plato_helmholtz_value": ([vp, vp, vp, vp], C.c_int),
        "plato_helmholtz_gradient_u": ([vp, vp], C.c_int),
        "plato_helmholtz_gradient_z": ([vp, vp], C.c_int),
        "plato_helmholtz_solution": ([vp, vp, vp, C.POINTER(SolveStats)], C.c_int),
        "plato_helmholtz_criterion_gradient": ([vp, vp, vp, C.POINTER(SolveStats)], C.c_int),
        "plato_app_create": ([C.c_char_p, C.c_char_p, C.c_char_p, C.POINTER(vp)], C.c_int),
        "plato_app_destroy": ([vp], C.c_int),
        "plato_app_last_error": ([vp], C.c_char_p),
        "plato_app_num_nodes": ([vp, i32p], C.c_int),
        "plato_app_compute": ([vp, C.c_char_p], C.c_int),
        "plato_app_import": ([vp, C.c_char_p, C.c_int32, C.c_char_p, vp, C.c_int64], C.c_int),
        "plato_app_export": ([vp, C.c_char_p, C.c_int32, vp, C.c_int64], C.c_int),
        "plato_app_validate": ([C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_int64], C.c_int),
        "plato_deck_to_text": ([C.c_char_p, C.c_char_p, C.c_int64, C.POINTER(C.c_int64)], C.c_int),
        "plato_coarse_operator": ([vp, vp, i32p, vp, vp], C.c_int),
        "plato_mesh_file_open": ([C.c_char_p, C.POINTER(vp)], C.c_int),
        "plato_mesh_file_last_error": ([], C.c_char_p),
        "plato_mesh_file_close": ([vp], C.c_int),
        "plato_mesh_file_info": ([vp, i32p, i32p, i32p, i32p], C.c_int),
        "plato_mesh_file_mesh": ([vp, vp, vp], C.c_int),
        "plato_mesh_file_node_set": ([vp, C.c_int32, C.c_char_p, C.c_int64, vp, i32p], C.c_int),
        "plato_mesh_file_side_set": ([vp, C.c_int32, C.c_char_p, C.c_int64, vp, vp, i32p], C.c_int),
        "plato_box_mesh_sizes": ([C.c_int32] * 3 + [i32p, i32p], C.c_int),
        "plato_box_mesh_tet4": ([C.c_int32] * 3 + [C.c_double] * 3 + [vp, vp], C.c_int),
        "plato_box_nodeset": ([C.c_int32] * 4 + [vp, i32p], C.c_int),
        "plato_box_sideset": ([C.c_int32] * 4 + [vp, vp, i32p], C.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return lib


lib = _load()


def check(rc: int, handle=None) -> int:
    if rc != OK:
        msg = lib.plato_last_error(handle)
        raise PlatoError(rc, msg.decode() if msg else "")
    return rc
