"""The MPMD application over the C ABI: `AnalyzeApp` mirrors the reference's MPMD_App
(src/Analyze_App.hpp) as a PlatoEngine driver sees it - construct from an input deck and an
operations file, import shared data, compute named operations, export shared data.

    app = AnalyzeApp(deck_xml, operations_xml)
    app.import_field("Topology", z)
    app.compute("Compute Objective")
    f = app.export_value("Objective Value")
    g = app.export_field("Objective Gradient")

Decks and operation files are XML text or file names (relative to `base_dir`).  Shared data
crosses as host numpy arrays; the problem lives on the GPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi
from .capi import lib


def _b(s):
    return None if s is None else (s.encode() if isinstance(s, str) else s)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def validate(input_config: str, operations: str, base_dir: str | None = None) -> None:
    """Host-only check of a deck and operations file (no GPU): raises PlatoError on the first
    problem found."""
    buf = C.create_string_buffer(4096)
    rc = lib.plato_app_validate(_b(input_config), _b(operations), _b(base_dir), buf, len(buf))
    if rc != capi.OK:
        raise capi.PlatoError(rc, buf.value.decode())


def deck_text(input_config: str) -> str:
    """The deck as parsed: one 'name (type) = value' line per parameter, sublists indented."""
    need = C.c_int64(0)
    rc = lib.plato_deck_to_text(_b(input_config), None, 0, C.byref(need))
    if rc != capi.OK:
        raise capi.PlatoError(rc, (lib.plato_app_last_error(None) or b"").decode())
    buf = C.create_string_buffer(need.value)
    lib.plato_deck_to_text(_b(input_config), buf, need.value, C.byref(need))
    return buf.value.decode()


class AnalyzeApp:
    def __init__(self, input_config: str, operations: str, base_dir: str | None = None):
        h = C.c_void_p()
        rc = lib.plato_app_create(_b(input_config), _b(operations), _b(base_dir), C.byref(h))
        if rc != capi.OK:
            raise capi.PlatoError(rc, (lib.plato_app_last_error(None) or b"").decode())
        self.h = h
        n = C.c_int32()
        self._check(lib.plato_app_num_nodes(h, C.byref(n)))
        self.num_nodes = n.value

    def _check(self, rc):
        if rc != capi.OK:
            raise capi.PlatoError(rc, (lib.plato_app_last_error(self.h) or b"").decode())

    def close(self):
        if getattr(self, "h", None):
            lib.plato_app_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def compute(self, operation: str) -> None:
        self._check(lib.plato_app_compute(self.h, _b(operation)))

    def import_field(self, name: str, values) -> None:
        a = np.ascontiguousarray(values, dtype=np.float64)
        self._check(lib.plato_app_import(self.h, _b(name), capi.LAYOUT_SCALAR_FIELD, None, _ptr(a), a.size))

    def import_parameter(self, operation: str, name: str, value: float) -> None:
        a = np.array([value], dtype=np.float64)
        self._check(lib.plato_app_import(self.h, _b(name), capi.LAYOUT_SCALAR_PARAMETER, _b(operation), _ptr(a), 1))

    def export_field(self, name: str) -> np.ndarray:
        out = np.empty(self.num_nodes, dtype=np.float64)
        self._check(lib.plato_app_export(self.h, _b(name), capi.LAYOUT_SCALAR_FIELD, _ptr(out), out.size))
        return out

    def export_value(self, name: str) -> float:
        out = np.empty(1, dtype=np.float64)
        self._check(lib.plato_app_export(self.h, _b(name), capi.LAYOUT_SCALAR_VALUE, _ptr(out), 1))
        return float(out[0])
