"""The allocation-free compliance entry point, plato_sf_value_noalloc.

It exists for callers that cannot allocate device memory when they need the criterion
(their device memory is owned by another allocator's pool, or they must not risk the
implicit synchronisation of cudaMalloc / cudaFree).  It takes caller-owned device arrays
and keeps its reduction scratch in a static device array, so the checks are: the value
matches the handle-based plato_sf_value within the suite's 1e-11 relative tolerance, on two
calls in a row (the shared scratch must not carry state from one call into the next), on a
small mesh (47 blocks) and on one of 768,000 cells (3,000 blocks, so the last-block sum runs
over thousands of partials); meshes beyond the scratch limit are rejected with a clear
error; a connectivity id outside [0, num_nodes) is rejected with PLATO_BAD_INPUT and a NaN
value (the kernel skips the cell instead of reading out of bounds); a NaN control gives
PLATO_NONFINITE; and a good call after those failures is exact again.  This file is collected
last so that a run stopping at the first failure has already run every other test; it
passes alone in a fresh process as well.
"""
import ctypes as C

import numpy as np
import pytest

from platoanalyze_b200 import capi
from platoanalyze_b200.problem import EllipticProblem
from platoanalyze_b200.workloads import cantilever, splitmix_uniform

pytestmark = pytest.mark.gpu
TOL = 1e-11


def call_noalloc(prob, spec, conn_d, coords_d, u_d, z_d, out_d, stream):
    mat = capi.Material(spec.youngs_modulus, spec.poissons_ratio)
    pen = capi.Penalty(spec.penalty_exponent, spec.penalty_minimum)
    vp = C.c_void_p
    return capi.lib.plato_sf_value_noalloc(prob.num_nodes, conn_d.shape[0], vp(conn_d.data_ptr()),
                                           vp(coords_d.data_ptr()), vp(u_d.data_ptr()), vp(z_d.data_ptr()),
                                           C.byref(mat), C.byref(pen), vp(out_d.data_ptr()), vp(stream.cuda_stream))


def _device_inputs(spec):
    import torch

    conn_d = torch.from_numpy(np.ascontiguousarray(spec.connectivity, dtype=np.int32)).cuda()
    coords_d = torch.from_numpy(np.ascontiguousarray(spec.coords, dtype=np.float64)).cuda()
    return conn_d, coords_d


@pytest.mark.parametrize("size", [(20, 10, 10), (80, 40, 40)])
def test_noalloc_compliance_matches_handle_entry_point(size):
    import torch

    spec = cantilever(*size)
    prob = EllipticProblem(spec)
    z = splitmix_uniform(prob.num_nodes, 0x5EED0003)
    u1 = np.sin(np.arange(prob.num_dofs) * 0.013) * 1e-2
    u2 = np.cos(np.arange(prob.num_dofs) * 0.029) * 3e-3
    zd, u1d, u2d = prob.to_dev(z), prob.to_dev(u1), prob.to_dev(u2)
    ref1, ref2 = prob.sf_value(u1d, zd), prob.sf_value(u2d, zd)

    conn_d, coords_d = _device_inputs(spec)
    out = torch.full((1,), np.nan, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    # two calls in a row on different states: the second must not see the first's scratch
    for ud, ref in ((u1d, ref1), (u2d, ref2), (u1d, ref1)):
        out.fill_(np.nan)
        rc = call_noalloc(prob, spec, conn_d, coords_d, ud, zd, out, stream)
        assert rc == capi.OK, capi.lib.plato_last_error(None)
        torch.cuda.synchronize()
        v = float(out.item())
        assert abs(v - ref) <= TOL * abs(ref), (v, ref)
    prob.close()


def test_noalloc_rejects_out_of_range_ids_and_reports_nonfinite():
    import torch

    spec = cantilever(20, 10, 10)
    prob = EllipticProblem(spec)
    z = splitmix_uniform(prob.num_nodes, 0x5EED0003)
    u = np.sin(np.arange(prob.num_dofs) * 0.013) * 1e-2
    zd, ud = prob.to_dev(z), prob.to_dev(u)
    ref = prob.sf_value(ud, zd)
    conn_d, coords_d = _device_inputs(spec)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    for bad_id in (prob.num_nodes, -1, 2**31 - 1):
        bad = conn_d.clone()
        bad[len(bad) // 2, 2] = bad_id
        rc = call_noalloc(prob, spec, bad, coords_d, ud, zd, out, stream)
        assert rc == capi.BAD_INPUT, rc
        assert b"node id outside" in capi.lib.plato_last_error(None)
        assert np.isnan(float(out.item()))
    z_nan = z.copy()
    z_nan[7] = np.nan
    rc = call_noalloc(prob, spec, conn_d, coords_d, ud, prob.to_dev(z_nan), out, stream)
    assert rc == capi.NONFINITE, rc
    # the counters start from zero again: a good call right after the failures is exact
    rc = call_noalloc(prob, spec, conn_d, coords_d, ud, zd, out, stream)
    assert rc == capi.OK, capi.lib.plato_last_error(None)
    assert abs(float(out.item()) - ref) <= TOL * abs(ref)
    # non-finite material parameters are refused before any launch
    vp = C.c_void_p
    for mat, pen in ((capi.Material(np.inf, 0.3), capi.Penalty(3.0, 1e-9)),
                     (capi.Material(1.0, 0.3), capi.Penalty(3.0, np.nan))):
        rc = capi.lib.plato_sf_value_noalloc(prob.num_nodes, conn_d.shape[0], vp(conn_d.data_ptr()),
                                             vp(coords_d.data_ptr()), vp(ud.data_ptr()), vp(zd.data_ptr()),
                                             C.byref(mat), C.byref(pen), vp(out.data_ptr()), vp(stream.cuda_stream))
        assert rc == capi.BAD_INPUT
    prob.close()


def test_noalloc_rejects_sizes_beyond_the_scratch():
    import torch

    d = torch.zeros(16, dtype=torch.float64, device="cuda")
    mat, pen = capi.Material(1.0, 0.3), capi.Penalty(3.0, 1e-9)
    vp = C.c_void_p(d.data_ptr())
    rc = capi.lib.plato_sf_value_noalloc(4, 16_777_217, vp, vp, vp, vp, C.byref(mat), C.byref(pen), vp, None)
    assert rc == capi.BAD_INPUT
    assert b"16777216" in capi.lib.plato_last_error(None)
