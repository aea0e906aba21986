"""The x-slab decomposition with the product's per-rank operations on the GPU (C ABI):
2 and 3 ranks emulated as threads of one process on one GPU (host-side rendezvous only; no
kernel waits on another rank's kernel).  u, compliance and dC/dz must match the single-handle
GPU solve and the oracle; interface copies must agree."""
import numpy as np
import pytest

import workload as ow
from helpers import rel_l2
from platoanalyze_b200.distributed import GpuBackend, SlabSolver, gather_global, run_threads, slab_partition
from platoanalyze_b200.distributed import thread_comms

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("world,size", [(2, (16, 6, 6)), (3, (24, 6, 6))])
def test_thread_ranks_on_one_gpu_match_one_rank(world, size):
    import torch

    orc = ow.cantilever_oracle(*size)
    z = ow.splitmix_uniform(orc.N, 0x5EED0003)
    parts = slab_partition(orc.coords, orc.conn, world, orc.bc_dofs, orc.bc_values,
                           [(orc.fc, orc.fl, (0.0, -1.0, 0.0))])
    comms = thread_comms(world)

    def rank(p):
        torch.cuda.set_device(0)
        part = parts[p]
        be = GpuBackend(part)
        try:
            solver = SlabSolver(part, be, comms[p], tol=1e-12)
            zl = be.vec(z[part.nodes])
            u, st = solver.solution(zl)
            f = solver.criterion_value(zl, u)
            g = solver.criterion_gradient(zl, u)
            torch.cuda.synchronize()
            return be.host(u), f, be.host(g), st
        finally:
            be.close()

    out = run_threads(world, rank)
    assert all(o[3]["converged"] == 1 and o[3]["relative_residual"] <= 1e-12 for o in out), [o[3] for o in out]
    u = gather_global(parts, [o[0] for o in out], orc.N, 3)
    g = gather_global(parts, [o[2] for o in out], orc.N, 1)
    uo, _, _ = orc.solution_refined(z, tol=1e-14)
    fo = orc.sf_value(uo, z)
    go = orc.criterion_gradient(z, uo, self_adjoint=True)
    assert rel_l2(u, uo) <= 1e-10, rel_l2(u, uo)
    assert all(abs(o[1] - fo) <= 1e-10 * abs(fo) for o in out)
    assert rel_l2(g, go) <= 1e-10
    for p, o in zip(parts, out):  # consistent interface copies
        assert np.abs(o[0].reshape(-1, 3) - u.reshape(-1, 3)[p.nodes]).max() <= 1e-12 * np.abs(u).max()
