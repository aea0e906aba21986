"""The x-slab decomposition of one problem (platoanalyze_b200/distributed.py) on the CPU:
partition invariants, and the distributed Jacobi-PCG, compliance and dC/dz against the
single-rank oracle -- over 2 gloo processes (torch.distributed, the code path NCCL runs on
GPUs) and over 3 ranks emulated as threads (a middle slab with two interfaces)."""
import os
import socket

import numpy as np
import pytest

import workload as ow
from dist_cpu_backend import CpuBackend
from helpers import rel_l2
from platoanalyze_b200.distributed import SlabSolver, gather_global, run_threads, slab_partition, thread_comms

SIZE = (12, 4, 4)
TOL = 1e-12  # the FP64 residual floor of this small problem is about 1e-13


def problem():
    orc = ow.cantilever_oracle(*SIZE)
    z = ow.splitmix_uniform(orc.N, 0x5EED0003)
    return orc, z


def parts_of(orc, world):
    return slab_partition(orc.coords, orc.conn, world, orc.bc_dofs, orc.bc_values,
                          [(orc.fc, orc.fl, (0.0, -1.0, 0.0))])


def reference(orc, z):
    u, _, st = orc.solution_refined(z, tol=1e-14)
    return u, orc.sf_value(u, z), orc.criterion_gradient(z, u, self_adjoint=True)


@pytest.mark.parametrize("world", [2, 3, 5])
def test_partition_invariants(world):
    orc, _ = problem()
    parts = parts_of(orc, world)
    cells = np.concatenate([p.cells for p in parts])
    assert np.array_equal(np.sort(cells), np.arange(orc.C))          # every cell exactly once
    owned = np.concatenate([p.nodes[p.owned] for p in parts])
    assert np.array_equal(np.sort(owned), np.arange(orc.N))         # every node owned once
    for p in parts:
        assert np.array_equal(p.nodes[p.connectivity], orc.conn[p.cells])
        for q, idx in p.neighbours.items():                         # symmetric interface lists
            other = parts[q]
            assert np.array_equal(p.nodes[idx], other.nodes[other.neighbours[p.rank]])
    assert sum(p.bc_dofs.size for p in parts) >= orc.bc_dofs.size
    faces = sum(t[0].size for p in parts for t in p.tractions)
    assert faces == orc.fc.size


def _gloo_rank(rank, world, port, outdir):
    import torch.distributed as dist

    from platoanalyze_b200.distributed import TorchComm

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        orc, z = problem()
        part = parts_of(orc, world)[rank]
        be = CpuBackend(part)
        solver = SlabSolver(part, be, TorchComm(), tol=TOL)
        zl = z[part.nodes]
        u, st = solver.solution(zl)
        f = solver.criterion_value(zl, u)
        g = solver.criterion_gradient(zl, u)
        np.savez(os.path.join(outdir, f"r{rank}.npz"), u=u, g=g, f=f, it=st["iterations"], rel=st["relative_residual"])
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_two_gloo_ranks_match_one(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    mp.start_processes(_gloo_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    orc, z = problem()
    parts = parts_of(orc, world)
    res = [np.load(tmp_path / f"r{r}.npz") for r in range(world)]
    assert all(float(r["rel"]) <= TOL for r in res)
    u = gather_global(parts, [r["u"] for r in res], orc.N, 3)
    g = gather_global(parts, [r["g"] for r in res], orc.N, 1)
    uo, fo, go = reference(orc, z)
    assert rel_l2(u, uo) <= 1e-11
    assert all(abs(float(r["f"]) - fo) <= 1e-11 * abs(fo) for r in res)
    assert rel_l2(g, go) <= 1e-11
    # interface copies agree (consistent vectors)
    for p, r in zip(parts, res):
        assert np.allclose(r["u"].reshape(-1, 3), u.reshape(-1, 3)[p.nodes], rtol=0, atol=1e-13 * np.abs(u).max())


def test_three_thread_ranks_match_one():
    world = 3
    orc, z = problem()
    parts = parts_of(orc, world)
    comms = thread_comms(world)

    def rank(p):
        part = parts[p]
        solver = SlabSolver(part, CpuBackend(part), comms[p], tol=TOL)
        zl = z[part.nodes]
        u, st = solver.solution(zl)
        return u, solver.criterion_value(zl, u), solver.criterion_gradient(zl, u), st

    out = run_threads(world, rank)
    assert all(o[3]["converged"] == 1 for o in out)
    assert len({o[3]["iterations"] for o in out}) == 1  # lockstep: the same iterations everywhere
    u = gather_global(parts, [o[0] for o in out], orc.N, 3)
    g = gather_global(parts, [o[2] for o in out], orc.N, 1)
    uo, fo, go = reference(orc, z)
    assert rel_l2(u, uo) <= 1e-11
    assert all(abs(o[1] - fo) <= 1e-11 * abs(fo) for o in out)
    assert rel_l2(g, go) <= 1e-11
