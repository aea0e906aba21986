"""One problem split across GPUs: x-slab domain decomposition of the elliptic solve.

The reference's elliptic path runs one rank over a single Epetra block map of all nodes
(src/alg/EpetraLinearSolver.cpp:12-22) with MPI plumbing in src/alg/ParallelComm.cpp:49-94.
Here a problem too large for one GPU is split into P slabs of cells along x, one slab per
process (one GPU each):

* every rank owns the cells of its slab and holds every node those cells touch (local
  numbering); nodes on a slab interface are held by the ranks on both sides and owned by the
  lowest of them;
* each rank assembles K_p(z) from its own cells only, so the global operator is the sum of
  the ranks' operators: one operator apply is the local SpMV followed by one exchange of the
  interface nodes' partial sums with the neighbouring slabs (about 81 x 81 x 3 doubles per
  interface on the 160x80x80 bench mesh);
* Krylov vectors are kept consistent (equal on every copy of a shared node), dot products
  sum each dof once (on its owner) and are completed by an all-reduce;
* the compliance is the all-reduced sum of the slabs' cell sums, and dC/dz the exchanged
  sum of the slabs' nodal sums.

The solver is the reference's algorithm, FP64 Jacobi-PCG, with the same stop test as the
single-GPU solve (the recomputed FP64 residual must meet the tolerance).

The driver is written once against two small interfaces: a Backend (the per-rank local
operations; GpuBackend runs them through the library's C ABI on the rank's GPU) and a Comm
(the collectives; TorchComm uses torch.distributed -- NCCL between GPUs, gloo on CPU --
and ThreadComm runs several ranks as threads of one process).  Multi-GPU runs were not
possible on the hardware available to this build: the algorithm is checked by CPU ranks
over gloo and by ranks emulated as threads on one GPU.
"""
from __future__ import annotations

import threading
from dataclasses import dataclass, field

import numpy as np


# ---- partition ------------------------------------------------------------------------------

@dataclass
class RankPart:
    """One slab: global ids of its cells and nodes, local connectivity, the interface lists."""
    rank: int
    world: int
    cells: np.ndarray                 # global cell ids (ascending)
    nodes: np.ndarray                 # global node ids (ascending); local node k = nodes[k]
    connectivity: np.ndarray          # (cells, 4) local node ids
    coords: np.ndarray                # (nodes, 3)
    owned: np.ndarray                 # bool per local node: this rank owns it
    neighbours: dict = field(default_factory=dict)   # rank q -> local node ids shared with q (ascending global)
    bc_dofs: np.ndarray = None        # local constrained dofs
    bc_values: np.ndarray = None
    bc_multiplicity: np.ndarray = None  # ranks holding the node of each constrained dof
    tractions: list = field(default_factory=list)  # [(local face cells, local ordinals, vector)]

    @property
    def num_nodes(self) -> int:
        return self.nodes.size


def slab_partition(coords, connectivity, world: int, bc_dofs=None, bc_values=None, tractions=()):
    """Splits the cells into `world` slabs of (nearly) equal cell count by cell-centroid x
    (ties broken by cell id) and builds each slab's local mesh, ownership and interface lists.
    tractions: [(face_cells, face_local_nodes, vector)] in global cell ids."""
    coords = np.asarray(coords, dtype=np.float64)
    conn = np.asarray(connectivity, dtype=np.int64)
    C, N = conn.shape[0], coords.shape[0]
    if world < 1 or world > C:
        raise ValueError(f"cannot split {C} cells into {world} slabs")
    cx = coords[conn, 0].mean(axis=1)
    order = np.lexsort((np.arange(C), cx))
    cell_rank = np.empty(C, np.int64)
    bounds = np.linspace(0, C, world + 1).round().astype(np.int64)
    for p in range(world):
        cell_rank[order[bounds[p]:bounds[p + 1]]] = p
    # ranks holding each node; the lowest owns it
    node_mask = np.zeros((world, N), dtype=bool)
    for p in range(world):
        node_mask[p, np.unique(conn[cell_rank == p])] = True
    owner = np.argmax(node_mask, axis=0)  # first (lowest) holder
    multiplicity = node_mask.sum(axis=0)
    bc_dofs = np.zeros(0, np.int64) if bc_dofs is None else np.asarray(bc_dofs, np.int64)
    bc_values = np.zeros(bc_dofs.size) if bc_values is None else np.asarray(bc_values, np.float64)
    parts = []
    for p in range(world):
        cells = np.nonzero(cell_rank == p)[0]
        nodes = np.nonzero(node_mask[p])[0]
        local = np.full(N, -1, np.int64)
        local[nodes] = np.arange(nodes.size)
        part = RankPart(p, world, cells.astype(np.int32), nodes.astype(np.int32),
                        local[conn[cells]].astype(np.int32), coords[nodes], owner[nodes] == p)
        for q in range(world):
            if q != p:
                shared = np.nonzero(node_mask[p] & node_mask[q])[0]
                if shared.size:
                    part.neighbours[q] = local[shared].astype(np.int64)
        bn = bc_dofs // 3
        keep = node_mask[p, bn]
        part.bc_dofs = (3 * local[bn[keep]] + bc_dofs[keep] % 3).astype(np.int32)
        part.bc_values = bc_values[keep]
        part.bc_multiplicity = multiplicity[bn[keep]].astype(np.int32)
        cell_local = np.full(C, -1, np.int64)
        cell_local[cells] = np.arange(cells.size)
        for fc, fl, vec in tractions:
            fc = np.asarray(fc, np.int64)
            sel = cell_rank[fc] == p
            if sel.any():
                part.tractions.append((cell_local[fc[sel]].astype(np.int32),
                                       np.asarray(fl, np.int32)[sel], tuple(vec)))
        parts.append(part)
    return parts


# ---- collectives ----------------------------------------------------------------------------

def _as_torch(a):
    import torch

    return torch.from_numpy(a) if isinstance(a, np.ndarray) else a


class TorchComm:
    """Collectives over torch.distributed, one rank per process (NCCL between GPUs, gloo for
    host arrays).  Arrays are torch tensors or numpy arrays (shared with torch, in place)."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    def allreduce(self, a):
        self.dist.all_reduce(_as_torch(a), group=self.group)
        return a

    def exchange(self, sends: dict) -> dict:
        """sends: {q: array}; returns {q: array of the same shape received from q}.  Pairs
        post their send and receive in rank order, the same on both sides."""
        recvs = {q: (np.empty_like(a) if isinstance(a, np.ndarray) else a.new_empty(a.shape)) for q, a in sends.items()}
        reqs = []
        for q in sorted(sends):
            s_t, r_t = _as_torch(sends[q]), _as_torch(recvs[q])
            if q < self.rank:
                reqs.append(self.dist.irecv(r_t, src=q, group=self.group))
                reqs.append(self.dist.isend(s_t, dst=q, group=self.group))
            else:
                reqs.append(self.dist.isend(s_t, dst=q, group=self.group))
                reqs.append(self.dist.irecv(r_t, src=q, group=self.group))
        for r in reqs:
            r.wait()
        return recvs


class ThreadComm:
    """The same collectives for ranks that run as threads of one process: a host-side
    rendezvous (a barrier with a timeout), so no kernel of one rank ever waits on a kernel of
    another rank."""

    def __init__(self, world: int, timeout: float = 300.0):
        self.world = world
        self.barrier = threading.Barrier(world, timeout=timeout)
        self.slots = [None] * world
        self.mail = {}

    def allreduce(self, a, rank: int):
        self.slots[rank] = a.clone() if hasattr(a, "clone") else a.copy()
        self.barrier.wait()
        total = self.slots[0].clone() if hasattr(a, "clone") else self.slots[0].copy()
        for q in range(1, self.world):
            total += self.slots[q]
        self.barrier.wait()
        a[...] = total
        return a

    def exchange(self, rank: int, sends: dict) -> dict:
        for q, a in sends.items():
            self.mail[(rank, q)] = a.clone() if hasattr(a, "clone") else a.copy()
        self.barrier.wait()
        recvs = {q: self.mail.pop((q, rank)) for q in sends}
        self.barrier.wait()
        return recvs


class RankComm:
    """One rank's handle on a ThreadComm, with TorchComm's call signature."""

    def __init__(self, comm: ThreadComm, rank: int):
        self.comm, self.rank, self.world = comm, rank, comm.world

    def allreduce(self, a):
        return self.comm.allreduce(a, self.rank)

    def exchange(self, sends: dict) -> dict:
        return self.comm.exchange(self.rank, sends)


def thread_comms(world: int, timeout: float = 300.0) -> list:
    c = ThreadComm(world, timeout)
    return [RankComm(c, p) for p in range(world)]


def run_threads(world: int, fn):
    """Runs fn(rank) for every rank in its own thread; returns the results in rank order and
    re-raises the first failure."""
    out, errs = [None] * world, []

    def body(p):
        try:
            out[p] = fn(p)
        except BaseException as e:  # noqa: BLE001 -- reported below
            errs.append(e)

    ts = [threading.Thread(target=body, args=(p,)) for p in range(world)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    if errs:
        raise errs[0]
    return out


# ---- local operations on the rank's GPU (C ABI) -----------------------------------------------

class GpuBackend:
    """A rank's local operations on its slab through the library: element assembly, the
    symmetric Dirichlet elimination, the block-CRS matvec (MatrixTimesVectorPlusVector), the
    criterion and its nodal control derivative on the slab's cells.  Vectors are torch
    tensors on the rank's device."""

    def __init__(self, part: RankPart, E=1.0, nu=0.3, p=3.0, rho_min=1e-9):
        import torch

        from .problem import EllipticProblem, ProblemSpec

        self.torch = torch
        spec = ProblemSpec(part.coords, part.connectivity, E, nu, p, rho_min, list(part.tractions),
                           part.bc_dofs.astype(np.int32), part.bc_values)
        self.prob = EllipticProblem(spec)
        self.n = 3 * part.num_nodes
        rm, cols = self.prob.pattern()
        rm_h, cols_h = rm.cpu().numpy(), cols.cpu().numpy()
        diag_blk = np.array([rm_h[a] + np.searchsorted(cols_h[rm_h[a]:rm_h[a + 1]], a) for a in range(part.num_nodes)],
                            dtype=np.int64)
        self.diag_idx = torch.from_numpy((9 * diag_blk[:, None] + np.array([0, 4, 8])[None, :]).reshape(-1)).cuda()
        self.bc_diag_idx = self.diag_idx[torch.from_numpy(part.bc_dofs.astype(np.int64)).cuda()] if part.bc_dofs.size \
            else None
        self.bc_scale = torch.from_numpy(1.0 / part.bc_multiplicity.astype(np.float64)).cuda() \
            if part.bc_dofs.size else None
        self.K = None

    def vec(self, a=None):
        if a is None:
            return self.torch.zeros(self.n, dtype=self.torch.float64, device="cuda")
        return self.torch.as_tensor(np.ascontiguousarray(a), dtype=self.torch.float64).cuda()

    def host(self, v):
        return v.detach().cpu().numpy()

    def index(self, a):
        return self.torch.as_tensor(np.ascontiguousarray(a, dtype=np.int64)).cuda()

    def take(self, v, idx):
        return v[idx].contiguous()

    def add_at(self, v, idx, vals):
        v.index_add_(0, idx, vals)

    def put(self, v, idx, vals):
        v[idx] = vals

    def dot3(self, w, a, b):
        return (w * a * b).sum()

    def scalars(self, vals):
        return self.torch.stack([self.torch.as_tensor(v, dtype=self.torch.float64, device="cuda").reshape(())
                                 for v in vals])

    def assemble(self, z):
        """Local K_p(z) with the constraints applied and the partial right-hand side (the
        slab's load, lifted by its constrained columns).  A constrained dof shared by m slabs
        gets the diagonal 1/m on each, so the summed operator keeps its unit diagonal."""
        zero = self.vec()
        self.K = self.prob.vf_gradient_u(zero, z)
        b = -self.prob.vf_value(zero, z)
        self.prob.apply_constraints(self.K, b, 1.0)
        if self.bc_diag_idx is not None:
            self.K[self.bc_diag_idx] = self.bc_scale
        return b

    def diagonal(self):
        return self.K[self.diag_idx].clone()

    def matvec(self, x):
        return self.prob.matvec_plus(3, 3, self.K, x, self.vec())

    def energy(self, z, u) -> float:
        return self.prob.sf_value(u, z)

    def dcdz(self, z, u):
        g, _ = self.prob.criterion_gradient(z, u)
        return g

    def close(self):
        self.prob.close()


# ---- the distributed solve ---------------------------------------------------------------------

class SlabSolver:
    """The rank-local half of the distributed solve (SPMD: every rank makes the same calls in
    the same order, collectives included)."""

    def __init__(self, part: RankPart, backend, comm, tol=1e-10, max_iterations=200000, max_restarts=8):
        self.part, self.be, self.comm = part, backend, comm
        self.tol, self.max_it, self.max_restarts = tol, max_iterations, max_restarts
        self.owned3 = backend.vec(np.repeat(part.owned, 3).astype(np.float64))
        self.nbr3 = {q: backend.index((3 * idx[:, None] + np.arange(3)[None, :]).reshape(-1))
                     for q, idx in part.neighbours.items()}
        self.nbr1 = {q: backend.index(idx) for q, idx in part.neighbours.items()}
        self.bc = backend.index(part.bc_dofs.astype(np.int64))
        self.bc_values = backend.vec(part.bc_values)

    def exchange_add(self, v, per_node: int = 3):
        """Completes partial sums on interface nodes: adds the neighbours' partials (one
        exchange with each neighbouring slab)."""
        idx = self.nbr3 if per_node == 3 else self.nbr1
        if not idx:
            return v
        recvs = self.comm.exchange({q: self.be.take(v, i) for q, i in idx.items()})
        for q in sorted(idx):
            self.be.add_at(v, idx[q], recvs[q])
        return v

    def dots(self, pairs):
        """Dot products over the owned dofs of several vector pairs, in one all-reduce."""
        t = self.be.scalars([self.be.dot3(self.owned3, a, b) for a, b in pairs])
        self.comm.allreduce(t)
        return [float(v) for v in self.be.host(t)]

    def apply(self, x):
        return self.exchange_add(self.be.matvec(x))

    def solution(self, z):
        """Problem::solution on the slabs (src/elliptic/Problem.hpp:237-292, one Newton step
        from u = 0): local u on this rank's nodes, consistent across interfaces, and stats."""
        be = self.be
        b = be.assemble(z)
        if self.part.bc_dofs.size:  # constrained entries are set after the sum, not summed
            be.put(b, self.bc, 0.0 * self.bc_values)
        b = self.exchange_add(b)
        if self.part.bc_dofs.size:
            be.put(b, self.bc, self.bc_values)
        dinv = 1.0 / self.exchange_add(be.diagonal())
        x = be.vec()
        (bb,) = self.dots([(b, b)])
        stats = {"iterations": 0, "relative_residual": 0.0, "converged": 1, "restarts": 0}
        if bb == 0.0:
            return x, stats
        it, restarts = 0, 0
        while True:
            r = b - self.apply(x)
            zv = dinv * r
            p = zv * 1.0
            rz, rr = self.dots([(r, zv), (r, r)])
            true_rel = (rr / bb) ** 0.5
            # converged only on the recomputed FP64 residual; the recurrence decides when to
            # recompute it (restart from x with a fresh direction)
            if true_rel <= self.tol or it >= self.max_it or restarts > self.max_restarts:
                break
            while it < self.max_it and (rr / bb) ** 0.5 > self.tol:
                q = self.apply(p)
                (pq,) = self.dots([(p, q)])
                if not pq > 0.0:
                    break
                alpha = rz / pq
                x += alpha * p
                r -= alpha * q
                zv = dinv * r
                rz_new, rr = self.dots([(r, zv), (r, r)])
                p = zv + (rz_new / rz) * p
                rz = rz_new
                it += 1
            restarts += 1
        stats.update(iterations=it, relative_residual=true_rel, converged=int(true_rel <= self.tol),
                     restarts=max(0, restarts - 1))
        return x, stats

    def criterion_value(self, z, u) -> float:
        """Compliance (internal elastic energy): the all-reduced sum over the slabs' cells."""
        t = self.be.scalars([self.be.energy(z, u)])
        self.comm.allreduce(t)
        return float(self.be.host(t)[0])

    def criterion_gradient(self, z, u):
        """Self-adjoint dC/dz (Problem::criterionGradient, src/elliptic/Problem.hpp:423-448):
        the slab's nodal sums, completed across interfaces."""
        return self.exchange_add(self.be.dcdz(z, u), per_node=1)


def gather_global(parts, locals_, num_nodes: int, dofs_per_node: int):
    """Assembles per-rank local vectors (host arrays) into one global vector from the owners."""
    out = np.zeros(dofs_per_node * num_nodes)
    for part, v in zip(parts, locals_):
        nodes = part.nodes[part.owned].astype(np.int64)
        loc = np.nonzero(part.owned)[0]
        for d in range(dofs_per_node):
            out[dofs_per_node * nodes + d] = np.asarray(v)[dofs_per_node * loc + d]
    return out
