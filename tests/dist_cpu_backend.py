"""Host (numpy + oracle) local operations of one slab for the CPU tests of the distributed
driver: the same interface as platoanalyze_b200.distributed.GpuBackend, test infrastructure
only (the oracle is the checker; the product's per-rank operations run on the GPU)."""
from __future__ import annotations

import numpy as np

from oracle import Oracle


class CpuBackend:
    def __init__(self, part, E=1.0, nu=0.3, p=3.0, rho_min=1e-9):
        if len(part.tractions) > 1:
            raise ValueError("the oracle takes one traction side set")
        tr = part.tractions[0] if part.tractions else None
        self.orc = Oracle(part.coords, part.connectivity, E, nu, p, rho_min,
                          (tr[0], tr[1]) if tr else None, tr[2] if tr else (0.0, 0.0, 0.0),
                          part.bc_dofs, part.bc_values)
        self.n = 3 * part.num_nodes
        rm, cols = self.orc.graph()
        blk = np.array([rm[a] + np.searchsorted(cols[rm[a]:rm[a + 1]], a) for a in range(part.num_nodes)], np.int64)
        self.diag_idx = (9 * blk[:, None] + np.array([0, 4, 8])[None, :]).reshape(-1)
        self.bc = part.bc_dofs.astype(np.int64)
        self.bc_scale = 1.0 / part.bc_multiplicity.astype(np.float64)
        self.K = None

    def vec(self, a=None):
        return np.zeros(self.n) if a is None else np.array(a, dtype=np.float64)

    def host(self, v):
        return np.asarray(v)

    def index(self, a):
        return np.asarray(a, dtype=np.int64)

    def take(self, v, idx):
        return v[idx].copy()

    def add_at(self, v, idx, vals):
        np.add.at(v, idx, vals)

    def put(self, v, idx, vals):
        v[idx] = vals

    def dot3(self, w, a, b):
        return float(np.sum(w * a * b))

    def scalars(self, vals):
        return np.array([float(v) for v in vals], dtype=np.float64)

    def assemble(self, z):
        zero = np.zeros(self.n)
        self.K = self.orc.vf_gradient_u(zero, z)
        b = -self.orc.vf_value(zero, z)
        self.orc.apply_constraints(self.K, b, 1.0)
        if self.bc.size:
            self.K[self.diag_idx[self.bc]] = self.bc_scale
        return b

    def diagonal(self):
        return self.K[self.diag_idx].copy()

    def matvec(self, x):
        return self.orc.matvec_plus(3, 3, self.K, x, np.zeros(self.n))

    def energy(self, z, u):
        return self.orc.sf_value(u, z)

    def dcdz(self, z, u):
        return self.orc.criterion_gradient(z, u, self_adjoint=True)

    def close(self):
        pass
