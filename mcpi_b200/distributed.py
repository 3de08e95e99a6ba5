"""Row-sharded Lanczos over several processes (one per GPU).

The configurations are split into contiguous row blocks, one per rank. Each
rank stores only its rows of every Krylov vector. Per Lanczos step:

* all-gather of the new Krylov vector (every rank needs the whole vector: an
  H.psi row gathers from anywhere in the space);
* local H.psi of the owned rows (`mcpi_apply_h_rows` on the GPU);
* all-reduce of the partial dot products (alpha, the residual norm) and of
  the reorthogonalisation coefficients V^H r.

The recurrence is the reference's (groundStateLieb.c:217-344: full classical
Gram-Schmidt, breakdown when beta_i / max beta < 1e-15) and the final
tridiagonal is solved identically on every rank. Collectives go through
torch.distributed (NCCL on GPUs; the tests run the same driver on CPU with
gloo and an injected local operator).
"""
from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist

from . import tridiag_eig


def row_block(nc: int, world: int, rank: int):
    """Contiguous rows owned by `rank`: [r0, r1)."""
    base, extra = divmod(nc, world)
    r0 = rank * base + min(rank, extra)
    return r0, r0 + base + (1 if rank < extra else 0)


class ShardedLanczos:
    """local_apply(v_full) -> H v restricted to this rank's rows (a tensor of
    r1 - r0 entries on `device`). All vectors are complex128 tensors."""

    def __init__(self, nc: int, local_apply, device, group=None):
        self.nc = nc
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.r0, self.r1 = row_block(nc, self.world, self.rank)
        self.counts = [row_block(nc, self.world, r) for r in range(self.world)]
        self.local_apply = local_apply
        self.device = device

    # collectives ------------------------------------------------------------
    def _gather(self, shard):
        parts = [torch.empty(b - a, dtype=shard.dtype, device=shard.device) for a, b in self.counts]
        dist.all_gather(parts, shard.contiguous(), group=self.group)
        return torch.cat(parts)

    def _sum(self, t):
        t = t.clone()
        if t.is_complex():
            r = torch.view_as_real(t).contiguous()
            dist.all_reduce(r, group=self.group)
            return torch.view_as_complex(r)
        dist.all_reduce(t, group=self.group)
        return t

    def _dot(self, a, b):
        return self._sum(torch.vdot(a, b).reshape(1))[0]

    # Lanczos ----------------------------------------------------------------
    def lanczos(self, v0_shard, lm: int, tol: float = 1e-15):
        """Returns (iterations, alpha[lm] complex, beta[lm], Krylov shards [lm, r1-r0])."""
        V = torch.zeros((lm, self.r1 - self.r0), dtype=torch.complex128, device=self.device)
        V[0] = v0_shard
        alpha = np.zeros(lm, np.complex128)
        beta = np.zeros(lm)
        r = self.local_apply(self._gather(V[0]))
        a0 = self._dot(V[0], r)
        alpha[0] = complex(a0)
        r = r - a0 * V[0]
        maxb = 0.0
        for i in range(lm - 1):
            b = float(torch.sqrt(self._sum(torch.sum(r.real ** 2 + r.imag ** 2).reshape(1)))[0])
            beta[i] = b
            maxb = max(maxb, b)
            if maxb == 0.0 or not (b / maxb >= tol):     # breakdown (groundStateLieb.c:292)
                return i, alpha, beta, V
            V[i + 1] = r / b
            r = self.local_apply(self._gather(V[i + 1]))
            r = r - b * V[i]
            a = self._dot(V[i + 1], r)
            alpha[i + 1] = complex(a)
            r = r - a * V[i + 1]
            c = self._sum(torch.mv(V[: i + 2].conj(), r))       # <V_j, r>, j <= i+1
            r = r - torch.mv(V[: i + 2].transpose(0, 1), c)
        return lm, alpha, beta, V

    def ground(self, v0_shard, niter: int):
        """Lowest eigenpair (groundStateLieb.c:348-471): (E0, Ritz-vector shard, iterations)."""
        it, alpha, beta, V = self.lanczos(v0_shard, niter)
        n = max(it, 1)
        d, z = tridiag_eig(alpha[:n].real, beta[: max(n - 1, 1)])
        j = int(np.argmin(d))
        zz = torch.tensor(z[:, j], dtype=torch.complex128, device=self.device)
        return float(d[j]), torch.mv(V[:n].transpose(0, 1), zz), it
