"""Row-sharded Lanczos over several processes (one per GPU).

The configurations are split into contiguous row blocks, one per rank. Each
rank stores only its rows of every Krylov vector. Per Lanczos step:

* all-gather of the new Krylov vector (every rank needs the whole vector: an
  H.psi row gathers from anywhere in the space);
* local H.psi of the owned rows (`mcpi_apply_h_rows` on the GPU);
* all-reduce of this rank's alpha dot, of its reorthogonalisation
  coefficients V^H r and of its residual norm^2.

The recurrence is the reference's (groundStateLieb.c:217-344: full classical
Gram-Schmidt, breakdown when beta_i / max beta < 1e-15) and the final
tridiagonal is solved identically on every rank. On a GPU the per-shard math
runs in the library's own Lanczos kernels through the row-shard primitives of
the C ABI (`mcpi_shard_*`): alpha, beta, the coefficients and the breakdown
flag stay in device memory, so a solve enqueues its whole launch and
collective sequence without reading anything back until the end (after a
breakdown every kernel returns at entry while the ranks keep issuing the same
collectives). Collectives go through torch.distributed (NCCL on GPUs); the
tests run the same driver on CPU with gloo, `TorchShardOps` standing in for
the kernels and an injected local operator.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np
import torch
import torch.distributed as dist

from . import MCPIError, lib, tridiag_eig

_vp = ct.c_void_p


def row_block(nc: int, world: int, rank: int):
    """Contiguous rows owned by `rank`: [r0, r1)."""
    base, extra = divmod(nc, world)
    r0 = rank * base + min(rank, extra)
    return r0, r0 + base + (1 if rank < extra else 0)


def _p(t):
    return None if t is None else _vp(t.data_ptr())


class DeviceShardOps:
    """The row-shard primitives on the GPU (mcpi_shard_* of the C ABI), on the
    current torch stream. Arguments are device tensors; scalars are 1-element
    tensors that stay on the device."""

    def __init__(self, n: int, lm: int, device):
        L = lib()
        self.L = L
        L.mcpi_shard_scratch_elems.restype = ct.c_size_t
        L.mcpi_shard_scratch_elems.argtypes = [ct.c_int64, ct.c_int]
        for name, args in (("mcpi_shard_scale", [ct.c_int64, _vp, _vp, _vp, _vp, _vp]),
                           ("mcpi_shard_axpy_dot", [ct.c_int64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
                           ("mcpi_shard_multidot", [ct.c_int64, _vp, ct.c_int, _vp, _vp, _vp, _vp, _vp, _vp,
                                                    _vp]),
                           ("mcpi_shard_update", [ct.c_int64, _vp, ct.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                                  _vp]),
                           ("mcpi_shard_beta", [ct.c_int, ct.c_double, _vp, _vp, _vp, _vp, _vp, _vp]),
                           ("mcpi_shard_combine", [ct.c_int64, _vp, ct.c_int, _vp, _vp, _vp])):
            f = getattr(L, name)
            f.restype = ct.c_int
            f.argtypes = args
        self.scratch = torch.empty(max(int(L.mcpi_shard_scratch_elems(n, lm)), 1), dtype=torch.complex128,
                                   device=device)
        self.device = device

    def _st(self):
        return _vp(torch.cuda.current_stream(self.device).cuda_stream)

    def _ck(self, rc):
        if rc != 0:
            raise MCPIError(rc, lib().mcpi_last_error().decode())

    def scale(self, r, vnext, beta_i, done):
        self._ck(self.L.mcpi_shard_scale(r.numel(), _p(r), _p(vnext), _p(beta_i), _p(done), self._st()))

    def axpy_dot(self, vprev, vcur, r, beta_i, dot, done):
        self._ck(self.L.mcpi_shard_axpy_dot(r.numel(), _p(vprev), _p(vcur), _p(r), _p(beta_i), _p(self.scratch),
                                            _p(dot), _p(done), self._st()))

    def multidot(self, V, nvec, r, vcur, alpha, coef, done):
        self._ck(self.L.mcpi_shard_multidot(r.numel(), _p(V), nvec, _p(r), _p(vcur), _p(alpha),
                                            _p(self.scratch), _p(coef), _p(done), self._st()))

    def update(self, V, nvec, r, vcur, alpha, coef, norm2, done):
        self._ck(self.L.mcpi_shard_update(r.numel(), _p(V), nvec, _p(r), _p(vcur), _p(alpha), _p(coef),
                                          _p(self.scratch), _p(norm2), _p(done), self._st()))

    def beta(self, i, tol, norm2, beta, maxbeta, done, iters):
        self._ck(self.L.mcpi_shard_beta(i, tol, _p(norm2), _p(beta), _p(maxbeta), _p(done), _p(iters),
                                        self._st()))

    def combine(self, V, nvec, z, out):
        self._ck(self.L.mcpi_shard_combine(out.numel(), _p(V), nvec, _p(z), _p(out), self._st()))


class TorchShardOps:
    """The same primitives in plain torch (any device): the stand-in the CPU
    tests use for the kernels, with the same semantics and the same device
    scalars (the breakdown flag makes every later call a no-op)."""

    def __init__(self, n: int, lm: int, device):
        self.device = device

    def scale(self, r, vnext, beta_i, done):
        if not int(done[0]):
            vnext.copy_(r / beta_i[0])

    def axpy_dot(self, vprev, vcur, r, beta_i, dot, done):
        if int(done[0]):
            return
        if vprev is not None:
            r.sub_(beta_i[0] * vprev)
        dot[0] = torch.vdot(vcur, r)

    def multidot(self, V, nvec, r, vcur, alpha, coef, done):
        if not int(done[0]):
            coef[:nvec] = torch.mv(V[:nvec].conj(), r - alpha[0] * vcur)

    def update(self, V, nvec, r, vcur, alpha, coef, norm2, done):
        if int(done[0]):
            return
        x = r - alpha[0] * vcur
        if nvec:
            x = x - torch.mv(V[:nvec].transpose(0, 1), coef[:nvec])
        r.copy_(x)
        norm2[0] = torch.sum(r.real ** 2 + r.imag ** 2)

    def beta(self, i, tol, norm2, beta, maxbeta, done, iters):
        if int(done[0]):
            return
        b = float(torch.sqrt(norm2[0]))
        beta[i] = b
        maxbeta[0] = max(float(maxbeta[0]), b)
        if not (b / float(maxbeta[0]) >= tol):     # breakdown (groundStateLieb.c:292); 0/0 too
            done[0] = 1
            iters[0] = i

    def combine(self, V, nvec, z, out):
        out.copy_(torch.mv(V[:nvec].transpose(0, 1), z[:nvec].to(V.dtype)))


class ShardedLanczos:
    """local_apply(v_full) -> H v restricted to this rank's rows (a tensor of
    r1 - r0 entries on `device`). All vectors are complex128 tensors. ops:
    the per-shard primitives (default: the library's kernels on a CUDA device,
    plain torch elsewhere)."""

    def __init__(self, nc: int, local_apply, device, group=None, ops=None):
        self.nc = nc
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.r0, self.r1 = row_block(nc, self.world, self.rank)
        self.counts = [row_block(nc, self.world, r) for r in range(self.world)]
        self.maxb = max(b - a for a, b in self.counts)
        self.local_apply = local_apply
        self.device = torch.device(device)
        self.ops_cls = ops or (DeviceShardOps if self.device.type == "cuda" else TorchShardOps)

    # collectives ------------------------------------------------------------
    def _gather(self, shard, send, gbuf):
        """The whole vector from every rank's shard (equal-size all-gather of
        shards padded to the largest block)."""
        n = shard.numel()
        send[:n].copy_(shard)
        # complex as (re, im) pairs: every backend gathers float64
        dist.all_gather_into_tensor(torch.view_as_real(gbuf), torch.view_as_real(send), group=self.group)
        g = gbuf.view(self.world, self.maxb)
        if all(b - a == self.maxb for a, b in self.counts):
            return gbuf[: self.nc]
        return torch.cat([g[k, : b - a] for k, (a, b) in enumerate(self.counts)])

    def _sum(self, t):
        """In-place all-reduce of a device scalar or vector (complex as pairs)."""
        dist.all_reduce(torch.view_as_real(t) if t.is_complex() else t, group=self.group)

    # Lanczos ----------------------------------------------------------------
    def lanczos(self, v0_shard, lm: int, tol: float = 1e-15):
        """Returns (iterations, alpha[lm] complex, beta[lm], Krylov shards [lm, r1-r0])."""
        dev, n = self.device, self.r1 - self.r0
        ops = self.ops_cls(n, lm, dev)
        V = torch.zeros((lm, n), dtype=torch.complex128, device=dev)
        V[0] = v0_shard
        alpha = torch.zeros(lm, dtype=torch.complex128, device=dev)
        beta = torch.zeros(lm, dtype=torch.float64, device=dev)
        coef = torch.zeros(lm, dtype=torch.complex128, device=dev)
        maxb = torch.zeros(1, dtype=torch.float64, device=dev)
        norm2 = torch.zeros(1, dtype=torch.float64, device=dev)
        done = torch.zeros(1, dtype=torch.int32, device=dev)
        iters = torch.full((1,), lm, dtype=torch.int32, device=dev)
        send = torch.zeros(self.maxb, dtype=torch.complex128, device=dev)
        gbuf = torch.empty(self.world * self.maxb, dtype=torch.complex128, device=dev)

        r = self.local_apply(self._gather(V[0], send, gbuf))
        ops.axpy_dot(None, V[0], r, None, alpha[0:1], done)          # alpha_0 = <v0, H v0>
        self._sum(alpha[0:1])
        ops.update(None, 0, r, V[0], alpha[0:1], None, norm2, done)  # r -= alpha_0 v0
        self._sum(norm2)
        for i in range(lm - 1):
            ops.beta(i, tol, norm2, beta, maxb, done, iters)
            ops.scale(r, V[i + 1], beta[i:i + 1], done)
            r = self.local_apply(self._gather(V[i + 1], send, gbuf))
            ops.axpy_dot(V[i], V[i + 1], r, beta[i:i + 1], alpha[i + 1:i + 2], done)
            self._sum(alpha[i + 1:i + 2])
            ops.multidot(V, i + 2, r, V[i + 1], alpha[i + 1:i + 2], coef, done)
            self._sum(coef[: i + 2])
            ops.update(V, i + 2, r, V[i + 1], alpha[i + 1:i + 2], coef, norm2, done)
            self._sum(norm2)
        it = int(iters[0])
        return it, alpha.cpu().numpy(), beta.cpu().numpy(), V

    def ground(self, v0_shard, niter: int):
        """Lowest eigenpair (groundStateLieb.c:348-471): (E0, Ritz-vector shard, iterations)."""
        it, alpha, beta, V = self.lanczos(v0_shard, niter)
        n = max(it, 1)
        d, z = tridiag_eig(alpha[:n].real, beta[: max(n - 1, 1)])
        j = int(np.argmin(d))
        zz = torch.tensor(np.ascontiguousarray(z[:, j]), dtype=torch.float64, device=self.device)
        out = torch.empty(self.r1 - self.r0, dtype=torch.complex128, device=self.device)
        self.ops_cls(self.r1 - self.r0, niter, self.device).combine(V, n, zz, out)
        return float(d[j]), out, it
