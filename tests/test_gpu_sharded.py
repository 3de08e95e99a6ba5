"""Row-range H.psi on the GPU and the sharded Lanczos driver over NCCL (one rank
here: the only GPU count these runs have); the multi-rank logic is covered on
CPU by tests/test_distributed.py."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist

import mcpi_b200 as mc
from conftest import rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["random", "lieb"])
def test_apply_h_rows_matches_full(kind):
    # with Lieb integrals (momentum-block form) the pair-annihilation kernel runs
    # only over the (N-2)-configurations the row block reads
    N, M = 9, 8
    C, Ho, Hint = mc.random_problem(N, M, 101)
    if kind == "lieb":
        Ho, Hint = mc.lieb_integrals(M, 2.5)
    sp = mc.FockSpace(N, M)
    sp.set_integrals(Ho, Hint)
    full = sp.apply_h(C).cpu().numpy()
    nc = sp.nc
    for r0, r1 in [(0, nc), (0, 1), (nc - 1, nc), (123, 4567), (nc // 3, nc // 3 + 257), (5, 5),
                   (nc // 2, nc), (0, nc // 8), (nc // 8, 2 * nc // 8), (7 * nc // 8, nc)]:
        part = sp.apply_h_rows(C, r0, r1).cpu().numpy()
        assert np.array_equal(part, full[r0:r1])        # same kernels, same arithmetic
    for r0, r1 in [(0, nc // 8), (nc // 8, 2 * nc // 8), (0, nc // 8)]:   # the cached range, and a new one
        C2 = np.roll(C, r0 + 1)
        assert np.array_equal(sp.apply_h_rows(C2, r0, r1).cpu().numpy(), sp.apply_h(C2).cpu().numpy()[r0:r1])


def test_sharded_lanczos_nccl_one_rank():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        from mcpi_b200.distributed import ShardedLanczos
        N, M = 10, 9
        sp = mc.FockSpace(N, M)
        sp.set_integrals(*mc.lieb_integrals(M, 5.0))
        C0 = torch.from_numpy(mc.random_problem(N, M, 102)[0]).cuda()
        sl = ShardedLanczos(sp.nc, lambda v: sp.apply_h_rows(v, sl.r0, sl.r1), torch.device("cuda"))
        # one rank runs the same kernels in the same order as mcpi_lanczos: bit for bit
        it, alpha, beta, _ = sl.lanczos(C0[sl.r0:sl.r1].clone(), 80)
        it1, alpha1, beta1, _ = sp.lanczos(C0, 80)
        assert it == it1 == 80
        assert np.array_equal(alpha, alpha1) and np.array_equal(beta[:79], beta1[:79])
        E, psi, it = sl.ground(C0[sl.r0:sl.r1].clone(), 80)
        E1, psi1, it1 = sp.ground(C0, 80)
        assert it == it1 and abs(E - E1) <= 1e-10 * abs(E1)
        assert rel(psi.cpu().numpy() * np.sign(np.vdot(psi1.cpu().numpy(), psi.cpu().numpy()).real),
                   psi1.cpu().numpy()) < 1e-8
    finally:
        dist.destroy_process_group()


def _virtual_ranks(sp, C0, lm, W):
    """W ranks with uneven row blocks emulated in one process on one GPU: each
    rank's shard of every step runs in the library's kernels (mcpi_shard_*,
    mcpi_apply_h_rows on the gathered vector), and the all-reduce is the sum of
    the ranks' device scalars. Returns (iterations, alpha, beta) on the host."""
    from mcpi_b200.distributed import DeviceShardOps, row_block
    nc = sp.nc
    blocks = [row_block(nc, W, r) for r in range(W)]
    dev = torch.device("cuda")
    ops = [DeviceShardOps(b - a, lm, dev) for a, b in blocks]
    V = [torch.zeros((lm, b - a), dtype=torch.complex128, device=dev) for a, b in blocks]
    for r, (a, b) in enumerate(blocks):
        V[r][0] = C0[a:b]
    alpha = [torch.zeros(lm, dtype=torch.complex128, device=dev) for _ in range(W)]
    beta = torch.zeros(lm, dtype=torch.float64, device=dev)
    coef = [torch.zeros(lm, dtype=torch.complex128, device=dev) for _ in range(W)]
    norm2 = [torch.zeros(1, dtype=torch.float64, device=dev) for _ in range(W)]
    maxb = torch.zeros(1, dtype=torch.float64, device=dev)
    done = torch.zeros(1, dtype=torch.int32, device=dev)
    iters = torch.full((1,), lm, dtype=torch.int32, device=dev)

    def allsum(ts, sl):
        tot = sum(t[sl] for t in ts)
        for t in ts:
            t[sl] = tot

    def gather(i):
        return torch.cat([V[r][i] for r in range(W)])

    full = gather(0)
    R = [sp.apply_h_rows(full, a, b) for a, b in blocks]
    for r in range(W):
        ops[r].axpy_dot(None, V[r][0], R[r], None, alpha[r][0:1], done)
    allsum(alpha, slice(0, 1))
    for r in range(W):
        ops[r].update(None, 0, R[r], V[r][0], alpha[r][0:1], None, norm2[r], done)
    allsum(norm2, slice(0, 1))
    for i in range(lm - 1):
        ops[0].beta(i, 1e-15, norm2[0], beta, maxb, done, iters)
        for r in range(W):
            ops[r].scale(R[r], V[r][i + 1], beta[i:i + 1], done)
        full = gather(i + 1)
        R = [sp.apply_h_rows(full, a, b) for a, b in blocks]
        for r in range(W):
            ops[r].axpy_dot(V[r][i], V[r][i + 1], R[r], beta[i:i + 1], alpha[r][i + 1:i + 2], done)
        allsum(alpha, slice(i + 1, i + 2))
        for r in range(W):
            ops[r].multidot(V[r], i + 2, R[r], V[r][i + 1], alpha[r][i + 1:i + 2], coef[r], done)
        allsum(coef, slice(0, i + 2))
        for r in range(W):
            ops[r].update(V[r], i + 2, R[r], V[r][i + 1], alpha[r][i + 1:i + 2], coef[r], norm2[r], done)
        allsum(norm2, slice(0, 1))
    out = int(iters[0]), alpha[0].cpu().numpy(), beta.cpu().numpy()
    del V, R, full
    return out


@pytest.mark.parametrize("N,M,lm,W,g,direct", [(10, 8, 60, 3, 4.0, 2), (20, 11, 12, 4, 1.0, 2),
                                                (20, 11, 12, 4, 1.0, 0)])
def test_shard_primitives_virtual_ranks(N, M, lm, W, g, direct):
    # uneven row blocks; the direct H.psi form on each rank's rows, or (direct
    # = 0) the two pair kernels with kernel 1 over each block's E columns; N=20,
    # M=11 (nc = 30,045,015) is beyond the reference's int32 maps. The
    # recurrence must match mcpi_lanczos on the whole space.
    sp = mc.FockSpace(N, M)
    sp.set_option(mc.OPT_DIRECT_HPSI, direct)
    sp.set_integrals(*mc.lieb_integrals(M, g))
    assert sp.nc % W != 0
    gen = torch.Generator(device="cuda")
    gen.manual_seed(103)
    C0 = torch.randn(sp.nc, dtype=torch.complex128, device="cuda", generator=gen)
    C0 /= torch.linalg.vector_norm(C0)
    it, a, b = _virtual_ranks(sp, C0, lm, W)
    it1, alpha1, beta1, lvec = sp.lanczos(C0, lm)
    del lvec
    assert it == it1 == lm
    scale = np.abs(alpha1).max()
    assert np.abs(a - alpha1).max() <= 1e-10 * scale
    assert np.abs(b[: lm - 1] - beta1[: lm - 1]).max() <= 1e-10 * scale
    sp.close()
