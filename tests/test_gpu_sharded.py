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


def test_apply_h_rows_matches_full():
    N, M = 9, 8
    C, Ho, Hint = mc.random_problem(N, M, 101)
    sp = mc.FockSpace(N, M)
    sp.set_integrals(Ho, Hint)
    full = sp.apply_h(C).cpu().numpy()
    nc = sp.nc
    for r0, r1 in [(0, nc), (0, 1), (nc - 1, nc), (123, 4567), (nc // 3, nc // 3 + 257), (5, 5)]:
        part = sp.apply_h_rows(C, r0, r1).cpu().numpy()
        assert np.array_equal(part, full[r0:r1])        # same kernels, same arithmetic


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
        E, psi, it = sl.ground(C0[sl.r0:sl.r1].clone(), 80)
        E1, psi1, it1 = sp.ground(C0, 80)
        assert it == it1 and abs(E - E1) <= 1e-10 * abs(E1)
        assert rel(psi.cpu().numpy() * np.sign(np.vdot(psi1.cpu().numpy(), psi.cpu().numpy()).real),
                   psi1.cpu().numpy()) < 1e-8
    finally:
        dist.destroy_process_group()
