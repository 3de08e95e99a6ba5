"""Row-sharded Lanczos (mcpi_b200/distributed.py) with world sizes 2 and 3 on CPU (gloo).

The local operator is the oracle's row-range H.psi (the GPU path uses
mcpi_apply_h_rows); what is tested is the sharding, the all-gathers and the
all-reduces of dots and reorthogonalisation coefficients. The sharded
tridiagonal and ground-state energy must match the single-process oracle."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, N, M, kind, lm, out_dir):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from mcpi_b200.distributed import ShardedLanczos, row_block
    orc = oracle.Orc()
    if kind == "lieb":
        Ho, Hint = orc.lieb(M, 3.0)
    else:
        _, Ho, Hint = oracle.random_inputs(N, M, 11)
    nc = orc.nc(N, M)
    IF = orc.focks(N, M)
    C0 = oracle.random_inputs(N, M, 12)[0]
    r0, r1 = row_block(nc, world, rank)

    def local_apply(v_full):
        out = orc.apply_h(N, M, v_full.numpy(), Ho, Hint, mode=2, IF=IF, row0=r0, row1=r1, threads=1)
        return torch.from_numpy(out[r0:r1].copy())

    sl = ShardedLanczos(nc, local_apply, torch.device("cpu"))
    it, alpha, beta, _ = sl.lanczos(torch.from_numpy(C0[r0:r1].copy()), lm)
    E, psi, it2 = sl.ground(torch.from_numpy(C0[r0:r1].copy()), lm)
    np.savez(os.path.join(out_dir, f"r{rank}.npz"), it=it, alpha=alpha, beta=beta, E=E,
             psi=psi.numpy(), r0=r0, r1=r1)
    dist.destroy_process_group()


@pytest.mark.parametrize("world,N,M,kind,lm", [(2, 6, 7, "lieb", 40), (2, 5, 5, "random", 30),
                                               (3, 9, 5, "lieb", 40), (3, 10, 4, "random", 30)])
def test_sharded_lanczos(tmp_path, orc, world, N, M, kind, lm):
    # world 3: nc = 715 and 286 split into uneven row blocks (239/238/238, 96/95/95)
    if world == 3:
        assert orc.nc(N, M) % world != 0
    mp.start_processes(_worker, args=(world, _free_port(), N, M, kind, lm, str(tmp_path)), nprocs=world,
                       start_method="spawn")
    r = [dict(np.load(tmp_path / f"r{k}.npz")) for k in range(world)]
    if kind == "lieb":
        Ho, Hint = orc.lieb(M, 3.0)
    else:
        _, Ho, Hint = oracle.random_inputs(N, M, 11)
    C0 = oracle.random_inputs(N, M, 12)[0]
    it, alpha, beta, _ = orc.lanczos(N, M, Ho, Hint, C0, lm, mode=2)
    E, psi, _ = orc.ground(N, M, Ho, Hint, C0, lm, mode=2)
    for x in r:
        assert int(x["it"]) == it
        scale = np.abs(alpha).max()
        assert np.abs(x["alpha"][:it] - alpha[:it]).max() <= 1e-10 * scale
        assert np.abs(x["beta"][: it - 1] - beta[: it - 1].real).max() <= 1e-10 * scale
        assert abs(float(x["E"]) - E) <= 1e-10 * max(1.0, abs(E))
    full = np.concatenate([x["psi"] for x in r])
    ov = abs(np.vdot(full, psi)) / (np.linalg.norm(full) * np.linalg.norm(psi))
    assert abs(ov - 1) < 1e-9
