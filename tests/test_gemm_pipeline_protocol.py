"""The buffer hand-over of the warp-specialised dense-product kernel
(mcpi_b200/csrc/hpsi.cu, k_pair_annihilate_gemm_ws), simulated at warp
granularity on the CPU under random schedules.

The kernel's schedule, restated: a block owns ntb tiles; tile i uses buffer
b = i % NS.
  gather warps (G groups of 2 warps; group g fills tiles i = g, g+G, ...):
      if i >= NS: wait(empty[b], parity (i / NS - 1) & 1)
      gather + coefficients into buffer b
      arrive(full[b])                        (full[b] counts the group's threads)
  product warps (16):
      wait(full[b], parity (i / NS) & 1)
      read buffer b
      if i + NS < ntb: arrive(empty[b])      (empty[b] counts the 16 warps)
mbarrier semantics: a phase completes when its arrival count is reached; a wait
on parity P passes once the barrier's completed-phase count has parity != P.
Checked for NS = 2, 3 and one or two gather groups, every tile count 1..12:
no deadlock, no wait passing on the wrong phase, no buffer overwritten before
all product warps read it, no product warp reading a buffer before the whole
tile landed, and no arrivals left pending when the kernel ends."""
import random

import pytest

N_PROD = 16          # product warps
N_GATHER = 4         # gather warps


def _program(role, ntb, ns, groups, grp):
    ops = []
    for i in range(ntb):
        b = i % ns
        if role == "gather":
            if i % groups != grp:
                continue
            if i >= ns:
                ops.append(("wait", ("empty", b), ((i - ns) // ns) & 1, (i - ns) // ns))
            ops.append(("gather", i))
            ops.append(("arrive", ("full", b)))
        else:
            ops.append(("wait", ("full", b), (i // ns) & 1, i // ns))
            ops.append(("read", i))
            if i + ns < ntb:
                ops.append(("arrive", ("empty", b)))
    return ops


def _run(ntb, ns, groups, seed):
    rng = random.Random(seed)
    warps = [_program("prod", ntb, ns, groups, 0) for _ in range(N_PROD)]
    warps += [_program("gather", ntb, ns, groups, w % groups) for w in range(N_GATHER)]
    pc = [0] * len(warps)
    bars = [(k, b) for k in ("full", "empty") for b in range(ns)]
    count = dict.fromkeys(bars, 0)
    phases = dict.fromkeys(bars, 0)
    need = {bar: (N_GATHER // groups if bar[0] == "full" else N_PROD) for bar in bars}
    tile_in = [None] * ns
    landed = [0] * ns
    readers = [0] * ns
    while True:
        ready = []
        for w, prog in enumerate(warps):
            if pc[w] == len(prog):
                continue
            op = prog[pc[w]]
            if op[0] == "wait":
                if (phases[op[1]] & 1) != op[2]:
                    assert phases[op[1]] == op[3] + 1, "a wait passed on the wrong phase"
                    ready.append(w)
            else:
                ready.append(w)
        if not ready:
            assert all(pc[w] == len(p) for w, p in enumerate(warps)), "deadlock"
            assert all(v == 0 for v in count.values()), "arrivals left pending"
            return
        w = rng.choice(ready)
        op = warps[w][pc[w]]
        pc[w] += 1
        if op[0] == "arrive":
            count[op[1]] += 1
            if count[op[1]] == need[op[1]]:
                count[op[1]] = 0
                phases[op[1]] += 1
        elif op[0] == "gather":
            i = op[1]
            b = i % ns
            if tile_in[b] != i:
                if tile_in[b] is not None:
                    assert readers[b] == N_PROD, "buffer overwritten before every product warp read it"
                tile_in[b], landed[b], readers[b] = i, 0, 0
            landed[b] += 1
        elif op[0] == "read":
            i = op[1]
            b = i % ns
            assert tile_in[b] == i and landed[b] == N_GATHER // groups, "read before the tile landed"
            readers[b] += 1


@pytest.mark.parametrize("ns", [2, 3])
@pytest.mark.parametrize("groups", [1, 2])
def test_handover_protocol(ns, groups):
    for ntb in range(1, 13):
        for seed in range(60):
            _run(ntb, ns, groups, seed)


def test_simulator_catches_a_broken_schedule():
    # plant a mistake in the restated schedule (product warps release a buffer
    # without having read it) and check that the simulation rejects it
    global _program
    original = _program

    def broken(role, ntb, ns, groups, grp):
        ops = original(role, ntb, ns, groups, grp)
        return [op for op in ops if op[0] != "read"] if role == "prod" else ops

    try:
        _program = broken
        with pytest.raises(AssertionError):
            for seed in range(50):
                _run(6, 2, 2, seed)
    finally:
        _program = original
