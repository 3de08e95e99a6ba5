#!/usr/bin/env python
"""Benchmark of the mcpi hot path on B200.

Workload (N=1): the Lieb-Liniger gas of N=16 bosons in M=10 plane waves on a
ring of length L=1, g=1.0 (dimension 2,042,975; integrals of
groundStateLieb.c:129-213), seeded synthetic complex-normal states.

A step is one H.psi of that configuration; `value` is whole-job H.psi/s with
the states resident in HBM, eight distinct states rotating between steps
(8 x 32.7 MB > the 126 MB L2, so every step reads a state that is not cached).
`e2e` is the same metric through the C ABI's host-buffer call
(mcpi_apply_h_host) with every step's state copied in from pinned host memory
and its result copied back out; the call overlaps one step's copies with its
neighbours' H.psi. The line
also carries the roofline of the dominant kernel (CUDA events, measured live),
a 150-step Lanczos ground-state solve of the same configuration, H.psi with
general (dense pair matrix) integrals at N=10 and N=16, M=10, and the CPU
baseline: the oracle's restatement of the reference's applyHconf_X
(hamiltonianMatrix.h:431-887; the reference's fastest CPU H.psi that runs at
this size) on a bounded row sample with all host threads.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mcpi|reference]

With --gpus N > 1 (under torchrun) each rank runs an independent replica of
the H.psi workload on its own GPU (weak scaling); the `sharded` section runs
one row-sharded Lanczos solve across all ranks (NCCL all-gather of each new
Krylov vector and all-reduces of the dots; at N=1 a one-rank group), timed end
to end from a pinned host start vector to the energy and Ritz shard on the
host. The `adjoint` section times H.psi, its adjoint and the transition
densities at N=8, M=8.
`--impl reference` times the CPU oracle port alone (rank 0), on the same
config, metric and unit.
"""
import argparse
import json
import os
import re
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "H·ψ/s (HBM GB/s) & batched E0 solves/s vs plain GPU path at |ΔE0|≤1e-10"
UNIT = "H·ψ/s"
N_PART, M_ORB, G, L_RING = 16, 10, 1.0, 1.0
ROTATE = 8
LANCZOS_ITERS = 150


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=2000)
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", default="mcpi", choices=["mcpi", "reference"])
    p.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU baseline sample budget")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-lanczos", action="store_true")
    p.add_argument("--no-batch", action="store_true")
    p.add_argument("--no-large", action="store_true")
    p.add_argument("--no-general", action="store_true")
    p.add_argument("--no-sharded", action="store_true")
    p.add_argument("--no-adjoint", action="store_true")
    p.add_argument("--profile", choices=["batch", "lanczos", "density", "hpsi"], default=None,
                   help="run only this section (for profiler launch lists), print its timings")
    p.add_argument("--particles", type=int, default=None,
                   help="--profile density: particles of the Lieb-Liniger workload (default 16; M = 10)")
    return p.parse_args()


def config(extra=None):
    c = {"workload": "Lieb-Liniger N=16 M=10 g=1 L=1, H.psi (nc=2042975)",
         "N": N_PART, "M": M_ORB, "g": G, "nc": 2042975,
         "l2": f"{ROTATE} rotating states of 32.7 MB (> 126 MB L2)",
         "parallelism": "replicas"}
    if extra:
        c.update(extra)
    return c


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------

class Clocks:
    """nvidia-smi sampling during the timed region. start() returns once the
    sampler has written its first row (nvidia-smi takes about a second to come
    up), and only the rows written after that count."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.n0 = 0

    def _target(self):
        """nvidia-smi -i selector of the torch device: its PCI bus id where torch has it."""
        try:
            import torch
            p = torch.cuda.get_device_properties(self.device)
            return f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"
        except Exception:
            return str(self.device)

    def _rows(self):
        self.f.flush()
        return [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]

    def start(self):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-i", self._target(), "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
            return
        t0 = time.time()
        while time.time() - t0 < 10.0 and self.proc.poll() is None and not self._rows():
            time.sleep(0.05)
        self.n0 = len(self._rows())

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.15)   # one more sample interval
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = self._rows()[self.n0:]
        os.unlink(self.f.name)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# roofline inputs
# ---------------------------------------------------------------------------

def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_figure(key, kernel):
    """A per-kernel figure (`key kernel value` line) from the committed ncu summaries, or None."""
    for name in ("hpsi_direct_lieb_n16_m10.md", "hpsi_lieb_n16_m10.md"):
        p = os.path.join(ROOT, "profiles", name)
        if not os.path.exists(p):
            continue
        m = re.search(rf"^{key}\s+{kernel}\s+([0-9.eE+]+)", open(p).read(), re.M)
        if m:
            return float(m.group(1))
    return None


def ncu_traffic(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summaries, or None."""
    return ncu_figure("traffic_bytes_per_launch", kernel)


def hpsi_bytes(nc, nc2, P):
    """Algorithmic HBM bytes per launch of the two H.psi kernels: kernel 1
    reads psi once and writes the P x nc2 intermediate E; kernel 2 reads E and
    psi and writes out (16 B per complex)."""
    return {"pair_annihilate": 16 * nc + 16 * P * nc2, "pair_create": 16 * P * nc2 + 32 * nc}


def direct_bytes(nc):
    """Algorithmic HBM bytes per launch of the direct H.psi kernel: psi in, out,
    and the 8-byte packed occupations of every row (the psi gathers are served
    from L2: psi is 16 nc bytes, well under the 126 MB L2 at N=16, M=10)."""
    return 16 * nc + 16 * nc + 8 * nc


def mom_block_sizes(M):
    """Pairs per momentum block K = k + s, K = 0 .. 2M-2."""
    return [K // 2 - max(0, K - (M - 1)) + 1 for K in range(2 * M - 1)]


def direct_gathers(M, nc2):
    """psi gathers of one direct H.psi: every pair a of a block is in
    NC(N-2,M) rows, each gathering the block's other n - 1 pairs."""
    return nc2 * sum(n * (n - 1) for n in mom_block_sizes(M))


def hpsi_terms(M, nc2):
    """Terms (b, a) of one H.psi with momentum-block integrals, diagonal included."""
    return nc2 * sum(n * n for n in mom_block_sizes(M))


# ---------------------------------------------------------------------------
# CPU baseline: oracle restatement of applyHconf_X on a row sample
# ---------------------------------------------------------------------------

def batch_members(count=64, seed=2024):
    """The batched sweep: g log-uniform in [0.01, 100], N uniform in 6..14,
    M uniform in {7, 9, 11}, from one fixed seed."""
    rng = np.random.default_rng(seed)
    N = rng.integers(6, 15, count)
    M = rng.choice([7, 9, 11], count)
    g = 10.0 ** rng.uniform(-2.0, 2.0, count)
    return [(int(n), int(m), float(x)) for n, m, x in zip(N, M, g)]


def run_batch(mc, torch, device, iters=120):
    """64 Lieb-Liniger solves: one graph-captured batch against one solve at a time."""
    members = batch_members()
    starts = []
    b = mc.Batch([(n, m) for n, m, _ in members], iters, device=device)
    for k, (n, m, g) in enumerate(members):
        b.set_integrals(k, *mc.lieb_integrals(m, g, L_RING))
        rng = np.random.default_rng(300 + k)
        C = rng.standard_normal(b.nc[k]) + 1j * rng.standard_normal(b.nc[k])
        C /= np.linalg.norm(C)
        starts.append(C)
        b.set_start(k, C)
    b.run()                                   # capture + instantiate + one run
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    E, it = b.run()
    t_batch = time.perf_counter() - t0
    arena = b.arena_bytes()
    tile, tune_ms = b.schedule()
    hsched, hsched_ms = b.hpsi_schedule()
    b.close()
    spaces = []
    for k, (n, m, g) in enumerate(members):
        sp = mc.FockSpace(n, m, device=device)
        sp.set_integrals(*mc.lieb_integrals(m, g, L_RING))
        spaces.append((sp, torch.from_numpy(starts[k]).to(sp.torch_device)))
    for sp, c in spaces:                       # warm-up: each space allocates its Krylov basis
        sp.ground(c, iters)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    Es = [sp.ground(c, iters)[0] for sp, c in spaces]
    torch.cuda.synchronize()
    t_seq = time.perf_counter() - t0
    for sp, _ in spaces:
        sp.close()
    dE = float(np.max(np.abs(np.array(Es) - E) / np.maximum(1.0, np.abs(np.array(Es)))))
    ncs = [mc.nc_of(n, m) for n, m, _ in members]
    return {"members": len(members), "iterations": iters, "solves_per_s": len(members) / t_batch,
            "seconds": t_batch, "sequential_solves_per_s": len(members) / t_seq,
            "sequential_seconds": t_seq, "speedup_vs_sequential": t_seq / t_batch,
            "max_rel_dE0_vs_sequential": dE, "steps_done_min": int(it.min()),
            "nc_min": min(ncs), "nc_max": max(ncs), "arena_gb": arena / 1e9,
            "tile_rows": tile, "tile_probe_ms": {str(t): float(x) for t, x in zip((512, 1024, 2048), tune_ms)},
            "hpsi_schedule": hsched, "hpsi_schedule_probe_ms": [float(x) for x in hsched_ms]}


def run_sharded(mc, torch, dev, local, world, rank, barrier, max_over_ranks, iters=LANCZOS_ITERS):
    """The row-sharded Lanczos ground state (mcpi_b200/distributed.py) of the
    N=16, M=10 workload over all ranks (NCCL; at one GPU a one-rank group):
    each rank owns nc / world rows of every Krylov vector, all-gathers the new
    vector each step and runs its rows' H.psi and its shard of the
    reorthogonalisation in the library's kernels. Timed end to end: the start
    vector's shard comes from pinned host memory and the ground-state energy
    and Ritz-vector shard go back to the host."""
    import socket

    import torch.distributed as dist

    from mcpi_b200.distributed import ShardedLanczos
    own = not dist.is_initialized()
    if own:
        s = socket.socket()
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
        s.close()
        dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        N, M = N_PART, M_ORB
        sp = mc.FockSpace(N, M, device=local)
        sp.set_integrals(*mc.lieb_integrals(M, G, L_RING))
        sl = ShardedLanczos(sp.nc, lambda v: sp.apply_h_rows(v, sl.r0, sl.r1), dev)
        rng = np.random.default_rng(4321)
        C0 = rng.standard_normal(sp.nc) + 1j * rng.standard_normal(sp.nc)
        C0 /= np.linalg.norm(C0)
        host = torch.from_numpy(C0[sl.r0:sl.r1].copy()).pin_memory()
        sl.ground(host.to(dev), iters)                    # warm-up
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        E0, psi, it = sl.ground(host.to(dev, non_blocking=True), iters)
        psi_h = psi.cpu()
        dt = max_over_ranks(time.perf_counter() - t0)
        n = sl.r1 - sl.r0
        sp.close()
        return {"ranks": world, "rows_per_rank": n, "iterations": it, "E0": E0, "seconds": dt,
                "solves_per_s": 1.0 / dt,
                "e2e": {"value": 1.0 / dt, "unit": "solves/s", "h2d_bytes_per_step": 16 * n,
                        "d2h_bytes_per_step": 16 * n + 8, "api": "ShardedLanczos.ground (mcpi_shard_*, NCCL)"},
                "ritz_shard_norm2": float((psi_h.abs() ** 2).sum())}
    finally:
        if own:
            dist.destroy_process_group()


def run_adjoint(mc, torch, device, reps=200):
    """The adjoint configuration (N=8, M=8, nc = 6,435; random Hermitian Ho and
    8-fold symmetrised Hint): H.psi, its adjoint and the transition densities
    that give the gradients with respect to Ho and Hint, timed with CUDA
    events (mean over reps calls)."""
    N, M = 8, 8
    C, Ho, Hint = mc.random_problem(N, M, 8)
    phi = mc.random_problem(N, M, 9)[0]
    sp = mc.FockSpace(N, M, device=device)
    sp.set_integrals(Ho, Hint)
    x = torch.from_numpy(C).to(sp.torch_device)
    y = torch.from_numpy(phi).to(sp.torch_device)
    out = sp.empty()
    res = {"N": N, "M": M, "nc": sp.nc}
    for name, f in (("apply_h", lambda: sp.apply_h(x, out)), ("apply_h_adjoint", lambda: sp.apply_h_adjoint(y)),
                    ("trans_rho1", lambda: sp.trans_rho1(y, x)), ("trans_rho2", lambda: sp.trans_rho2(y, x))):
        for _ in range(5):
            f()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            f()
        b.record()
        torch.cuda.synchronize()
        res[name + "_us"] = a.elapsed_time(b) / reps * 1e3
    sp.close()
    return res


def run_large(mc, torch, device):
    """N=20, M=10 Lieb-Liniger at g=10 (nc = 10,015,005; 160 MB state): H.psi
    throughput and HBM GB/s, 100 Lanczos steps, rho1 and rho2 of the result."""
    N, M, g = 20, 10, 10.0
    sp = mc.FockSpace(N, M, device=device)
    sp.set_integrals(*mc.lieb_integrals(M, g, L_RING))
    gen = torch.Generator(device=sp.torch_device)
    gen.manual_seed(77)
    x = torch.randn(sp.nc, dtype=torch.complex128, device=sp.torch_device, generator=gen)
    x /= torch.linalg.vector_norm(x)
    out = torch.empty_like(x)
    for _ in range(3):
        sp.apply_h(x, out)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(20):
        sp.apply_h(x, out)
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / 20
    direct = sp.apply_h_profile(x, out, reps=1)[1] == 0.0
    byts = direct_bytes(sp.nc) if direct else sum(hpsi_bytes(sp.nc, mc.nc_of(N - 2, M), sp.P).values())
    sp.ground(x.clone(), 100)                    # warm-up: the space keeps its Krylov basis
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    E0, psi, it = sp.ground(x, 100)
    t_lz = time.perf_counter() - t0
    r1 = sp.rho1(psi)                            # first calls allocate their buffers
    r2 = sp.rho2(psi)
    torch.cuda.synchronize()

    def timed(f, reps=10, v=None):
        # back-to-back calls: the mean device time per call (the host's launch
        # latency overlaps the previous call)
        v = psi if v is None else v
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            y = f(v)
        b.record()
        b.synchronize()
        return y, a.elapsed_time(b) * 1e-3 / reps

    # the densities are timed with the SM clocks sampled around them: right
    # after the Lanczos solve the clocks can still be recovering from it
    # (measured: the first rho2 calls 2.40 ms, the same data seconds later 2.01)
    clk = Clocks(device)
    clk.start()
    r1, t_r1 = timed(sp.rho1, reps=20)
    r2, t_r2 = timed(sp.rho2, reps=20)
    xr = torch.randn(sp.nc, dtype=torch.complex128, device=sp.torch_device, generator=gen)
    _, t_r2x = timed(sp.rho2, reps=20, v=xr)     # the same on a random state: the work is data-independent
    dclk = clk.stop()
    del xr
    occ = r1.diagonal().real.cpu().numpy()
    sp.close()
    return {"workload": "Lieb-Liniger N=20 M=10 g=10 (nc=10015005)", "hpsi_ms": ms,
            "hpsi_per_s": 1e3 / ms, "hpsi_form": "direct" if direct else "two kernels",
            "hpsi_gbs": byts / (ms * 1e-3) / 1e9,
            "lanczos_iterations": it, "E0": E0, "lanczos_seconds": t_lz,
            "rho1_ms": 1e3 * t_r1, "rho2_ms": 1e3 * t_r2, "rho2_random_state_ms": 1e3 * t_r2x,
            "density_clocks": dclk,
            "occupations": [round(float(o), 6) for o in occ]}


def fp64_gemm_peak(torch, device):
    """Measured FP64 reference: cuBLAS DGEMM 8192^3, best of 5 (TFLOP/s)."""
    a = torch.randn(8192, 8192, dtype=torch.float64, device=device)
    b = torch.randn_like(a)
    for _ in range(2):
        c = a @ b
    best = float("inf")
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        c = a @ b
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b, c
    torch.cuda.empty_cache()
    return 2 * 8192 ** 3 / (best * 1e-3) / 1e12


def run_general(mc, torch, device):
    """General (non-momentum-conserving) integrals: random Hermitian Ho and an
    8-fold-symmetrised random Hint, so the pair matrix is dense and kernel 1
    runs as the FP64 tensor-core product. N=10, M=10 (nc = 92,378) and N=16,
    M=10 (nc = 2,042,975); kernel 1 against the measured cuBLAS DGEMM rate
    (algorithmic 8 P^2 nc2 FLOP per launch)."""
    peak = fp64_gemm_peak(torch, device)
    out = {"fp64_peak_tflops": peak, "fp64_peak_source": "cuBLAS DGEMM 8192^3 measured in this run"}
    for (N, M) in [(10, 10), (16, 10)]:
        sp = mc.FockSpace(N, M, device=device)
        _, Ho, Hint = mc.random_problem(4, M, 91)
        sp.set_integrals(Ho, Hint)
        nc2, P = mc.nc_of(N - 2, M), sp.P
        gen = torch.Generator(device=sp.torch_device)
        gen.manual_seed(500 + N)
        X = torch.randn((ROTATE, sp.nc), dtype=torch.complex128, device=sp.torch_device, generator=gen)
        y = torch.empty(sp.nc, dtype=torch.complex128, device=sp.torch_device)
        for w in range(5):
            sp.apply_h(X[w % ROTATE], y)
        torch.cuda.synchronize()
        reps = 50
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for k in range(reps):
            sp.apply_h(X[k % ROTATE], y)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / reps
        k1, k2 = sp.apply_h_profile(X[0], y, reps=20)
        dens = {}
        for name, f in (("rho1_ms", sp.rho1), ("rho2_ms", sp.rho2)):
            f(X[0])                                   # first call allocates its buffer
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for k in range(10):                       # back to back: mean device time per call
                f(X[k % ROTATE])
            b.record()
            b.synchronize()
            dens[name] = a.elapsed_time(b) / 10
        flops = 8.0 * P * P * nc2
        tf = flops / (k1 * 1e-3) / 1e12
        out[f"n{N}_m{M}"] = {"workload": f"random integrals N={N} M={M} (nc={sp.nc})", "hpsi_ms": ms,
                             "hpsi_per_s": 1e3 / ms, "pair_annihilate_ms": k1, "pair_create_ms": k2,
                             "pair_annihilate_tflops": tf, "pair_annihilate_frac_of_dgemm": tf / peak,
                             "pair_annihilate_flops": flops, **dens}
        sp.close()
        del X, y
        torch.cuda.empty_cache()
    return out


def cpu_setup(N, M, g):
    import oracle
    O = oracle.Orc()
    IF = O.focks(N, M)
    Map = O.one_one_map(N, M, IF)
    MapOT, sOT = O.one_two_map(N, M, IF)
    Ho, Hint = O.lieb(M, g, L_RING)
    C = np.random.default_rng(5).standard_normal(O.nc(N, M)) + 0j
    return O, IF, (Map, MapOT, sOT, None, None), Ho, Hint, C


def cpu_rows(O, st, row0, nrows, threads, out):
    IF, maps, Ho, Hint, C = st
    nc = O.nc(N_PART, M_ORB)
    O.apply_h(N_PART, M_ORB, C, Ho, Hint, mode=1, IF=IF, maps=maps, row0=row0,
              row1=min(nc, row0 + nrows), threads=threads, out=out)


def cpu_baseline(budget_s):
    threads = len(os.sched_getaffinity(0))
    O, IF, maps, Ho, Hint, C = cpu_setup(N_PART, M_ORB, G)
    st = (IF, maps, Ho, Hint, C)
    nc = O.nc(N_PART, M_ORB)
    out = np.zeros(nc, np.complex128)
    # calibrate on a strided sample of 16 chunks spread over the index range
    chunks = 16
    rows = 256
    while True:
        t0 = time.perf_counter()
        for c in range(chunks):
            cpu_rows(O, st, c * (nc // chunks), rows, threads, out)
        dt = time.perf_counter() - t0
        if dt > budget_s / 8 or rows * chunks >= nc:
            break
        rows *= 2
    target = int(rows * budget_s / max(dt, 1e-6))
    rows = max(1, min(nc // chunks, target))
    t0 = time.perf_counter()
    for c in range(chunks):
        cpu_rows(O, st, c * (nc // chunks), rows, threads, out)
    dt = time.perf_counter() - t0
    sampled = rows * chunks
    return {"value": (sampled / nc) / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{sampled} of {nc} rows ({chunks} chunks spread over the index range) of "
                      f"the applyHconf_X restatement (oracle/mcpi_oracle.c), {dt:.1f} s, "
                      f"OpenMP over rows; value = sampled fraction / time",
            "seconds": dt}


# ---------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------

def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = len(os.sched_getaffinity(0))
    O, IF, maps, Ho, Hint, C = cpu_setup(N_PART, M_ORB, G)
    st = (IF, maps, Ho, Hint, C)
    nc = O.nc(N_PART, M_ORB)
    out = np.zeros(nc, np.complex128)
    # size each step so that warm-up + steps stay within ~2 minutes
    t0 = time.perf_counter()
    cpu_rows(O, st, nc // 3, 2048, threads, out)
    per_row = (time.perf_counter() - t0) / 2048
    rows = int(max(64, min(nc, 120.0 / max(1, args.steps + args.warmup) / per_row)))
    starts = np.linspace(0, nc - rows, 97).astype(np.int64)
    for w in range(args.warmup):
        cpu_rows(O, st, int(starts[w % len(starts)]), rows, threads, out)
    t0 = time.perf_counter()
    for k in range(args.steps):
        cpu_rows(O, st, int(starts[k % len(starts)]), rows, threads, out)
    dt = time.perf_counter() - t0
    value = args.steps * (rows / nc) / dt
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "data": "synthetic", "impl": "reference",
            "config": config({"parallelism": "cpu", "rows_per_step": rows}),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{rows} rows per step of the applyHconf_X restatement "
                                       f"(oracle/mcpi_oracle.c), steps rotate over 97 offsets"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# mcpi arm
# ---------------------------------------------------------------------------

def run_mcpi(args):
    import torch
    import torch.distributed as dist

    import mcpi_b200 as mc

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    N, M = N_PART, M_ORB
    sp = mc.FockSpace(N, M, device=local)
    Ho, Hint = mc.lieb_integrals(M, G, L_RING)
    sp.set_integrals(Ho, Hint)
    nc, P, nc2 = sp.nc, sp.P, mc.nc_of(N - 2, M)
    gen = torch.Generator(device=dev)
    gen.manual_seed(1234 + rank)
    X = torch.randn((ROTATE, nc), dtype=torch.complex128, device=dev, generator=gen)
    X /= torch.linalg.vector_norm(X, dim=1, keepdim=True)
    out = torch.empty(nc, dtype=torch.complex128, device=dev)

    # ---- device-resident H.psi ----
    for w in range(args.warmup):
        sp.apply_h(X[w % ROTATE], out)
    torch.cuda.synchronize()
    clocks = Clocks(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for k in range(args.steps):
        sp.apply_h(X[k % ROTATE], out)
    e1.record()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1))
    value = world * args.steps / (ms / 1e3)

    # ---- roofline of the dominant kernel (CUDA events on the launching stream,
    # the same rotating states as the timed region) ----
    k1 = k2 = 0.0
    for k in range(2 * ROTATE):
        a, b = sp.apply_h_profile(X[k % ROTATE], out, reps=1)
        k1 += a / (2 * ROTATE)
        k2 += b / (2 * ROTATE)
    peak, peak_kind = measured_peak()
    launches_per_step = 1 if k2 == 0.0 else 2
    if k2 == 0.0:
        # the direct kernel (the default form for these real momentum blocks)
        dom, t_dom, b_dom = "hpsi_direct", k1, direct_bytes(nc)
        kernel_ms = {dom: k1}
        gathers = direct_gathers(M, nc2)
        extra = {"irreducible_bytes": 32 * nc, "terms_per_launch": hpsi_terms(M, nc2),
                 "psi_gathers_per_launch": gathers,
                 "l2_gather_tbs": 16 * gathers / (k1 * 1e-3) / 1e12,
                 # what bounds this kernel instead of HBM (ncu, one launch of the same workload)
                 "binding": {"unit": "SM L1 data pipe (psi gathers + per-row index tables), then issue",
                             "l1_data_pipe_pct": ncu_figure("l1_data_pipe_pct", dom),
                             "issue_active_pct": ncu_figure("issue_active_pct", dom),
                             "source": "profiles/hpsi_direct_lieb_n16_m10.md"}}
    else:
        names = ["pair_annihilate", "pair_create"]
        times = {"pair_annihilate": k1, "pair_create": k2}
        dom = max(names, key=lambda n: times[n])
        byts = hpsi_bytes(nc, nc2, P)
        t_dom, b_dom, kernel_ms = times[dom], byts[dom], times
        extra = {"irreducible_bytes": 32 * nc}
    achieved = b_dom / (t_dom * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": ncu_traffic(dom), "algorithmic_bytes": b_dom, **extra, "kernel_ms": kernel_ms}
    # the two pair kernels on the same states, for comparison (MCPI_OPT_DIRECT_HPSI = 0)
    if k2 == 0.0:
        sp.set_option(mc.OPT_DIRECT_HPSI, 0)
        for w in range(3):
            sp.apply_h(X[w % ROTATE], out)
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record()
        for k in range(args.steps):
            sp.apply_h(X[k % ROTATE], out)
        t1.record()
        torch.cuda.synchronize()
        roofline["two_kernel_form_ms"] = t0.elapsed_time(t1) / args.steps
        sp.set_option(mc.OPT_DIRECT_HPSI, 2)

    # ---- e2e through the C ABI with HOST buffers (mcpi_apply_h_host) ----
    # every step copies its state in from pinned host memory and its result
    # back out; the call pipelines copy-in, H.psi and copy-out across steps
    hX = [torch.empty(nc, dtype=torch.complex128).pin_memory() for _ in range(ROTATE)]
    for k in range(ROTATE):
        hX[k].copy_(X[k].cpu())
    hO = [torch.empty(nc, dtype=torch.complex128).pin_memory() for _ in range(ROTATE)]
    ke = max(10, min(args.steps, 200))
    ins = [hX[k % ROTATE] for k in range(ke)]
    outs = [hO[k % ROTATE] for k in range(ke)]
    sp.apply_h_host(ins[:4], outs[:4])           # warm-up (creates the pipeline buffers)
    torch.cuda.synchronize()
    barrier()
    h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    h0.record()
    sp.apply_h_host(ins, outs)                   # returns when every result is in host memory
    h1.record()
    h1.synchronize()
    ems = max_over_ranks(h0.elapsed_time(h1))
    e2e = {"value": world * ke / (ems / 1e3), "unit": UNIT, "h2d_bytes_per_step": 16 * nc,
           "d2h_bytes_per_step": 16 * nc, "steps": ke, "api": "mcpi_apply_h_host (C ABI, host buffers)"}
    # the same, one state per call (copy in, H.psi, copy out, synchronise)
    dx = torch.empty(nc, dtype=torch.complex128, device=dev)
    for w in range(3):
        dx.copy_(hX[0], non_blocking=True)
        sp.apply_h(dx, out)
        hO[0].copy_(out, non_blocking=True)
    torch.cuda.synchronize()
    barrier()
    a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a0.record()
    for k in range(ke):
        dx.copy_(hX[k % ROTATE], non_blocking=True)
        sp.apply_h(dx, out)
        hO[k % ROTATE].copy_(out, non_blocking=True)
    a1.record()
    torch.cuda.synchronize()
    barrier()
    sms = max_over_ranks(a0.elapsed_time(a1))
    e2e["one_state_per_call"] = {"value": world * ke / (sms / 1e3), "unit": UNIT}
    # the host link's own bound: the same state-sized copies in and out at once
    # on two streams with no H.psi (states per second = what e2e can reach)
    s_in, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    dy = torch.empty_like(dx)
    torch.cuda.synchronize()
    l0, l1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0.record()
    s_in.wait_event(l0)
    s_out.wait_event(l0)
    for k in range(ke):
        with torch.cuda.stream(s_in):
            dx.copy_(hX[k % ROTATE], non_blocking=True)
        with torch.cuda.stream(s_out):
            hO[k % ROTATE].copy_(dy, non_blocking=True)
    torch.cuda.current_stream(dev).wait_stream(s_in)
    torch.cuda.current_stream(dev).wait_stream(s_out)
    l1.record()
    torch.cuda.synchronize()
    lms = max_over_ranks(l0.elapsed_time(l1))
    e2e["host_link_bound"] = {"value": world * ke / (lms / 1e3), "unit": UNIT,
                              "gbs_each_way": 16 * nc * ke / (lms / 1e3) / 1e9,
                              "what": "state-sized copies in and out at once, no H.psi"}

    # ---- Lanczos ground state of the same configuration ----
    lanczos = None
    if not args.no_lanczos:
        sp.ground(X[1].clone(), LANCZOS_ITERS)          # warm-up: the space keeps its Krylov basis
        C0 = X[0].clone()
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        E0, psi, it = sp.ground(C0, LANCZOS_ITERS)
        dt = max_over_ranks(time.perf_counter() - t0)
        occ = sp.rho1(psi).diagonal().real.cpu().numpy()
        lanczos = {"iterations": it, "E0": E0, "E0_per_N": E0 / N, "seconds": dt,
                   "solves_per_s": world / dt, "occupations": [round(float(o), 6) for o in occ]}

    sharded = None
    if not args.no_sharded:
        sharded = run_sharded(mc, torch, dev, local, world, rank, barrier, max_over_ranks)
        if lanczos is not None:
            sharded["single_gpu_seconds"] = lanczos["seconds"]
    adjoint = None
    if not args.no_adjoint:
        adjoint = run_adjoint(mc, torch, local)

    batched = None
    if not args.no_batch:
        batched = run_batch(mc, torch, local)
    large = None
    if not args.no_large:
        large = run_large(mc, torch, local)
    general = None
    if not args.no_general:
        general = run_general(mc, torch, local)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.cpu_seconds)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
                "config": config(), "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": launches_per_step * args.steps, "clocks": clk, "lanczos": lanczos, "sharded": sharded,
                "adjoint": adjoint, "batched": batched, "large": large, "general": general}
        print(json.dumps(line), flush=True)
    sp.close()
    if world > 1:
        dist.destroy_process_group()


def run_profile(args):
    """One section alone, for ncu: 'batch' = the 64-member sweep (graph capture
    with the autotuner, then one replay); 'lanczos' = one 150-step ground state
    of the N=16, M=10 workload after a warm-up solve; 'density' = rho1, rho2
    and the transition rho2 of seeded N=16, M=10 states (--steps calls each
    after --warmup, CUDA events); 'hpsi' = H.psi of the N=16, M=10 workload
    with the two pair kernels, the fused kernel and the direct kernel."""
    import torch

    import mcpi_b200 as mc
    if args.profile == "batch":
        members = batch_members()
        b = mc.Batch([(n, m) for n, m, _ in members], 120, device=0)
        for k, (n, m, g) in enumerate(members):
            b.set_integrals(k, *mc.lieb_integrals(m, g, L_RING))
            rng = np.random.default_rng(300 + k)
            C = rng.standard_normal(b.nc[k]) + 1j * rng.standard_normal(b.nc[k])
            b.set_start(k, C / np.linalg.norm(C))
        b.run()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b.run()
        dt = time.perf_counter() - t0
        out = {"section": "batch", "seconds": dt, "schedule": b.schedule()[0]}
        b.close()
    elif args.profile == "density":
        n_part = args.particles or N_PART
        sp = mc.FockSpace(n_part, M_ORB, device=0)
        sp.set_integrals(*mc.lieb_integrals(M_ORB, G, L_RING))
        gen = torch.Generator(device=sp.torch_device)
        gen.manual_seed(1234)
        x, y = (torch.randn(sp.nc, dtype=torch.complex128, device=sp.torch_device, generator=gen)
                for _ in range(2))
        x /= torch.linalg.vector_norm(x)
        y /= torch.linalg.vector_norm(y)
        out = {"section": "density", "workload": f"Lieb-Liniger N={n_part} M={M_ORB} (nc={sp.nc})"}
        for name, f in (("rho1", lambda: sp.rho1(x)), ("rho2", lambda: sp.rho2(x)),
                        ("trans_rho2", lambda: sp.trans_rho2(y, x))):
            for _ in range(args.warmup):
                f()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            a.record()
            for _ in range(args.steps):
                f()
            b.record()
            torch.cuda.synchronize()
            out[name + "_ms"] = a.elapsed_time(b) / args.steps
        sp.close()
    elif args.profile == "hpsi":
        # H.psi of the N=16, M=10 workload in its three forms: the two pair
        # kernels, the fused kernel (MCPI_OPT_FUSED_HPSI; lead 192) and the
        # direct kernel (MCPI_OPT_DIRECT_HPSI), --steps calls each on rotating
        # states after --warmup. The fused form agrees with the two kernels bit
        # for bit; the direct form sums in another order (relative difference)
        gen = torch.Generator(device="cuda:0")
        gen.manual_seed(1234)
        X = None
        out = {"section": "hpsi", "workload": f"Lieb-Liniger N={N_PART} M={M_ORB}"}
        ref = None
        for name, fused, direct in (("two_kernels", 0, 0), ("fused", 1, 0), ("direct", 0, 1)):
            sp = mc.FockSpace(N_PART, M_ORB, device=0)
            sp.set_option(mc.OPT_DIRECT_HPSI, direct)
            sp.set_option(mc.OPT_FUSED_HPSI, fused)
            sp.set_option(mc.OPT_FUSED_LEAD, 192)
            sp.set_integrals(*mc.lieb_integrals(M_ORB, G, L_RING))
            if X is None:
                X = torch.randn((ROTATE, sp.nc), dtype=torch.complex128, device=sp.torch_device, generator=gen)
            y = sp.empty()
            for w in range(args.warmup):
                sp.apply_h(X[w % ROTATE], y)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            a.record()
            for k in range(args.steps):
                sp.apply_h(X[k % ROTATE], y)
            b.record()
            torch.cuda.synchronize()
            out[name + "_ms"] = a.elapsed_time(b) / args.steps
            z = sp.apply_h(X[0])
            if ref is None:
                ref = z
            elif name == "fused":
                out["fused_bitwise_equal"] = bool(torch.equal(ref, z))
            else:
                out["direct_rel_diff"] = float(torch.linalg.vector_norm(z - ref) / torch.linalg.vector_norm(ref))
            sp.close()
    else:
        sp = mc.FockSpace(N_PART, M_ORB, device=0)
        sp.set_integrals(*mc.lieb_integrals(M_ORB, G, L_RING))
        gen = torch.Generator(device=sp.torch_device)
        gen.manual_seed(1234)
        x = torch.randn(sp.nc, dtype=torch.complex128, device=sp.torch_device, generator=gen)
        x /= torch.linalg.vector_norm(x)
        sp.ground(x, LANCZOS_ITERS)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        E0, _, it = sp.ground(x, LANCZOS_ITERS)
        out = {"section": "lanczos", "seconds": time.perf_counter() - t0, "E0": E0, "iterations": it}
        sp.close()
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    if args.profile:
        run_profile(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_mcpi(args)


if __name__ == "__main__":
    main()
