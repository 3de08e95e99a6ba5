"""The reference's own CUDA H.psi kernel (cuda/hamiltonianMatrix.cuh:60-626,
launched as cuda/performanceTest.cu:315-323) on this GPU, through the harness
oracle/refcuda.cu: its output against the oracle and against the B200 path on
the same inputs, and both timed with CUDA events on the same GPU at N=10, M=10
(the reference's own CPU-runnable configuration, nc = 92,378), the largest
workload its int32 maps allow in reasonable host build time. Its indexing is
checked on the CPU first (tests/test_refcuda_host.py)."""
import pytest
import torch

import mcpi_b200 as mc
import oracle
from conftest import rel

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.refcuda_available(),
                                 reason="reference CUDA harness not built (needs the reference sources)")]


@pytest.fixture(scope="module")
def refcuda():
    return oracle.RefCuda()


def _inputs(orc, N, M, kind):
    if kind == "perf":
        return orc.perf_inputs(N, M)
    if kind == "lieb":
        C = oracle.random_inputs(N, M, 11)[0]
        return (C,) + mc.lieb_integrals(M, 1.0)
    return oracle.random_inputs(N, M, 12)


@pytest.mark.parametrize("N,M", [(1, 4), (3, 5), (5, 5), (8, 8), (10, 10)])
@pytest.mark.parametrize("kind", ["perf", "random", "lieb"])
def test_reference_kernel_parity(orc, refcuda, N, M, kind):
    C, Ho, Hint = _inputs(orc, N, M, kind)
    got, _, _ = refcuda.apply_h(N, M, C, Ho, Hint)
    want = orc.apply_h(N, M, C, Ho, Hint, mode=2)
    assert rel(got, want) <= 1e-12
    sp = mc.FockSpace(N, M)
    sp.set_integrals(Ho, Hint)
    ours = sp.apply_h(C).cpu().numpy()
    assert rel(ours, got) <= 1e-12


def _time_ours(sp, C, reps):
    x = torch.tensor(C, device="cuda")
    out = torch.empty_like(x)
    for _ in range(3):
        sp.apply_h(x, out)
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(s)
    for _ in range(reps):
        sp.apply_h(x, out)
    e1.record(s)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps, out


@pytest.mark.parametrize("kind", ["random", "lieb"])
def test_reference_kernel_timing_n10_m10(orc, refcuda, kind):
    N, M, reps = 10, 10, 50
    C, Ho, Hint = _inputs(orc, N, M, kind)
    got, ms_ref, map_bytes = refcuda.apply_h(N, M, C, Ho, Hint, reps=reps)
    sp = mc.FockSpace(N, M)
    sp.set_integrals(Ho, Hint)
    ms_ours, out = _time_ours(sp, C, reps)
    assert rel(out.cpu().numpy(), got) <= 1e-12
    print(f"\nN=10 M=10 {kind}: reference CUDA applyHconf {ms_ref:.4f} ms/H.psi "
          f"(int32 tables {map_bytes / 1e9:.3f} GB), B200 path {ms_ours:.4f} ms/H.psi, "
          f"speed-up {ms_ref / ms_ours:.1f}x")
    assert ms_ours < ms_ref
