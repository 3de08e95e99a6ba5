"""The reference's CUDA H.psi kernel (cuda/hamiltonianMatrix.cuh:60-626), its
source compiled as host C++ under AddressSanitizer and run over every row
(oracle/refcuda_host.cpp): no access outside the reference's own exact-size
maps, and the same H C as the oracle, on the reference driver's deterministic
inputs (performanceTest.c:169-219) and on seeded random ones, up to N=10, M=10.
This is the CPU check of the kernel's indexing that precedes running it on a GPU
(tests/test_gpu_refcuda.py)."""
import pytest

import oracle
from conftest import rel

pytestmark = pytest.mark.skipif(not oracle.refcuda_available(),
                                reason="reference CUDA harness not built (needs the reference sources)")


@pytest.mark.parametrize("N,M", [(1, 4), (2, 3), (3, 5), (5, 5), (6, 7), (8, 8), (10, 10)])
def test_reference_cuda_kernel_on_host(orc, tmp_path, N, M):
    cases = [orc.perf_inputs(N, M)]
    if N * M <= 64:
        cases.append(oracle.random_inputs(N, M, 7))
    for C, Ho, Hint in cases:
        out = oracle.refcuda_host_apply_h(N, M, C, Ho, Hint, str(tmp_path))
        assert rel(out, orc.apply_h(N, M, C, Ho, Hint, mode=2)) <= 1e-14
