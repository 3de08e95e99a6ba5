"""mcpi_apply_h_static: H.psi for callers that cannot allocate device memory.

The entry point takes all its scratch from a fixed array inside the library.
This file is collected last on purpose (its name sorts last), so that a run
that stops at the first failure has already run every other test; it also
passes on its own in a fresh process. Each check compares the allocation-free
result with mcpi_apply_h on a FockSpace, the library's regular entry point,
over two calls in a row (the second call reuses the array the first one left
behind)."""
import ctypes as ct

import numpy as np
import pytest
import torch

import mcpi_b200 as mc
from conftest import rel

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _static(N, M, Ho, Hint, C, variant=mc.VARIANT_MAPS):
    L = mc.lib()
    f = L.mcpi_apply_h_static
    f.restype = ct.c_int
    f.argtypes = [ct.c_int, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_void_p,
                  ct.c_void_p]
    Ho = np.ascontiguousarray(Ho, np.complex128)
    Hint = np.ascontiguousarray(Hint, np.complex128)
    x = torch.from_numpy(np.ascontiguousarray(C, np.complex128)).cuda()
    out = torch.empty_like(x)
    stream = torch.cuda.current_stream().cuda_stream
    rc = f(N, M, Ho.ctypes.data, Hint.ctypes.data, variant, x.data_ptr(), out.data_ptr(),
           ct.c_void_p(stream))
    torch.cuda.synchronize()
    return rc, out.cpu().numpy()


def _regular(N, M, Ho, Hint, C, variant=mc.VARIANT_MAPS, same_kernels=False):
    sp = mc.FockSpace(N, M)
    if same_kernels:
        # the compressed-row pair kernel and index decoding, as the static path runs
        for opt in (mc.OPT_DENSE_PAIR_KERNEL, mc.OPT_NO_MOMENTUM_KERNEL, mc.OPT_NO_GEMM_KERNEL,
                    mc.OPT_NO_OCC_TABLES):
            sp.set_option(opt, 1)
    sp.set_integrals(Ho, Hint, variant)
    out = sp.apply_h(C).cpu().numpy()
    sp.close()
    return out


def test_static_matches_regular_two_calls():
    # 1st call: random integrals with the 8-fold symmetry, N=8, M=8
    C1, Ho1, Hint1 = mc.random_problem(8, 8, 71)
    rc, got1 = _static(8, 8, Ho1, Hint1, C1)
    assert rc == 0
    assert rel(got1, _regular(8, 8, Ho1, Hint1, C1)) <= TOL
    # 2nd call, different space and integrals, on the same array
    Ho2, Hint2 = mc.lieb_integrals(10, 3.0)
    C2 = mc.random_problem(10, 10, 72)[0]
    rc, got2 = _static(10, 10, Ho2, Hint2, C2)
    assert rc == 0
    assert rel(got2, _regular(10, 10, Ho2, Hint2, C2)) <= TOL


def test_static_variants_and_small_spaces():
    for N, M, variant in [(6, 5, mc.VARIANT_HASH), (1, 4, mc.VARIANT_MAPS), (0, 3, mc.VARIANT_MAPS)]:
        rng = np.random.default_rng(N + M)
        C, Ho, _ = mc.random_problem(N, M, 73)
        Hint = rng.standard_normal(M ** 4) + 1j * rng.standard_normal(M ** 4)   # no symmetry
        for _ in range(2):
            rc, got = _static(N, M, Ho, Hint, C, variant)
            assert rc == 0
            assert rel(got, _regular(N, M, Ho, Hint, C, variant)) <= TOL, (N, M)


def test_static_rejects_oversize():
    # N=16, M=10 needs ~720 MB of intermediate: far beyond the fixed array
    Ho, Hint = mc.lieb_integrals(10, 1.0)
    L = mc.lib()
    f = L.mcpi_apply_h_static
    f.restype = ct.c_int
    f.argtypes = [ct.c_int, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_void_p,
                  ct.c_void_p]
    x = torch.zeros(4, dtype=torch.complex128, device="cuda")   # never touched
    y = torch.zeros(4, dtype=torch.complex128, device="cuda")
    rc = f(16, 10, Ho.ctypes.data, Hint.ctypes.data, mc.VARIANT_MAPS, x.data_ptr(), y.data_ptr(), None)
    assert rc == 2   # MCPI_ERR_RANGE
    rc = f(3, 11, np.zeros(121, np.complex128).ctypes.data, np.zeros(11 ** 4, np.complex128).ctypes.data,
           mc.VARIANT_MAPS, x.data_ptr(), y.data_ptr(), None)
    assert rc == 2   # M beyond the static path's limit


def test_static_folds_the_same_pair_matrix():
    # both paths fold the integrals with one shared routine: with the regular
    # space held to the same kernels the two results agree bit for bit
    for N, M, variant in [(8, 8, mc.VARIANT_MAPS), (7, 6, mc.VARIANT_HASH)]:
        C, Ho, Hint = mc.random_problem(N, M, 75)
        for _ in range(2):
            rc, got = _static(N, M, Ho, Hint, C, variant)
            assert rc == 0
            assert np.array_equal(got, _regular(N, M, Ho, Hint, C, variant, same_kernels=True)), (N, M)


def test_static_refuses_stream_capture():
    # a call on a capturing stream returns MCPI_ERR_ARG with nothing enqueued,
    # and the caller's graph still captures and replays
    N, M = 6, 5
    C, Ho, Hint = mc.random_problem(N, M, 76)
    rc, ref = _static(N, M, Ho, Hint, C)
    assert rc == 0
    f = mc.lib().mcpi_apply_h_static
    Ho = np.ascontiguousarray(Ho, np.complex128)
    Hint = np.ascontiguousarray(Hint, np.complex128)
    x = torch.from_numpy(np.ascontiguousarray(C, np.complex128)).cuda()
    out = torch.zeros_like(x)
    y = torch.zeros(16, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        y.add_(1.0)
        rc = f(N, M, Ho.ctypes.data, Hint.ctypes.data, mc.VARIANT_MAPS, x.data_ptr(), out.data_ptr(),
               ct.c_void_p(torch.cuda.current_stream().cuda_stream))
        y.add_(1.0)
    assert rc == 1   # MCPI_ERR_ARG
    g.replay()
    torch.cuda.synchronize()
    assert torch.all(y == 2.0).item()
    assert torch.count_nonzero(out).item() == 0          # nothing of the refused call ran
    rc, again = _static(N, M, Ho, Hint, C)               # outside the capture it works again
    assert rc == 0 and np.array_equal(again, ref)
    del g
