"""The reference-named drop-in library (include/mcpi_dropin.h, libmcpi_dropin.so).

CPU tests cover the host-only entry points; GPU tests call the table builders
and operators through the reference's signatures (Cmatrix row pointers and all)
and run the reference's own drivers, compiled unmodified against the drop-in
headers (oracle/Makefile, target `dropin`)."""
import ctypes as ct
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, rel

LIB = os.path.join(ROOT, "mcpi_b200", "libmcpi_dropin.so")
DRIVERS = os.path.join(ROOT, "oracle", "_ref")
_vp = ct.c_void_p


@pytest.fixture(scope="module")
def dl():
    L = ct.CDLL(LIB)
    L.NC.restype = ct.c_int
    L.NC.argtypes = [ct.c_int, ct.c_int]
    for n in ("setupNCmat", "setupFocks"):
        getattr(L, n).restype = ct.POINTER(ct.c_int)
        getattr(L, n).argtypes = [ct.c_int, ct.c_int]
    L.FockToIndex.restype = ct.c_int
    L.FockToIndex.argtypes = [ct.c_int, ct.c_int, _vp, _vp]
    L.IndexToFock.argtypes = [ct.c_int, ct.c_int, ct.c_int, _vp]
    L.LAPACKE_dstev.restype = ct.c_int
    L.LAPACKE_dstev.argtypes = [ct.c_int, ct.c_char, ct.c_int, _vp, _vp, _vp, ct.c_int]
    L.OneOneMap.restype = ct.POINTER(ct.c_int)
    L.OneOneMap.argtypes = [ct.c_int, ct.c_int, _vp, _vp]
    for n in ("OneTwoMap", "TwoTwoMap"):
        getattr(L, n).restype = ct.POINTER(ct.c_int)
        getattr(L, n).argtypes = [ct.c_int, ct.c_int, _vp, _vp, _vp]
    L.applyHconf_XX.argtypes = [ct.c_int, ct.c_int] + [_vp] * 10
    L.applyHconf.argtypes = [ct.c_int, ct.c_int] + [_vp] * 6
    L.OBrho_XM.argtypes = [ct.c_int, ct.c_int] + [_vp] * 5
    L.TBrho_XX.argtypes = [ct.c_int, ct.c_int] + [_vp] * 9
    libc = ct.CDLL(None)
    libc.free.argtypes = [_vp]
    L.libc = libc
    return L


def _take(L, p, n):
    a = np.ctypeslib.as_array(p, shape=(n,)).copy() if n else np.zeros(0, np.int32)
    L.libc.free(ct.cast(p, _vp))
    return a


def _rows(mat):
    mat = np.ascontiguousarray(mat, np.complex128)
    return mat, (_vp * mat.shape[0])(*[mat[i].ctypes.data for i in range(mat.shape[0])])


def test_host_entry_points(dl, golden_tables):
    assert dl.NC(16, 10) == 2042975
    for k in golden_tables:
        if k.startswith("NCmat_"):
            N, M = map(int, k.split("_")[1:])
            assert np.array_equal(_take(dl, dl.setupNCmat(N, M), (N + 1) * (M + 1)), golden_tables[k])
        if k.startswith("IF_"):
            N, M = map(int, k.split("_")[1:])
            IF = golden_tables[k].reshape(-1, M)
            v = np.zeros(M, np.int32)
            for i in range(IF.shape[0]):
                dl.IndexToFock(i, N, M, v.ctypes.data)
                assert np.array_equal(v, IF[i])
                assert dl.FockToIndex(N, M, None, np.ascontiguousarray(IF[i]).ctypes.data) == i


def test_lapacke_dstev(dl):
    from scipy.linalg import eigh_tridiagonal
    rng = np.random.default_rng(5)
    n = 40
    d, e = rng.standard_normal(n), rng.standard_normal(n)
    dd, ee, z = d.copy(), e.copy(), np.zeros((n, n))
    assert dl.LAPACKE_dstev(101, b"V", n, dd.ctypes.data, ee.ctypes.data, z.ctypes.data, n) == 0
    assert np.allclose(dd, eigh_tridiagonal(d, e[: n - 1], eigvals_only=True), atol=1e-12)
    T = np.diag(d) + np.diag(e[: n - 1], 1) + np.diag(e[: n - 1], -1)
    assert np.allclose(T @ z, z * dd, atol=1e-10)


@pytest.mark.gpu
def test_tables_and_operators(dl, golden_tables, golden_ops):
    N, M = 6, 5
    nc = dl.NC(N, M)
    IF = _take(dl, dl.setupFocks(N, M), nc * M)
    assert np.array_equal(IF, golden_tables[f"IF_{N}_{M}"])
    assert np.array_equal(_take(dl, dl.OneOneMap(N, M, None, None), nc * M * M), golden_tables[f"Map_{N}_{M}"])
    for name, key in (("OneTwoMap", "OT"), ("TwoTwoMap", "TT")):
        stride = np.zeros(nc, np.int32)
        size = golden_tables[f"Map{key}_{N}_{M}"].size
        m = _take(dl, getattr(dl, name)(N, M, None, None, stride.ctypes.data), size)
        assert np.array_equal(m, golden_tables[f"Map{key}_{N}_{M}"])
        assert np.array_equal(stride, golden_tables[f"stride{key}_{N}_{M}"])
    for kind in ("perf", "rand"):
        key = f"{kind}_{N}_{M}"
        C, Hint = golden_ops[f"C_{key}"], golden_ops[f"Hint_{key}"]
        hm, hp = _rows(golden_ops[f"Ho_{key}"])
        out = np.zeros(nc, np.complex128)
        dl.applyHconf_XX(N, M, None, None, None, None, None, None, C.ctypes.data, hp, Hint.ctypes.data,
                         out.ctypes.data)
        assert rel(out, golden_ops[f"hxx_{key}"]) <= 1e-12
        dl.applyHconf(N, M, None, None, C.ctypes.data, hp, Hint.ctypes.data, out.ctypes.data)
        assert rel(out, golden_ops[f"hplain_{key}"]) <= 1e-12
        rho = np.zeros((M, M), np.complex128)
        rm, rp = _rows(rho)
        dl.OBrho_XM(N, M, None, None, None, C.ctypes.data, rp)
        assert rel(rm, golden_ops[f"rho1_{key}"]) <= 1e-12
        r2 = np.zeros(M ** 4, np.complex128)
        dl.TBrho_XX(N, M, None, None, None, None, None, None, None, C.ctypes.data, r2.ctypes.data)
        assert rel(r2, golden_ops[f"rho2_{key}"]) <= 1e-12


@pytest.mark.gpu
def test_reference_ground_state_driver(golden_lieb):
    """groundStateLieb.c compiled unmodified against the drop-in reproduces the
    published 11-orbital energies of liebGS.dat (N=5, g = 1, 10, 100)."""
    exe = os.path.join(DRIVERS, "groundStateLieb_dropin")
    if not os.path.exists(exe):
        pytest.skip("drop-in drivers not built (needs the reference sources at build time)")
    pub = dict(zip(golden_lieb["published_g"], golden_lieb["published_E0_per_N"]))
    for g in (1.0, 10.0, 100.0):
        r = subprocess.run([exe, "5", "11", str(g)], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
        m = re.search(r"Eo = ([0-9.]+)", r.stdout)
        assert m and float(m.group(1)) == pytest.approx(pub[g], abs=1e-5), r.stdout[-500:]


@pytest.mark.gpu
def test_reference_benchmark_driver():
    exe = os.path.join(DRIVERS, "performanceTest_dropin")
    if not os.path.exists(exe):
        pytest.skip("drop-in drivers not built (needs the reference sources at build time)")
    r = subprocess.run([exe, "6", "5"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "Done." in r.stdout, r.stdout[-2000:]
    assert "Time to apply H with all mappings" in r.stdout
