"""The C ABI without a GPU: the library loads, exports every symbol its headers
declare, and its host-only entry points agree with the reference's outputs."""
import ctypes as ct
import os
import re

import numpy as np
import pytest

import mcpi_b200 as mc
from conftest import ROOT

HEADERS = [os.path.join(ROOT, "include", h) for h in os.listdir(os.path.join(ROOT, "include"))
           if h.endswith(".h")]


def _declared(path):
    text = open(path).read()
    return set(re.findall(r"^(?:MCPI_API|MCPI_DROPIN_API)\s+[\w\s\*]*?\b(\w+)\s*\(", text,
                          flags=re.M))


def _lib_for(header):
    name = os.path.basename(header)
    return {"mcpi_b200.h": mc.LIB_PATH,
            "mcpi_dropin.h": os.path.join(ROOT, "mcpi_b200", "libmcpi_dropin.so")}[name]


@pytest.mark.parametrize("header", HEADERS, ids=os.path.basename)
def test_library_exports_declared_symbols(header):
    syms = _declared(header)
    assert syms, f"no MCPI_API declarations parsed from {header}"
    lib = ct.CDLL(_lib_for(header))
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_nc_and_ncmat(golden_tables):
    assert mc.nc_of(16, 10) == 2042975 and mc.nc_of(20, 10) == 10015005 and mc.nc_of(10, 10) == 92378
    for k in golden_tables:
        if k.startswith("NCmat_"):
            N, M = map(int, k.split("_")[1:])
            assert np.array_equal(mc.setupNCmat(N, M), golden_tables[k])


def test_index_fock_host(golden_tables):
    for k in golden_tables:
        if k.startswith("IF_"):
            N, M = map(int, k.split("_")[1:])
            IF = golden_tables[k].reshape(-1, M)
            for i, v in enumerate(IF):
                assert np.array_equal(mc.IndexToFock(i, N, M), v)
                assert mc.FockToIndex(N, M, v) == i
    with pytest.raises(mc.MCPIError):
        mc.FockToIndex(3, 3, [1, 1, 0])       # does not hold N particles
    with pytest.raises(mc.MCPIError):
        mc.IndexToFock(10, 3, 3)              # index beyond NC(3,3)


def test_tridiag_eig_against_scipy():
    from scipy.linalg import eigh_tridiagonal
    rng = np.random.default_rng(0)
    for n in [1, 2, 3, 17, 150, 400]:
        d = rng.standard_normal(n) * 10
        e = rng.standard_normal(max(n - 1, 1))
        w, z = mc.tridiag_eig(d, e)
        if n > 1:
            ws = eigh_tridiagonal(d, e[: n - 1], eigvals_only=True)
            assert np.allclose(w, ws, rtol=0, atol=1e-11 * max(1, np.abs(ws).max()))
            T = np.diag(d) + np.diag(e[: n - 1], 1) + np.diag(e[: n - 1], -1)
            assert np.linalg.norm(T @ z - z * w) < 1e-11 * np.abs(w).max() * n
            assert np.allclose(z.T @ z, np.eye(n), atol=1e-12)
        else:
            assert w[0] == d[0]
    # zero couplings and repeated eigenvalues
    w, z = mc.tridiag_eig(np.array([2.0, 2.0, -1.0]), np.array([0.0, 0.0]))
    assert np.array_equal(w, [-1.0, 2.0, 2.0])


def test_lieb_integrals_match_reference(orc):
    for M, g in [(10, 1.0), (11, 100.0), (7, 0.01)]:
        Ho, Hint = mc.lieb_integrals(M, g)
        Ho2, Hint2 = orc.lieb(M, g)
        assert np.array_equal(Ho, Ho2) and np.array_equal(Hint, Hint2)


def test_hint_symmetrisation():
    M = 4
    h = mc.symmetrize_hint(np.random.default_rng(1).standard_normal(M ** 4) * (1 + 1j), M)
    H = h.reshape(M, M, M, M)   # axes (l, q, s, k)
    for k, s, q, l in np.ndindex(M, M, M, M):
        v = H[l, q, s, k]
        assert np.isclose(v, H[l, q, k, s]) and np.isclose(v, H[q, l, s, k])
        assert np.isclose(v, np.conj(H[s, k, l, q]))


def test_no_cpu_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(mc.MCPIError):
        mc.FockSpace(4, 4)
