"""Pins the oracle (oracle/mcpi_oracle.c) against the reference's own outputs.

Golden fixtures (tests/golden/, made by make_golden.py from the reference
compiled unmodified) are always checked; where oracle/_ref/libmcpi_ref.so is
present the restatement is also compared live against the reference.
No GPU needed.
"""
import os

import numpy as np
import pytest

import oracle
from conftest import GOLDEN, case_keys, rel

TABLE_NAMES = ["NCmat", "IF", "Map", "MapOT", "strideOT", "MapTT", "strideTT"]


def _cases(golden):
    return sorted({tuple(map(int, k.split("_")[1:])) for k in golden if k.startswith("IF_")})


def test_tables_bit_exact(orc, golden_tables):
    for N, M in _cases(golden_tables):
        g = {n: golden_tables[f"{n}_{N}_{M}"] for n in TABLE_NAMES}
        assert np.array_equal(orc.ncmat(N, M), g["NCmat"])
        IF = orc.focks(N, M)
        assert np.array_equal(IF, g["IF"]), (N, M)
        assert np.array_equal(orc.one_one_map(N, M, IF), g["Map"]), (N, M)
        m, s = orc.one_two_map(N, M, IF)
        assert np.array_equal(m, g["MapOT"]) and np.array_equal(s, g["strideOT"]), (N, M)
        m, s = orc.two_two_map(N, M, IF)
        assert np.array_equal(m, g["MapTT"]) and np.array_equal(s, g["strideTT"]), (N, M)


def test_fock_round_trip(orc):
    # demonstrateFockMap.c:131-138: FockToIndex(IF[i]) == i
    for N, M in [(5, 4), (3, 7), (6, 3)]:
        IF = orc.focks(N, M).reshape(-1, M)
        for i, v in enumerate(IF):
            assert orc.fock_to_index(N, M, v) == i
            assert np.array_equal(orc.index_to_fock(i, N, M), v)
    assert np.array_equal(orc.index_to_fock(0, 16, 10), [16] + [0] * 9)
    assert np.array_equal(orc.index_to_fock(orc.nc(16, 10) - 1, 16, 10), [0] * 9 + [16])


def test_hpsi_bit_exact(orc, golden_ops):
    for kind, N, M in case_keys(golden_ops, "hxx"):
        key = f"{kind}_{N}_{M}"
        C, Ho, Hint = golden_ops[f"C_{key}"], golden_ops[f"Ho_{key}"], golden_ops[f"Hint_{key}"]
        IF = orc.focks(N, M)
        Map = orc.one_one_map(N, M, IF)
        MapOT, sOT = orc.one_two_map(N, M, IF)
        MapTT, sTT = orc.two_two_map(N, M, IF)
        maps = (Map, MapOT, sOT, MapTT, sTT)
        assert np.array_equal(orc.apply_h(N, M, C, Ho, Hint, mode=2, IF=IF, maps=maps),
                              golden_ops[f"hxx_{key}"]), key
        assert np.array_equal(orc.apply_h(N, M, C, Ho, Hint, mode=1, IF=IF, maps=maps),
                              golden_ops[f"hxx_{key}"]), key
        assert np.array_equal(orc.apply_h(N, M, C, Ho, Hint, mode=0, IF=IF),
                              golden_ops[f"hplain_{key}"]), key
        # row ranges reproduce the same rows
        half = orc.nc(N, M) // 2
        part = orc.apply_h(N, M, C, Ho, Hint, mode=2, IF=IF, row0=half)
        assert np.array_equal(part[half:], golden_ops[f"hxx_{key}"][half:])


def test_densities(orc, golden_ops):
    for kind, N, M in case_keys(golden_ops, "rho1"):
        key = f"{kind}_{N}_{M}"
        C = golden_ops[f"C_{key}"]
        assert np.array_equal(orc.obrho(N, M, C), golden_ops[f"rho1_{key}"]), key
        assert rel(orc.density(N, M, 1, C, C).reshape(M, M).T, golden_ops[f"rho1_{key}"]) < 1e-14
        assert rel(orc.density(N, M, 2, C, C), golden_ops[f"rho2_{key}"]) < 1e-14, key


def test_generic_operator_matches_folded_rules(orc, golden_ops):
    # Hint with the 8-fold symmetry: every reference variant equals the unfolded operator
    for kind, N, M in case_keys(golden_ops, "hxx"):
        key = f"{kind}_{N}_{M}"
        C, Ho, Hint = golden_ops[f"C_{key}"], golden_ops[f"Ho_{key}"], golden_ops[f"Hint_{key}"]
        g = orc.apply_h_generic(N, M, Ho, Hint, C)
        assert rel(g, golden_ops[f"hxx_{key}"]) < 1e-13, key
        assert rel(g, golden_ops[f"hplain_{key}"]) < 1e-13, key


def test_energy_identity(orc, golden_ops):
    # <psi|H psi> = sum Ho[k][l] rho1[k][l] + 1/2 sum Hint rho2
    for kind, N, M in case_keys(golden_ops, "hxx"):
        key = f"{kind}_{N}_{M}"
        C, Ho, Hint = golden_ops[f"C_{key}"], golden_ops[f"Ho_{key}"], golden_ops[f"Hint_{key}"]
        e1 = np.vdot(C, golden_ops[f"hxx_{key}"])
        e2 = np.sum(Ho * golden_ops[f"rho1_{key}"]) + 0.5 * np.sum(Hint * golden_ops[f"rho2_{key}"])
        assert abs(e1 - e2) <= 1e-12 * max(1.0, abs(e1)), key


def test_lieb_known_answers(orc, golden_lieb):
    N, M, niter = int(golden_lieb["N"]), int(golden_lieb["M"]), int(golden_lieb["niter"])
    C0 = orc.perf_inputs(N, M)[0]
    pub = dict(zip(golden_lieb["published_g"], golden_lieb["published_E0_per_N"]))
    for g, Eref in zip(golden_lieb["g"], golden_lieb["E0"]):
        Ho, Hint = orc.lieb(M, g)
        E, _, it = orc.ground(N, M, Ho, Hint, C0, niter, mode=2)
        assert it == niter
        assert abs(E - Eref) <= 1e-10 * abs(Eref)
        assert round(E / N, 5) == pytest.approx(pub[g], abs=1e-5)


def test_jacobi_dstev_against_scipy(orc):
    from scipy.linalg import eigh_tridiagonal
    import ctypes as ct
    rng = np.random.default_rng(3)
    for n in [1, 2, 7, 60]:
        d = rng.standard_normal(n)
        e = rng.standard_normal(max(n - 1, 1))
        dd, ee = d.copy(), np.append(e[: n - 1], 0.0)
        z = np.zeros((n, n))
        rc = orc.lib.LAPACKE_dstev(101, ct.c_char(b"V"), n, dd.ctypes.data_as(ct.c_void_p),
                                   ee.ctypes.data_as(ct.c_void_p), z.ctypes.data_as(ct.c_void_p), n)
        assert rc == 0
        w, V = eigh_tridiagonal(d, e[: n - 1]) if n > 1 else (d, np.ones((1, 1)))
        assert np.allclose(dd, w, atol=1e-12)
        T = np.diag(d) + (np.diag(e[: n - 1], 1) + np.diag(e[: n - 1], -1) if n > 1 else 0)
        assert np.allclose(T @ z, z * dd, atol=1e-10)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built here")
def test_restatement_against_live_reference(orc):
    R = oracle.Ref()
    for N, M, seed in [(5, 5, 1), (7, 4, 2), (3, 9, 3)]:
        t = R.tables(N, M)
        C, Ho, Hint = oracle.random_inputs(N, M, seed)
        # a Hint WITHOUT the 8-fold symmetry: the folded and plain variants differ,
        # and the restatement must still match each reference variant exactly
        Hint = Hint + 0.3 * np.random.default_rng(seed).standard_normal(M ** 4)
        assert np.array_equal(orc.apply_h(N, M, C, Ho, Hint, mode=2), R.apply_h("XX", N, M, C, Ho, Hint, t))
        assert np.array_equal(orc.apply_h(N, M, C, Ho, Hint, mode=0), R.apply_h("plain", N, M, C, Ho, Hint, t))
        assert np.array_equal(orc.apply_h(N, M, C, Ho, Hint, mode=2),
                              R.apply_h("omp", N, M, C, Ho, Hint, t))


def test_density_rows_add_up(orc):
    # the ket row ranges of orc_density_rows partition the full definition
    N, M = 5, 6
    rng = np.random.default_rng(3)
    nc = orc.nc(N, M)
    phi = rng.standard_normal(nc) + 1j * rng.standard_normal(nc)
    psi = rng.standard_normal(nc) + 1j * rng.standard_normal(nc)
    for order in (1, 2):
        full = orc.density(N, M, order, phi, psi)
        parts = orc.density_rows(N, M, order, phi, psi, 0, 97) + orc.density_rows(N, M, order, phi, psi, 97, nc)
        assert np.abs(full - parts).max() <= 1e-13 * np.abs(full).max()
        cut = psi.copy()
        cut[97:] = 0
        assert np.abs(orc.density(N, M, order, phi, cut) - orc.density_rows(N, M, order, phi, psi, 0, 97)).max() \
            <= 1e-13 * np.abs(full).max()


def test_c0_density_fixture_against_oracle(orc):
    # the reference's TBrho_XX / OBrho_XM at N=10, M=10 (tests/golden/c0_densities.npz)
    # against the oracle's own restatements
    f = np.load(os.path.join(GOLDEN, "c0_densities.npz"))
    N, M = int(f["N"]), int(f["M"])
    C = oracle.random_inputs(N, M, int(f["seed"]))[0]
    assert np.array_equal(C[:8], f["C_head"]) and C.sum() == f["C_sum"]
    assert np.abs(orc.obrho(N, M, C) - f["rho1"]).max() <= 1e-13
    r2 = orc.density_rows(N, M, 2, C, C, 0, orc.nc(N, M))
    assert np.linalg.norm(r2 - f["rho2"]) <= 1e-12 * np.linalg.norm(f["rho2"])


def test_lanczos_fixtures_are_consistent():
    # the configuration-size fixtures' own arithmetic: E0 is the lowest Ritz
    # value of the stored tridiagonal, occupations add up to N, and the sweep
    # members are the draw the batched benchmark makes
    from scipy.linalg import eigh_tridiagonal
    f = np.load(os.path.join(GOLDEN, "lanczos_c1.npz"))
    w = eigh_tridiagonal(f["alpha"], f["beta"], eigvals_only=True)
    assert abs(w[0] - f["E0"]) <= 1e-12 * abs(f["E0"])
    assert abs(f["occupations"].sum() - f["N"]) <= 1e-10
    s = np.load(os.path.join(GOLDEN, "sweep_c2.npz"))
    rng = np.random.default_rng(2024)
    n = rng.integers(6, 15, 64)
    m = rng.choice([7, 9, 11], 64)
    g = 10.0 ** rng.uniform(-2.0, 2.0, 64)
    assert np.array_equal(s["N"], n) and np.array_equal(s["M"], m) and np.array_equal(s["g"], g)
    assert len(s["pick"]) == len(s["E0"]) >= 4
