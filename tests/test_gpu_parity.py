"""Parity of the CUDA path with the reference (golden fixtures) and the oracle.

Bars: tables bit-exact; H.psi, rho1, rho2 and the transition densities within
1e-12 relative Frobenius error of the reference's FP64 CPU routines; Lanczos
E0 within 1e-10 (relative to max(1,|E0|)).
"""
import numpy as np
import pytest
import torch

import mcpi_b200 as mc
import oracle
from conftest import case_keys, rel

pytestmark = pytest.mark.gpu
TOL = 1e-12
TABLE_NAMES = ["IF", "Map", "MapOT", "strideOT", "MapTT", "strideTT"]


def _space(N, M):
    return mc.FockSpace(N, M, device=0)


# ---------------------------------------------------------------- tables ----

def test_tables_bit_exact_golden(golden_tables):
    cases = sorted({tuple(map(int, k.split("_")[1:])) for k in golden_tables if k.startswith("IF_")})
    for N, M in cases:
        sp = _space(N, M)
        g = {n: golden_tables[f"{n}_{N}_{M}"] for n in TABLE_NAMES}
        assert np.array_equal(sp.focks().cpu().numpy(), g["IF"]), (N, M)
        assert np.array_equal(sp.one_one_map().cpu().numpy(), g["Map"]), (N, M)
        m, s = sp.two_map(False)
        assert np.array_equal(m.cpu().numpy(), g["MapOT"]) and np.array_equal(s.cpu().numpy(), g["strideOT"])
        m, s = sp.two_map(True)
        assert np.array_equal(m.cpu().numpy(), g["MapTT"]) and np.array_equal(s.cpu().numpy(), g["strideTT"])
        sp.close()


@pytest.mark.parametrize("N,M", [(10, 6), (8, 8), (10, 10), (6, 13)])
def test_tables_bit_exact_oracle(orc, N, M):
    sp = _space(N, M)
    IF = orc.focks(N, M)
    assert np.array_equal(sp.focks().cpu().numpy(), IF)
    assert np.array_equal(sp.one_one_map().cpu().numpy(), orc.one_one_map(N, M, IF))
    mo, so = orc.one_two_map(N, M, IF)
    m, s = sp.two_map(False)
    assert np.array_equal(m.cpu().numpy(), mo) and np.array_equal(s.cpu().numpy(), so)
    mo, so = orc.two_two_map(N, M, IF)
    m, s = sp.two_map(True)
    assert np.array_equal(m.cpu().numpy(), mo) and np.array_equal(s.cpu().numpy(), so)


# ----------------------------------------------------------------- H.psi ----

def test_hpsi_golden(golden_ops):
    for kind, N, M in case_keys(golden_ops, "hxx"):
        key = f"{kind}_{N}_{M}"
        C, Ho, Hint = golden_ops[f"C_{key}"], golden_ops[f"Ho_{key}"], golden_ops[f"Hint_{key}"]
        sp = _space(N, M)
        sp.set_integrals(Ho, Hint, mc.VARIANT_MAPS)
        assert rel(sp.apply_h(C).cpu().numpy(), golden_ops[f"hxx_{key}"]) <= TOL, key
        sp.set_integrals(Ho, Hint, mc.VARIANT_HASH)
        assert rel(sp.apply_h(C).cpu().numpy(), golden_ops[f"hplain_{key}"]) <= TOL, key
        sp.close()


@pytest.mark.parametrize("N,M,seed", [(10, 10, 0), (6, 8, 1), (9, 5, 2), (4, 16, 3), (12, 4, 4)])
def test_hpsi_random_oracle(orc, N, M, seed):
    C, Ho, Hint = mc.random_problem(N, M, seed)
    sp = _space(N, M)
    sp.set_integrals(Ho, Hint)
    out = sp.apply_h(C).cpu().numpy()
    assert rel(out, orc.apply_h(N, M, C, Ho, Hint, mode=2)) <= TOL


@pytest.mark.parametrize("N,M", [(6, 5), (5, 7)])
def test_hpsi_unsymmetric_hint_follows_each_variant(orc, N, M):
    # Without the 8-fold symmetry the reference variants disagree with each
    # other; the device path must reproduce whichever one it is asked for.
    rng = np.random.default_rng(11)
    C, Ho, _ = mc.random_problem(N, M, 5)
    Ho = Ho + 0.2j * rng.standard_normal((M, M))            # not Hermitian either
    Hint = rng.standard_normal(M ** 4) + 1j * rng.standard_normal(M ** 4)
    sp = _space(N, M)
    sp.set_integrals(Ho, Hint, mc.VARIANT_MAPS)
    assert rel(sp.apply_h(C).cpu().numpy(), orc.apply_h(N, M, C, Ho, Hint, mode=2)) <= TOL
    sp.set_integrals(Ho, Hint, mc.VARIANT_HASH)
    assert rel(sp.apply_h(C).cpu().numpy(), orc.apply_h(N, M, C, Ho, Hint, mode=0)) <= TOL


@pytest.mark.parametrize("N,M", [(0, 4), (1, 1), (1, 6), (2, 1), (2, 5), (3, 2), (7, 1), (5, 16)])
def test_hpsi_edge_sizes(orc, N, M):
    C, Ho, Hint = mc.random_problem(N, M, 9)
    sp = _space(N, M)
    sp.set_integrals(Ho, Hint)
    out = sp.apply_h(C).cpu().numpy()
    ref = orc.apply_h(N, M, C, Ho, Hint, mode=2)
    assert rel(out, ref) <= TOL, (N, M)


def test_hpsi_lieb(orc):
    N, M = 8, 9
    Ho, Hint = mc.lieb_integrals(M, 2.5)
    C = orc.perf_inputs(N, M)[0]
    sp = _space(N, M)
    sp.set_integrals(Ho, Hint)
    assert rel(sp.apply_h(C).cpu().numpy(), orc.apply_h(N, M, C, Ho, Hint, mode=2)) <= TOL


def test_adjoint():
    N, M = 6, 6
    rng = np.random.default_rng(2)
    C, Ho, Hint = mc.random_problem(N, M, 3)
    Hint = Hint + 0.1 * (rng.standard_normal(M ** 4) + 1j * rng.standard_normal(M ** 4))
    Ho = Ho + 0.1j * rng.standard_normal((M, M))
    phi = mc.random_problem(N, M, 4)[0]
    sp = _space(N, M)
    sp.set_integrals(Ho, Hint)
    lhs = np.vdot(phi, sp.apply_h(C).cpu().numpy())
    rhs = np.vdot(sp.apply_h_adjoint(phi).cpu().numpy(), C)
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


# ------------------------------------------------------------- densities ----

def test_densities_golden(golden_ops):
    for kind, N, M in case_keys(golden_ops, "rho1"):
        key = f"{kind}_{N}_{M}"
        C = golden_ops[f"C_{key}"]
        sp = _space(N, M)
        assert rel(sp.rho1(C).cpu().numpy(), golden_ops[f"rho1_{key}"]) <= TOL, key
        assert rel(sp.rho2(C).cpu().numpy(), golden_ops[f"rho2_{key}"]) <= TOL, key
        sp.close()


@pytest.mark.parametrize("N,M", [(10, 10), (7, 11), (3, 16), (1, 5), (0, 3), (5, 12), (2, 12), (2, 9), (20, 3),
                                 (30, 2), (6, 13)])
def test_densities_oracle(orc, N, M):
    C = mc.random_problem(N, M, 21)[0]
    sp = _space(N, M)
    r1 = sp.rho1(C).cpu().numpy()
    assert rel(r1, orc.obrho(N, M, C)) <= TOL
    assert abs(np.trace(r1) - N) <= 1e-12 * max(N, 1)
    r2 = sp.rho2(C).cpu().numpy()
    assert rel(r2, orc.density_rows(N, M, 2, C, C, 0, orc.nc(N, M))) <= TOL
    R = r2.reshape(M, M, M, M)          # axes (l, q, s, k)
    tr = sum(R[k, s, s, k] for k in range(M) for s in range(M))   # sum <a+_k a+_s a_s a_k>
    assert abs(tr - N * (N - 1)) <= 1e-12 * max(1, N * N)


@pytest.mark.parametrize("N,M", [(5, 5), (6, 7), (2, 4), (8, 10), (9, 9), (2, 10), (4, 11), (3, 12)])
def test_transition_densities(orc, N, M):
    # M <= 10: FP64 tensor-core Gram; larger M: the CUDA-core Gram
    phi = mc.random_problem(N, M, 31)[0]
    psi = mc.random_problem(N, M, 32)[0]
    sp = _space(N, M)
    nc = orc.nc(N, M)
    t1 = sp.trans_rho1(phi, psi).cpu().numpy()
    o1 = orc.density_rows(N, M, 1, phi, psi, 0, nc).reshape(M, M).T      # oracle flat k + l*M
    assert rel(t1, o1) <= TOL
    t2 = sp.trans_rho2(phi, psi).cpu().numpy()
    assert rel(t2, orc.density_rows(N, M, 2, phi, psi, 0, nc)) <= TOL


def test_gram_wait_timeout_is_reported(orc):
    # the tensor-core Gram kernel's waits are bounded: with its gather warps held
    # back by the test switch the product warps give up after the (shortened)
    # limit, the next synchronisation reports MCPI_ERR_TIMEOUT, and the space
    # keeps working afterwards
    N, M = 8, 10
    C = mc.random_problem(N, M, 79)[0]
    sp = _space(N, M)
    sp.set_option(mc.OPT_WAIT_LIMIT_KCYCLES, 1000)
    sp.set_option(mc.OPT_TEST_STALL_GATHER, 1)
    sp.rho2(C)
    with pytest.raises(mc.MCPIError) as err:
        sp.sync()
    assert err.value.status == 7      # MCPI_ERR_TIMEOUT
    sp.set_option(mc.OPT_TEST_STALL_GATHER, 0)
    r2 = sp.rho2(C).cpu().numpy()
    sp.sync()
    assert rel(r2, orc.density_rows(N, M, 2, C, C, 0, orc.nc(N, M))) <= TOL
    sp.close()


def test_energy_identity_device():
    N, M = 7, 8
    C, Ho, Hint = mc.random_problem(N, M, 41)
    sp = _space(N, M)
    sp.set_integrals(Ho, Hint)
    e1 = np.vdot(C, sp.apply_h(C).cpu().numpy())
    e2 = np.sum(Ho * sp.rho1(C).cpu().numpy()) + 0.5 * np.sum(Hint * sp.rho2(C).cpu().numpy())
    assert abs(e1 - e2) <= 1e-12 * abs(e1)


# ---------------------------------------------------------------- Lanczos ----

def test_lanczos_coefficients(orc):
    N, M, lm = 6, 6, 30
    Ho, Hint = mc.lieb_integrals(M, 4.0)
    C0 = orc.perf_inputs(N, M)[0]
    sp = _space(N, M)
    sp.set_integrals(Ho, Hint)
    it, diag, off, _ = sp.lanczos(C0, lm)
    ito, diago, offo, _ = orc.lanczos(N, M, Ho, Hint, C0, lm, mode=2)
    assert it == ito == lm
    scale = np.abs(diago).max()
    assert np.abs(diag[:it] - diago[:it]).max() <= 1e-10 * scale
    assert np.abs(off[: it - 1] - offo[: it - 1].real).max() <= 1e-10 * scale


def test_ground_lieb_known_answers(orc, golden_lieb):
    N, M, niter = int(golden_lieb["N"]), int(golden_lieb["M"]), int(golden_lieb["niter"])
    C0 = orc.perf_inputs(N, M)[0]
    pub = dict(zip(golden_lieb["published_g"], golden_lieb["published_E0_per_N"]))
    sp = _space(N, M)
    for g, Eref in zip(golden_lieb["g"], golden_lieb["E0"]):
        Ho, Hint = mc.lieb_integrals(M, g)
        sp.set_integrals(Ho, Hint)
        E, psi, it = sp.ground(C0, niter)
        assert it == niter
        assert abs(E - Eref) <= 1e-10 * max(1.0, abs(Eref)), (g, E, Eref)
        assert round(E / N, 5) == pytest.approx(pub[g], abs=1e-5)
        # the Ritz vector is an eigenvector
        hpsi = sp.apply_h(psi)
        res = torch.linalg.vector_norm(hpsi - E * psi).item() / torch.linalg.vector_norm(psi).item()
        assert res < 1e-6 * abs(E)


def test_ground_random_against_oracle(orc):
    N, M, niter = 7, 6, 60
    C0, Ho, Hint = mc.random_problem(N, M, 51)
    sp = _space(N, M)
    sp.set_integrals(Ho, Hint)
    E, psi, it = sp.ground(C0, niter)
    Eo, psio, ito = orc.ground(N, M, Ho, Hint, C0, niter, mode=2)
    assert it == ito
    assert abs(E - Eo) <= 1e-10 * max(1.0, abs(Eo))
    ov = abs(np.vdot(psi.cpu().numpy(), psio)) / (np.linalg.norm(psio) ** 2)
    assert abs(ov - 1) < 1e-8


def test_lanczos_breakdown():
    # all particles in one plane wave of a non-interacting ring: the start
    # vector is an eigenvector, beta_0 = 0 and the solve stops at once
    N, M = 4, 5
    Ho, Hint = mc.lieb_integrals(M, 0.0)
    C0 = np.zeros(mc.nc_of(N, M), np.complex128)
    C0[mc.FockToIndex(N, M, [0, 0, 4, 0, 0])] = 1.0
    sp = _space(N, M)
    sp.set_integrals(Ho, Hint)
    it, diag, off, _ = sp.lanczos(C0, 10)
    assert it == 0
    E, psi, it2 = sp.ground(C0, 10)
    assert it2 == 0 and E == pytest.approx(diag[0].real)


@pytest.mark.parametrize("N,M,g", [(8, 9, 2.5), (6, 11, 0.7), (5, 16, 1.0), (9, 7, 30.0)])
def test_block_and_dense_pair_kernels_agree(orc, N, M, g):
    # plane-wave integrals conserve momentum, so the pair matrix splits into
    # one block per total momentum and the block-sparse kernel is used
    Ho, Hint = mc.lieb_integrals(M, g)
    C = mc.random_problem(N, M, 61)[0]
    sp = _space(N, M)
    sp.set_option(mc.OPT_DIRECT_HPSI, 0)
    sp.set_integrals(Ho, Hint)
    fast = sp.apply_h(C).cpu().numpy()                 # momentum-block pair kernels
    sp.set_option(mc.OPT_DIRECT_HPSI, 1)
    direct = sp.apply_h(C).cpu().numpy()               # direct kernel
    assert rel(direct, orc.apply_h(N, M, C, Ho, Hint, mode=2)) <= TOL
    sp.set_momentum_kernel(False)
    sp.set_integrals(Ho, Hint)
    blocks = sp.apply_h(C).cpu().numpy()               # generic block-sparse kernel
    sp.set_dense_pair_kernel(True)
    sp.set_integrals(Ho, Hint)
    dense = sp.apply_h(C).cpu().numpy()
    ref = orc.apply_h(N, M, C, Ho, Hint, mode=2)
    assert rel(fast, ref) <= TOL and rel(blocks, ref) <= TOL and rel(dense, ref) <= TOL
    assert rel(sp.apply_h_adjoint(C).cpu().numpy(), ref) <= TOL    # Hermitian here


@pytest.mark.parametrize("N,M", [(2, 2), (2, 7), (3, 12), (5, 11), (7, 9), (10, 10), (6, 12), (12, 4)])
def test_gemm_and_csr_pair_kernels_agree(orc, N, M):
    # general (random) integrals: the dense-product kernel by default, the
    # compressed-row kernel with MCPI_OPT_NO_GEMM_KERNEL; N=2 has one
    # (N-2)-configuration, N=10 M=10 more tiles than the persistent grid
    C, Ho, Hint = mc.random_problem(N, M, 71)
    ref = orc.apply_h(N, M, C, Ho, Hint, mode=2)
    sp = _space(N, M)
    sp.set_integrals(Ho, Hint)
    gemm = sp.apply_h(C).cpu().numpy()
    adj = sp.apply_h_adjoint(C).cpu().numpy()
    sp.set_option(4, 1)
    sp.set_integrals(Ho, Hint)
    csr = sp.apply_h(C).cpu().numpy()
    assert rel(gemm, ref) <= TOL and rel(csr, ref) <= TOL and rel(adj, ref) <= TOL
    sp.set_option(4, 0)
    sp.set_dense_pair_kernel(True)           # the dense product also for sparse (Lieb) integrals
    Ho2, Hint2 = mc.lieb_integrals(M, 1.5)
    sp.set_integrals(Ho2, Hint2)
    assert rel(sp.apply_h(C).cpu().numpy(), orc.apply_h(N, M, C, Ho2, Hint2, mode=2)) <= TOL


def test_apply_h_host_pipeline(orc):
    # host-buffer pipeline: numpy and pinned torch states, repeated states, an
    # odd count (the two device buffer pairs alternate), against the oracle
    import torch
    N, M = 7, 8
    sp = _space(N, M)
    _, Ho, Hint = mc.random_problem(N, M, 31)
    sp.set_integrals(Ho, Hint)
    states = [mc.random_problem(N, M, 40 + k)[0] for k in range(3)]
    refs = [orc.apply_h(N, M, C, Ho, Hint, mode=2) for C in states]
    order = [0, 1, 2, 1, 0]
    ins = [states[k] for k in order[:3]] + [torch.from_numpy(states[k]).pin_memory() for k in order[3:]]
    outs = [np.zeros(sp.nc, np.complex128) for _ in range(3)] + \
           [torch.zeros(sp.nc, dtype=torch.complex128).pin_memory() for _ in range(2)]
    sp.apply_h_host(ins, outs)
    for k, o in zip(order, outs):
        o = o.numpy() if hasattr(o, "numpy") else o
        assert rel(o, refs[k]) <= TOL
    assert sp.apply_h_host([], []) == []
    sp.close()


def test_dense_product_wait_timeout_is_reported(orc):
    # the warp-specialised dense-product kernel's waits are bounded: with its
    # gather warps held back by the test switch, its product warps give up
    # after the (shortened) limit, the next synchronisation reports
    # MCPI_ERR_TIMEOUT, and the space keeps working afterwards
    N, M = 8, 8
    C, Ho, Hint = mc.random_problem(N, M, 77)
    sp = _space(N, M)
    sp.set_integrals(Ho, Hint)
    sp.set_option(5, 1000)            # MCPI_OPT_WAIT_LIMIT_KCYCLES: 1e6 cycles
    sp.set_option(6, 1)               # MCPI_OPT_TEST_STALL_GATHER
    sp.apply_h(C)
    with pytest.raises(mc.MCPIError) as err:
        sp.sync()
    assert err.value.status == 7      # MCPI_ERR_TIMEOUT
    sp.set_option(6, 0)
    out = sp.apply_h(C).cpu().numpy()
    sp.sync()
    assert rel(out, orc.apply_h(N, M, C, Ho, Hint, mode=2)) <= TOL
    sp.close()


@pytest.mark.parametrize("N,M,kind", [(9, 8, "lieb"), (7, 9, "random"), (2, 6, "random"), (6, 11, "lieb")])
def test_occupation_tables_and_decode_agree(orc, N, M, kind):
    # the H.psi kernels read each row's occupations from the packed tables or,
    # without them, decode the row index: the results are bit for bit the same
    C, Ho, Hint = mc.random_problem(N, M, 88)
    if kind == "lieb":
        Ho, Hint = mc.lieb_integrals(M, 3.0)
    sp = _space(N, M)
    sp.set_integrals(Ho, Hint)
    with_tables = sp.apply_h(C).cpu().numpy()
    r1_tables = sp.rho1(C).cpu().numpy()         # (N-1)-space table, built by this first call
    sp.set_option(7, 1)               # MCPI_OPT_NO_OCC_TABLES
    sp.set_integrals(Ho, Hint)
    decoded = sp.apply_h(C).cpu().numpy()
    assert np.array_equal(with_tables, decoded)
    assert np.array_equal(r1_tables, sp.rho1(C).cpu().numpy())
    assert rel(decoded, orc.apply_h(N, M, C, Ho, Hint, mode=2)) <= TOL
    sp.close()
