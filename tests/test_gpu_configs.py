"""Parity at the sizes of the benchmark configurations.

* N=16, M=10 Lieb-Liniger (nc = 2,042,975), 150 Lanczos steps: alpha, beta,
  E0 and the ground state's occupations against the oracle's run of the
  reference recurrence (groundStateLieb.c:217-471 with applyHconf_X,
  hamiltonianMatrix.h:431-887), fixture tests/golden/lanczos_c1.npz.
* The 64-solve batched sweep: every member whose int32 maps fit the reference
  (45 of 64) against the oracle's ground state with applyHconf_XX,
  fixture tests/golden/sweep_c2.npz.
* N=10, M=10 (nc = 92,378): rho1 and rho2 against the reference's own
  OBrho_XM and TBrho_XX, fixture tests/golden/c0_densities.npz.
* N=20, M=10 (nc = 10,015,005): the transition densities of two random
  states with the ket restricted to sampled row ranges, entry by entry (all
  M^2 and M^4 of them) against the oracle's definition summed over the same
  rows; rho1 and rho2 of one state against the transition densities of the
  state with itself.

Bars: alpha, beta within 1e-10 of max |alpha|; E0 within 1e-10 relative to
max(1, |E0|); densities within 1e-12 relative Frobenius error.
"""
import os

import numpy as np
import pytest
import torch

import mcpi_b200 as mc
import oracle
from conftest import GOLDEN, rel

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _start(nc, seed):
    rng = np.random.default_rng(seed)
    C = rng.standard_normal(nc) + 1j * rng.standard_normal(nc)
    return C / np.linalg.norm(C)


def test_c1_lanczos_against_oracle():
    f = np.load(os.path.join(GOLDEN, "lanczos_c1.npz"))
    N, M, g, lm = int(f["N"]), int(f["M"]), float(f["g"]), int(f["steps"])
    sp = mc.FockSpace(N, M)
    sp.set_integrals(*mc.lieb_integrals(M, g, float(f["L"])))
    C0 = _start(sp.nc, int(f["start_seed"]))
    it, diag, off, lvec = sp.lanczos(C0, lm)
    del lvec
    assert it == lm
    scale = np.abs(f["alpha"]).max()
    assert np.abs(diag.real - f["alpha"]).max() <= 1e-10 * scale
    assert np.abs(off[: lm - 1] - f["beta"]).max() <= 1e-10 * scale
    E, psi, it2 = sp.ground(C0, lm)
    E0 = float(f["E0"])
    assert it2 == lm
    assert abs(E - E0) <= 1e-10 * max(1.0, abs(E0)), (E, E0)
    r1 = sp.rho1(psi).cpu().numpy()
    occ = r1.diagonal().real / torch.linalg.vector_norm(psi).item() ** 2
    assert np.abs(occ - f["occupations"]).max() <= 1e-8
    sp.close()


def test_c2_sweep_members_against_oracle():
    f = np.load(os.path.join(GOLDEN, "sweep_c2.npz"))
    members = [(int(n), int(m)) for n, m in zip(f["N"], f["M"])]
    steps = int(f["steps"])
    b = mc.Batch(members, steps)
    for k, ((n, m), g) in enumerate(zip(members, f["g"])):
        b.set_integrals(k, *mc.lieb_integrals(m, float(g)))
        b.set_start(k, _start(b.nc[k], int(f["start_seed_base"]) + k))
    E, it = b.run()
    b.close()
    pick = f["pick"]
    assert len(pick) >= 4
    for k, E0 in zip(pick, f["E0"]):
        assert abs(E[k] - E0) <= 1e-10 * max(1.0, abs(E0)), (int(k), E[k], E0)


def test_c0_densities_against_reference():
    f = np.load(os.path.join(GOLDEN, "c0_densities.npz"))
    N, M = int(f["N"]), int(f["M"])
    C = oracle.random_inputs(N, M, int(f["seed"]))[0]
    assert np.array_equal(C[:8], f["C_head"]) and C.sum() == f["C_sum"]   # same generator
    sp = mc.FockSpace(N, M)
    assert rel(sp.rho1(C).cpu().numpy(), f["rho1"]) <= TOL
    assert rel(sp.rho2(C).cpu().numpy(), f["rho2"]) <= TOL
    assert rel(sp.trans_rho2(C, C).cpu().numpy(), f["rho2"]) <= TOL
    sp.close()


def test_c4_transition_densities_row_sampled(orc):
    N, M = 20, 10
    nc = mc.nc_of(N, M)
    phi, psi = _start(nc, 41), _start(nc, 42)
    w = 3000
    ranges = [(0, w), (nc // 4, nc // 4 + w), (nc // 2, nc // 2 + w), (nc - w, nc)]
    psi_s = np.zeros_like(psi)
    for a, b in ranges:
        psi_s[a:b] = psi[a:b]
    want1 = sum(orc.density_rows(N, M, 1, phi, psi, a, b) for a, b in ranges)
    want2 = sum(orc.density_rows(N, M, 2, phi, psi, a, b) for a, b in ranges)
    sp = mc.FockSpace(N, M)
    x, y = torch.from_numpy(phi).cuda(), torch.from_numpy(psi_s).cuda()
    t1 = sp.trans_rho1(x, y).cpu().numpy()
    t2 = sp.trans_rho2(x, y).cpu().numpy()
    assert rel(t1, want1.reshape(M, M).T) <= TOL
    assert rel(t2, want2) <= TOL
    assert np.count_nonzero(np.abs(want2) > 0) > 0.9 * M ** 4     # the sample reaches the entries
    # one state: the Hermitian-half kernels against the full transition reduction
    z = torch.from_numpy(psi).cuda()
    assert rel(sp.rho1(z).cpu().numpy(), sp.trans_rho1(z, z).cpu().numpy()) <= TOL
    assert rel(sp.rho2(z).cpu().numpy(), sp.trans_rho2(z, z).cpu().numpy()) <= TOL
    sp.close()
