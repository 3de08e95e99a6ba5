"""Adjoint of psi -> H psi and the transition-density gradients (N=8, M=8).

The loss is L = Re <phi|H|psi> with seeded psi, phi, a random Hermitian Ho
and a random Hint averaged over the bosonic 8-fold group. Gradients from the
autograd wrapper (mcpi_b200/autograd.py, backed by mcpi_apply_h_adjoint and
the transition-density kernels) are checked against central finite
differences with step 1e-6: on random directions in psi, on single entries of
Ho and Hint (representatives the folded rules read and entries they do not),
and on perturbations of whole symmetry orbits of Hint. dE0/dg of the
Lieb-Liniger ground state at g=2 is checked against the Hellmann-Feynman
gradient built from rho2 -- the device's and the reference's own TBrho_XX."""
import numpy as np
import pytest
import torch

import mcpi_b200 as mc
import oracle
from mcpi_b200 import autograd as ag

pytestmark = pytest.mark.gpu
N, M = 8, 8
H_FD = 1e-6


@pytest.fixture(scope="module")
def problem():
    psi, Ho, Hint = mc.random_problem(N, M, 81)
    phi = mc.random_problem(N, M, 82)[0]
    sp = mc.FockSpace(N, M)
    return sp, psi, phi, Ho, Hint


def _loss(sp, psi, phi, Ho, Hint):
    sp.set_integrals(Ho, Hint)
    return float(np.real(np.vdot(phi, sp.apply_h(psi).cpu().numpy())))


def _grads(sp, psi, phi, Ho, Hint):
    tpsi = torch.tensor(psi, device="cuda", requires_grad=True)
    tho = torch.tensor(Ho, requires_grad=True)
    thint = torch.tensor(Hint, requires_grad=True)
    out = ag.apply_h(tpsi, tho, thint, sp)
    L = (torch.tensor(phi, device="cuda").conj() * out).sum().real
    L.backward()
    return tpsi.grad.cpu().numpy(), tho.grad.numpy(), thint.grad.numpy()


def _fd(f, x0, d):
    return (f(x0 + H_FD * d) - f(x0 - H_FD * d)) / (2 * H_FD)


def test_gradient_psi(problem, orc):
    sp, psi, phi, Ho, Hint = problem
    gpsi, _, _ = _grads(sp, psi, phi, Ho, Hint)
    # H is Hermitian here, so dL/dpsi = H phi; compare with the oracle's operator
    assert np.linalg.norm(gpsi - orc.apply_h(N, M, phi, Ho, Hint, mode=2)) <= 1e-12 * np.linalg.norm(gpsi)
    rng = np.random.default_rng(1)
    for _ in range(3):
        d = rng.standard_normal(psi.size) + 1j * rng.standard_normal(psi.size)
        fd = _fd(lambda x: _loss(sp, x, phi, Ho, Hint), psi, d)
        an = float(np.real(np.vdot(gpsi, d)))
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(an))


def test_gradient_ho(problem):
    sp, psi, phi, Ho, Hint = problem
    _, gho, _ = _grads(sp, psi, phi, Ho, Hint)
    for (k, l) in [(0, 0), (2, 5), (7, 1), (3, 3)]:
        for unit in (1.0, 1.0j):
            d = np.zeros((M, M), np.complex128)
            d[k, l] = unit
            fd = _fd(lambda x: _loss(sp, psi, phi, x, Hint), Ho, d)
            an = float(np.real(np.conj(gho[k, l]) * unit))
            assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (k, l, unit, fd, an)


def test_gradient_hint_entries(problem):
    sp, psi, phi, Ho, Hint = problem
    _, _, ghint = _grads(sp, psi, phi, Ho, Hint)
    M2, M3 = M * M, M * M * M
    idx = lambda k, s, q, l: k + s * M + q * M2 + l * M3
    # representatives of several rules, and entries no rule reads (gradient 0)
    for (k, s, q, l) in [(1, 1, 1, 1), (1, 3, 1, 3), (2, 2, 5, 5), (4, 4, 4, 6), (0, 6, 6, 6),
                         (3, 3, 1, 7), (1, 4, 6, 6), (2, 5, 5, 7), (0, 3, 4, 6), (3, 1, 4, 6),
                         (5, 2, 5, 2)]:
        x = idx(k, s, q, l)
        for unit in (1.0, 1.0j):
            d = np.zeros(M ** 4, np.complex128)
            d[x] = unit
            fd = _fd(lambda h: _loss(sp, psi, phi, Ho, h), Hint, d)
            an = float(np.real(np.conj(ghint[x]) * unit))
            assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), ((k, s, q, l), unit, fd, an)


def test_gradient_hint_orbits(problem):
    sp, psi, phi, Ho, Hint = problem
    _, _, ghint = _grads(sp, psi, phi, Ho, Hint)
    rng = np.random.default_rng(5)
    for _ in range(4):
        # a perturbation with the full 8-fold symmetry (whole orbits move together)
        d = mc.symmetrize_hint(rng.standard_normal(M ** 4) + 1j * rng.standard_normal(M ** 4), M)
        fd = _fd(lambda h: _loss(sp, psi, phi, Ho, h), Hint, d)
        an = float(np.real(np.vdot(ghint, d)))
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(an))


def test_hellmann_feynman_lieb_g2():
    g, niter = 2.0, 200
    sp = mc.FockSpace(N, M)
    C0 = mc.random_problem(N, M, 83)[0]

    def E0(gg):
        sp.set_integrals(*mc.lieb_integrals(M, gg))
        return sp.ground(C0, niter)

    E, psi0, _ = E0(g)
    psi0 = psi0 / torch.linalg.vector_norm(psi0)
    hf = ag.hellmann_feynman_lieb(sp.rho2(psi0).cpu().numpy(), M)
    fd = (E0(g + H_FD)[0] - E0(g - H_FD)[0]) / (2 * H_FD)
    assert abs(fd - hf) <= 2e-5 * abs(hf), (fd, hf)
    # the same gradient from the reference's own two-body density routine
    if oracle.ref_available():
        R = oracle.Ref()
        t = R.tables(N, M)
        rho2_ref = R.rho2("XX", N, M, psi0.cpu().numpy(), t)
        assert abs(ag.hellmann_feynman_lieb(rho2_ref, M) - hf) <= 1e-12 * abs(hf)


def test_lowmem_ground_matches_stored_basis():
    sp = mc.FockSpace(7, 7)
    sp.set_integrals(*mc.lieb_integrals(7, 5.0))
    C0 = mc.random_problem(7, 7, 84)[0]
    E1, v1, it1 = sp.ground(C0, 120)
    E2, v2, it2 = sp.ground(C0, 120, lowmem=True)
    assert it1 == it2
    assert abs(E1 - E2) <= 1e-10 * abs(E1)
    ov = abs(torch.vdot(v1, v2).item()) / (torch.linalg.vector_norm(v1) * torch.linalg.vector_norm(v2)).item()
    assert abs(ov - 1) < 1e-9
