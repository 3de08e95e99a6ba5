"""Parity at the full benchmark sizes, where the oracle cannot do whole vectors.

N=16, M=10 (nc = 2,042,975) and N=20, M=10 (nc = 10,015,005, a 160 MB state):
H.psi is compared with the oracle on row samples spread over the index range
(the oracle evaluates any row range), and size-independent properties are
checked on whole vectors: Hermiticity, linearity, the energy identity
<psi|H|psi> = sum Ho rho1 + 1/2 sum Hint rho2, the density traces, and the
Lanczos ground state's Ritz residual."""
import numpy as np
import pytest
import torch

import mcpi_b200 as mc
from conftest import rel

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _rand(nc, seed):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    x = torch.randn(nc, dtype=torch.complex128, device="cuda", generator=g)
    return x / torch.linalg.vector_norm(x)


def _sampled_parity(orc, N, M, Ho, Hint, psi, out, chunks=6, rows=400):
    nc = mc.nc_of(N, M)
    IF = orc.focks(N, M)
    C = psi.cpu().numpy()
    got = out.cpu().numpy()
    ref = np.zeros(nc, np.complex128)
    starts = np.linspace(0, nc - rows, chunks).astype(np.int64)
    sel = np.concatenate([np.arange(s, s + rows) for s in starts])
    for s in starts:
        orc.apply_h(N, M, C, Ho, Hint, mode=2, IF=IF, row0=int(s), row1=int(s + rows), out=ref)
    return rel(got[sel], ref[sel])


@pytest.mark.parametrize("N,M,kind", [(16, 10, "lieb"), (16, 10, "random"), (20, 10, "lieb")])
def test_hpsi_row_samples(orc, N, M, kind):
    if kind == "lieb":
        Ho, Hint = mc.lieb_integrals(M, 1.0 if N == 16 else 10.0)
    else:
        _, Ho, Hint = mc.random_problem(4, M, 91)   # dense pair matrix
    sp = mc.FockSpace(N, M)
    sp.set_integrals(Ho, Hint)
    psi = _rand(sp.nc, 1)
    out = sp.apply_h(psi)
    assert _sampled_parity(orc, N, M, Ho, Hint, psi, out) <= TOL


@pytest.mark.parametrize("N,M,g", [(16, 10, 1.0), (20, 10, 10.0)])
def test_hermiticity_linearity_energy(N, M, g):
    Ho, Hint = mc.lieb_integrals(M, g)
    sp = mc.FockSpace(N, M)
    sp.set_integrals(Ho, Hint)
    a, b = _rand(sp.nc, 2), _rand(sp.nc, 3)
    Ha, Hb = sp.apply_h(a), sp.apply_h(b)
    x = torch.vdot(a, Hb).item()
    y = torch.vdot(b, Ha).item()
    assert abs(x - np.conj(y)) <= 1e-12 * abs(x)
    s, t = 0.3 - 1.1j, -0.7 + 0.2j
    lin = sp.apply_h(s * a + t * b) - (s * Ha + t * Hb)
    assert (torch.linalg.vector_norm(lin) / torch.linalg.vector_norm(Ha)).item() <= 1e-13
    e1 = torch.vdot(a, Ha).item()
    r1 = sp.rho1(a).cpu().numpy()
    r2 = sp.rho2(a).cpu().numpy()
    e2 = np.sum(Ho * r1) + 0.5 * np.sum(Hint * r2)
    assert abs(e1 - e2) <= 1e-12 * abs(e1)
    assert abs(np.trace(r1) - N) <= 1e-11 * N
    R = r2.reshape(M, M, M, M)
    assert abs(sum(R[k, s_, s_, k] for k in range(M) for s_ in range(M)) - N * (N - 1)) <= 1e-10 * N * N


def test_large_ground_state():
    # N=20, M=10, g=10: 100 Lanczos steps (16 GB Krylov basis), then rho1/rho2 of the result
    N, M, g = 20, 10, 10.0
    sp = mc.FockSpace(N, M)
    Ho, Hint = mc.lieb_integrals(M, g)
    sp.set_integrals(Ho, Hint)
    E, psi, it = sp.ground(_rand(sp.nc, 4), 100)
    assert it == 100
    nrm = torch.linalg.vector_norm(psi).item()
    assert abs(nrm - 1) < 1e-8
    res = torch.linalg.vector_norm(sp.apply_h(psi) - E * psi).item()
    assert res < 1e-3 * abs(E)          # 100 steps: converged to a small Ritz residual
    r1 = sp.rho1(psi).cpu().numpy()
    r2 = sp.rho2(psi).cpu().numpy()
    assert abs(np.trace(r1).real - N) < 1e-8 * N
    e2 = np.sum(Ho * r1) + 0.5 * np.sum(Hint * r2)
    assert abs(e2 - E) <= 1e-3 * abs(E)  # energy of the Ritz vector (residual-limited)
    assert abs(e2 - torch.vdot(psi, sp.apply_h(psi)).item()) <= 1e-11 * abs(E)
