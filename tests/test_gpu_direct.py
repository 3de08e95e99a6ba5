"""The direct H.psi kernel (MCPI_OPT_DIRECT_HPSI) for momentum-block integrals.

The direct kernel applies the same pair matrix as the two pair kernels, row by
row with no intermediate, so it sums the same terms in another order: it is
checked against the oracle's restatement of the reference
(hamiltonianMatrix.h:891-1425, applyHconf_XX) where that is cheap, against the
two-kernel form (MCPI_OPT_DIRECT_HPSI = 0) at the benchmark sizes, in the
real-coefficient specialisation (Lieb-Liniger) and the general complex one
(random complex momentum-conserving integrals), on row ranges (bit for bit the
rows of the whole-vector call) and through a Lanczos run."""
import numpy as np
import pytest
import torch

import mcpi_b200 as mc
from conftest import complex_momentum_integrals, rel

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _space(N, M, direct, Ho, Hint):
    sp = mc.FockSpace(N, M, device=0)
    sp.set_option(mc.OPT_DIRECT_HPSI, direct)
    sp.set_integrals(Ho, Hint)
    return sp


def _state(nc, seed):
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    x = torch.randn(nc, dtype=torch.complex128, device="cuda", generator=gen)
    return x / torch.linalg.vector_norm(x)


@pytest.mark.parametrize("N,M,kind", [(2, 3, "lieb"), (9, 2, "lieb"), (7, 5, "lieb"), (8, 9, "lieb"),
                                      (6, 11, "lieb"), (5, 16, "lieb"), (3, 12, "complex"), (7, 6, "complex"),
                                      (5, 10, "complex"), (4, 14, "complex")])
def test_direct_against_oracle(orc, N, M, kind):
    Ho, Hint = mc.lieb_integrals(M, 2.5) if kind == "lieb" else complex_momentum_integrals(M, 10 * N + M)
    C = mc.random_problem(N, M, 5)[0]
    ref = orc.apply_h(N, M, C, Ho, Hint, mode=2)
    sp = _space(N, M, 1, Ho, Hint)
    got = sp.apply_h(C).cpu().numpy()
    assert rel(got, ref) <= TOL, (N, M, kind)
    if kind == "complex":     # Hermitian integrals: the adjoint operator (its own blocks) gives H.psi too
        assert rel(sp.apply_h_adjoint(C).cpu().numpy(), orc.apply_h(N, M, C, Ho, Hint, mode=2)) <= TOL
    sp.close()


@pytest.mark.parametrize("N,M", [(16, 10), (10, 10), (12, 7), (6, 16), (20, 6)])
def test_direct_against_two_kernels(N, M):
    Ho, Hint = mc.lieb_integrals(M, 1.0)
    two = _space(N, M, 0, Ho, Hint)
    x = _state(two.nc, N * 100 + M)
    ref = two.apply_h(x)
    two.close()
    sp = _space(N, M, 1, Ho, Hint)
    got = sp.apply_h(x)
    assert float(torch.linalg.vector_norm(got - ref) / torch.linalg.vector_norm(ref)) <= TOL
    ms = sp.apply_h_profile(x, reps=2)
    assert ms[0] > 0.0 and ms[1] == 0.0          # one kernel
    sp.close()


def test_direct_is_the_default_up_to_eleven_orbitals():
    for M, kind in ((7, "lieb"), (10, "lieb"), (11, "lieb"), (13, "lieb"), (8, "complex"), (12, "complex")):
        N = 6
        Ho, Hint = mc.lieb_integrals(M, 1.0) if kind == "lieb" else complex_momentum_integrals(M, 2)
        sp = mc.FockSpace(N, M, device=0)
        sp.set_integrals(Ho, Hint)
        x = _state(sp.nc, M)
        one = sp.apply_h_profile(x, reps=1)[1] == 0.0
        assert one == (M <= 11), (M, kind)
        sp.close()


@pytest.mark.parametrize("kind", ["lieb", "complex"])
def test_direct_row_ranges_bitwise(kind):
    N, M = 11, 9
    Ho, Hint = mc.lieb_integrals(M, 2.0) if kind == "lieb" else complex_momentum_integrals(M, 3)
    sp = _space(N, M, 1, Ho, Hint)
    x = _state(sp.nc, 7)
    full = sp.apply_h(x)
    nc = sp.nc
    for r0, r1 in [(0, nc), (0, 1), (nc - 1, nc), (123, 4567), (nc // 3, nc // 3 + 257), (nc // 2, nc)]:
        assert torch.equal(sp.apply_h_rows(x, r0, r1), full[r0:r1]), (r0, r1)
    sp.close()


def test_direct_lanczos_agrees_with_two_kernels():
    N, M = 12, 9
    Ho, Hint = mc.lieb_integrals(M, 3.0)
    C0 = mc.random_problem(N, M, 17)[0]
    runs = []
    for direct in (0, 1):
        sp = _space(N, M, direct, Ho, Hint)
        it, diag, off, lvec = sp.lanczos(C0, 60)
        del lvec
        E, _, _ = sp.ground(C0, 60)
        runs.append((it, diag.real, off[:59], E))
        sp.close()
    (i0, a0, b0, E0), (i1, a1, b1, E1) = runs
    assert i0 == i1 == 60
    scale = np.abs(a0).max()
    assert np.abs(a0 - a1).max() <= 1e-10 * scale and np.abs(b0 - b1).max() <= 1e-10 * scale
    assert abs(E0 - E1) <= 1e-10 * abs(E0)


@pytest.mark.parametrize("N,direct_expected", [(63, True), (64, False)])
def test_direct_form_particle_limit(orc, N, direct_expected):
    # the direct form's square-root table takes (N + 3)^2 doubles of shared
    # memory: from N = 64 on, whole-vector calls take the two pair kernels
    M = 3
    Ho, Hint = mc.lieb_integrals(M, 1.5)
    C = mc.random_problem(N, M, 9)[0]
    sp = _space(N, M, 1, Ho, Hint)
    got = sp.apply_h(C).cpu().numpy()
    assert rel(got, orc.apply_h(N, M, C, Ho, Hint, mode=2)) <= TOL
    assert (sp.apply_h_profile(torch.from_numpy(C).cuda(), reps=1)[1] == 0.0) == direct_expected
    sp.close()
