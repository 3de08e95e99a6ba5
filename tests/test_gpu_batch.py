"""Batched, graph-captured Lanczos ground states against the one-solve path.

Every member must give the same lowest eigenvalue (|dE0| <= 1e-10, relative to
max(1, |E0|)) and the same step count as mcpi_ground on the same start vector;
a member that breaks down at once is masked while the others run on."""
import numpy as np
import pytest

import mcpi_b200 as mc
from conftest import complex_momentum_integrals

pytestmark = pytest.mark.gpu


def _start(nc, seed):
    rng = np.random.default_rng(seed)
    C = rng.standard_normal(nc) + 1j * rng.standard_normal(nc)
    return C / np.linalg.norm(C)


def test_batch_matches_single_solves():
    members = [(6, 7), (8, 9), (5, 11), (9, 7), (7, 9), (4, 11), (10, 7), (6, 9)]
    gs = [0.05, 2.0, 30.0, 0.7, 11.0, 90.0, 0.01, 4.0]
    lm = 40
    b = mc.Batch(members, lm)
    starts = []
    for k, ((N, M), g) in enumerate(zip(members, gs)):
        Ho, Hint = mc.lieb_integrals(M, g)
        b.set_integrals(k, Ho, Hint)
        C = _start(b.nc[k], 100 + k)
        starts.append(C)
        b.set_start(k, C)
    E, it = b.run()
    E2, it2 = b.run()          # replay of the captured graph gives the same answers
    assert np.array_equal(E, E2) and np.array_equal(it, it2)
    for k, ((N, M), g) in enumerate(zip(members, gs)):
        sp = mc.FockSpace(N, M)
        sp.set_integrals(*mc.lieb_integrals(M, g))
        Es, _, its = sp.ground(starts[k], lm)
        assert it[k] == its, (k, it[k], its)
        assert abs(E[k] - Es) <= 1e-10 * max(1.0, abs(Es)), (k, E[k], Es)
        sp.close()
    b.close()


def test_batch_masks_a_breakdown():
    members = [(4, 5), (6, 7)]
    b = mc.Batch(members, 20)
    # member 0: all particles in the zero-momentum orbital of a free ring is an eigenvector
    Ho, Hint = mc.lieb_integrals(5, 0.0)
    b.set_integrals(0, Ho, Hint)
    C0 = np.zeros(b.nc[0], np.complex128)
    C0[mc.FockToIndex(4, 5, [0, 0, 4, 0, 0])] = 1.0
    b.set_start(0, C0)
    b.set_integrals(1, *mc.lieb_integrals(7, 3.0))
    C1 = _start(b.nc[1], 7)
    b.set_start(1, C1)
    E, it = b.run()
    assert it[0] == 0 and E[0] == pytest.approx(0.0, abs=1e-12)
    sp = mc.FockSpace(6, 7)
    sp.set_integrals(*mc.lieb_integrals(7, 3.0))
    Es, _, its = sp.ground(C1, 20)
    assert it[1] == its == 20 and abs(E[1] - Es) <= 1e-10 * abs(Es)


def test_batch_schedules_agree():
    # every tile schedule gives the single-solve eigenvalues; the autotuner picks
    # one of the candidates and reports a probe time for each
    members = [(7, 9), (5, 11), (9, 7), (12, 7)]
    gs = [1.5, 20.0, 0.3, 5.0]
    lm = 30
    starts = [_start(mc.nc_of(N, M), 200 + k) for k, (N, M) in enumerate(members)]
    ref = []
    for k, ((N, M), g) in enumerate(zip(members, gs)):
        sp = mc.FockSpace(N, M)
        sp.set_integrals(*mc.lieb_integrals(M, g))
        ref.append(sp.ground(starts[k], lm)[0])
    for tile in (512, 1024, 2048, 0):
        b = mc.Batch(members, lm)
        for k, ((N, M), g) in enumerate(zip(members, gs)):
            b.set_integrals(k, *mc.lieb_integrals(M, g))
            b.set_start(k, starts[k])
        b.set_schedule(tile)
        assert b.schedule()[0] == 0
        E, _ = b.run()
        used, ms = b.schedule()
        assert used == (tile if tile else used) and used in (512, 1024, 2048)
        if tile == 0:
            assert np.all(ms > 0) and ms[(512, 1024, 2048).index(used)] == ms.min()
        else:
            assert np.all(ms == 0)
        with pytest.raises(mc.MCPIError):
            b.set_schedule(512)            # the solve is captured
        for k in range(len(members)):
            assert abs(E[k] - ref[k]) <= 1e-10 * max(1.0, abs(ref[k])), (tile, k, E[k], ref[k])
        b.close()


def test_batch_hpsi_forms_against_single_solves():
    # one batch mixing the direct H.psi form (M <= 11: real Lieb blocks as a
    # kernel parameter, complex momentum blocks from shared memory) with the
    # two pair kernels (M = 12, 13): every member's E0 matches its own
    # single-space solve
    members = [(7, 9), (6, 8), (5, 12), (4, 13), (8, 11), (5, 8)]
    ints = [mc.lieb_integrals(9, 1.5), complex_momentum_integrals(8, 5), mc.lieb_integrals(12, 3.0),
            mc.lieb_integrals(13, 0.5), mc.lieb_integrals(11, 8.0), complex_momentum_integrals(8, 6)]
    lm = 40
    b = mc.Batch(members, lm)
    starts = []
    for k, ((N, M), (Ho, Hint)) in enumerate(zip(members, ints)):
        b.set_integrals(k, Ho, Hint)
        starts.append(_start(b.nc[k], 400 + k))
        b.set_start(k, starts[k])
    E, it = b.run()
    for k, ((N, M), (Ho, Hint)) in enumerate(zip(members, ints)):
        sp = mc.FockSpace(N, M)
        sp.set_integrals(Ho, Hint)
        Es, _, its = sp.ground(starts[k], lm)
        assert it[k] == its, (k, it[k], its)
        assert abs(E[k] - Es) <= 1e-10 * max(1.0, abs(Es)), (k, E[k], Es)
        sp.close()
    # a member's integrals turning complex after the capture: the batch captures again
    b.set_integrals(0, *complex_momentum_integrals(9, 7))
    E2, it2 = b.run()
    sp = mc.FockSpace(7, 9)
    sp.set_integrals(*complex_momentum_integrals(9, 7))
    Es = sp.ground(starts[0], lm)[0]
    assert abs(E2[0] - Es) <= 1e-10 * max(1.0, abs(Es))
    assert np.array_equal(E2[1:], E[1:])
    sp.close()
    b.close()


def test_batch_hpsi_schedules_agree():
    # the four batched H.psi schedules (concurrent M groups or not, interleaved
    # blocks or not) change no member's arithmetic: bitwise equal results
    members = [(6, 7), (8, 9), (5, 11), (9, 7), (7, 11)]
    gs = [0.3, 2.0, 30.0, 0.7, 5.0]
    lm = 30
    results = []
    for sched in range(4):
        b = mc.Batch(members, lm)
        b.set_schedule(1024)
        b.set_hpsi_schedule(sched)
        for k, ((N, M), g) in enumerate(zip(members, gs)):
            b.set_integrals(k, *mc.lieb_integrals(M, g))
            b.set_start(k, _start(b.nc[k], 200 + k))
        results.append(b.run())
        assert b.hpsi_schedule()[0] == sched
        b.close()
    for E, it in results[1:]:
        assert np.array_equal(E, results[0][0]) and np.array_equal(it, results[0][1])
    # autotuned: one of the four, with its probe times
    b = mc.Batch(members, lm)
    for k, ((N, M), g) in enumerate(zip(members, gs)):
        b.set_integrals(k, *mc.lieb_integrals(M, g))
        b.set_start(k, _start(b.nc[k], 200 + k))
    E, it = b.run()
    sched, ms = b.hpsi_schedule()
    assert 0 <= sched <= 3 and np.all(ms > 0)
    assert np.allclose(E, results[0][0], rtol=1e-10, atol=1e-10)
    b.close()
