"""Generate the configuration-size Lanczos fixtures in tests/golden/ from the oracle.

The oracle (oracle/mcpi_oracle.c, pinned bit for bit against the reference
compiled unmodified by tests/test_oracle.py) runs the reference's Lanczos
recurrence (groundStateLieb.c:217-344, orc_lanczos) with its applyHconf_X
restatement (hamiltonianMatrix.h:431-887) or, where every int32 map fits,
applyHconf_XX (hamiltonianMatrix.h:891-1425), on OpenMP threads:

    python tests/golden/make_lanczos.py            # both fixtures (about 40 min on 8 cores)
    python tests/golden/make_lanczos.py c1         # one of them
    python tests/golden/make_lanczos.py sweep

Fixtures:
  lanczos_c1.npz  Lieb-Liniger N=16, M=10, g=1, L=1 (nc = 2,042,975), 150 steps
                  from the normalised complex-normal start vector of
                  numpy.random.default_rng(START_SEED): the alpha and beta
                  coefficients, the lowest Ritz value E0 (scipy's
                  eigh_tridiagonal, cross-checked against numpy.linalg.eigh), and
                  the one-body occupations <n_k> of the Ritz vector (orc_obrho,
                  onebodyMatrix.h:190-251).
  sweep_c2.npz    members of the 64-solve Lieb-Liniger sweep (g log-uniform in
                  [0.01, 100], N uniform in 6..14, M in {7, 9, 11}, drawn from
                  numpy.random.default_rng(2024) in the order N, M, g); the start
                  vector of member k is the normalised complex-normal vector of
                  numpy.random.default_rng(300 + k). Stored: every member's
                  (N, M, g), and for the members with nc <= SWEEP_MAX_NC (45 of 64) the oracle's ground
                  state energy after 120 steps (groundStateLieb.c:348-471, with
                  applyHconf_XX).
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
import oracle  # noqa: E402

START_SEED = 2026
C1 = dict(N=16, M=10, g=1.0, steps=150)
SWEEP_SEED = 2024
SWEEP_COUNT = 64
SWEEP_STEPS = 120
SWEEP_MAX_NC = 120_000     # members whose MapTT fits and whose oracle solve takes seconds


def start_vector(nc, seed):
    rng = np.random.default_rng(seed)
    C = rng.standard_normal(nc) + 1j * rng.standard_normal(nc)
    return C / np.linalg.norm(C)


def sweep_members(count=SWEEP_COUNT, seed=SWEEP_SEED):
    rng = np.random.default_rng(seed)
    N = rng.integers(6, 15, count)
    M = rng.choice([7, 9, 11], count)
    g = 10.0 ** rng.uniform(-2.0, 2.0, count)
    return [(int(n), int(m), float(x)) for n, m, x in zip(N, M, g)]


def lowest_ritz(alpha, beta):
    from scipy.linalg import eigh_tridiagonal
    w, z = eigh_tridiagonal(alpha, beta)
    T = np.diag(alpha) + np.diag(beta, 1) + np.diag(beta, -1)
    w2 = np.linalg.eigvalsh(T)
    assert abs(w[0] - w2[0]) <= 1e-12 * max(1.0, abs(w[0])), (w[0], w2[0])
    return float(w[0]), z[:, 0]


def make_c1(O):
    N, M, g, lm = C1["N"], C1["M"], C1["g"], C1["steps"]
    nc = O.nc(N, M)
    Ho, Hint = O.lieb(M, g)
    C0 = start_vector(nc, START_SEED)
    t0 = time.time()
    IF = O.focks(N, M)
    Map = O.one_one_map(N, M, IF)
    MapOT, sOT = O.one_two_map(N, M, IF)
    print(f"c1: tables {time.time() - t0:.0f} s", flush=True)
    it, diag, off, lvec = O.lanczos(N, M, Ho, Hint, C0, lm, mode=1,
                                    maps=(Map, MapOT, sOT, None, None), IF=IF)
    print(f"c1: {it} Lanczos steps {time.time() - t0:.0f} s", flush=True)
    assert it == lm
    alpha = diag.real.copy()
    beta = off[: lm - 1].real.copy()
    E0, z = lowest_ritz(alpha, beta)
    psi0 = z @ lvec                      # sum_k z_k lvec[k]
    del lvec
    rho1 = O.obrho(N, M, psi0, IF=IF, Map=Map)
    occ = rho1.diagonal().real / np.vdot(psi0, psi0).real
    np.savez_compressed(os.path.join(HERE, "lanczos_c1.npz"), N=N, M=M, g=g, L=1.0, steps=lm,
                        start_seed=START_SEED, alpha=alpha, beta=beta, E0=E0, occupations=occ)
    print(f"c1: E0 = {E0!r}, occupations {np.round(occ, 6)}", flush=True)


def make_sweep(O):
    members = sweep_members()
    pick = [k for k, (n, m, _) in enumerate(members) if O.nc(n, m) <= SWEEP_MAX_NC]
    E0 = []
    t0 = time.time()
    for k in pick:
        n, m, g = members[k]
        Ho, Hint = O.lieb(m, g)
        IF = O.focks(n, m)
        maps = (O.one_one_map(n, m, IF), *O.one_two_map(n, m, IF), *O.two_two_map(n, m, IF))
        E, _, it = O.ground(n, m, Ho, Hint, start_vector(O.nc(n, m), 300 + k), SWEEP_STEPS,
                            mode=2, maps=maps, IF=IF)
        assert it == SWEEP_STEPS or it > 0
        E0.append(E)
        print(f"sweep member {k}: N={n} M={m} g={g:.4g} nc={O.nc(n, m)} steps={it} E0={E!r} "
              f"({time.time() - t0:.0f} s)", flush=True)
    np.savez_compressed(os.path.join(HERE, "sweep_c2.npz"),
                        N=np.array([x[0] for x in members]), M=np.array([x[1] for x in members]),
                        g=np.array([x[2] for x in members]), steps=SWEEP_STEPS,
                        start_seed_base=300, pick=np.array(pick), E0=np.array(E0))


def main():
    oracle.build(ref=False)
    O = oracle.Orc()
    which = sys.argv[1:] or ["sweep", "c1"]
    if "sweep" in which:
        make_sweep(O)
    if "c1" in which:
        make_c1(O)
    print("Lanczos fixtures written to", HERE)


if __name__ == "__main__":
    main()
