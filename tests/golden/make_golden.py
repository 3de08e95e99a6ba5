"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs the reference's own C routines (compiled unmodified into
oracle/_ref/libmcpi_ref.so, see oracle/Makefile) on small seeded cases and stores
inputs and outputs as compressed .npz files, so that the parity tests can pin
the oracle and the CUDA path on machines where the reference sources are absent.

    python tests/golden/make_golden.py

Fixtures (all arrays in the reference layouts):
  tables.npz    NCmat, IF, Map, MapOT/strideOT, MapTT/strideTT per (N, M)
                (setupNCmat, setupFocks, OneOneMap, OneTwoMap, TwoTwoMap)
  operators.npz C, Ho, Hint and applyHconf / applyHconf_XX outputs, OBrho_XM and
                TBrho_XX outputs, for the deterministic inputs of
                performanceTest.c:169-219 and for seeded random inputs whose Hint
                carries the bosonic 8-fold symmetry
  lieb.npz      E0 from the reference's ground() (groundStateLieb.c:348-471, with
                the oracle's Jacobi stand-in for LAPACKE_dstev) at N=5, M=11,
                g in {1, 10, 100}, nc/8 = 375 Lanczos steps, plus the published
                11-orbital E0/N column of liebGS.dat:1-10
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
import oracle  # noqa: E402

TABLE_CASES = [(0, 3), (1, 1), (1, 4), (2, 2), (3, 3), (4, 1), (4, 4), (5, 4), (2, 7), (6, 5),
               (4, 6), (7, 3), (3, 8)]
OP_CASES = [(2, 3), (3, 3), (4, 4), (6, 5), (3, 6), (5, 3), (8, 2), (2, 6)]
LIEB_G = [1.0, 10.0, 100.0]
# liebGS.dat:2-4,6 (g, E0/N with 11 orbitals) -- published known answers
LIEB_PUBLISHED = {1.0: 1.87209, 10.0: 13.34261, 30.0: 26.40431, 100.0: 39.94341}


def main():
    oracle.build(ref=True)
    R = oracle.Ref()
    O = oracle.Orc()
    tabs = {}
    for N, M in TABLE_CASES:
        t = R.tables(N, M)
        for k, v in t.items():
            tabs[f"{k}_{N}_{M}"] = v
    np.savez_compressed(os.path.join(HERE, "tables.npz"), **tabs)

    ops = {}
    for N, M in OP_CASES:
        t = R.tables(N, M)
        for kind, (C, Ho, Hint) in (("perf", O.perf_inputs(N, M)),
                                    ("rand", oracle.random_inputs(N, M, seed=100 + 10 * N + M))):
            key = f"{kind}_{N}_{M}"
            ops[f"C_{key}"] = C
            ops[f"Ho_{key}"] = Ho
            ops[f"Hint_{key}"] = Hint
            ops[f"hxx_{key}"] = R.apply_h("XX", N, M, C, Ho, Hint, t)
            ops[f"hplain_{key}"] = R.apply_h("plain", N, M, C, Ho, Hint, t)
            ops[f"rho1_{key}"] = R.rho1("XM", N, M, C, t)
            ops[f"rho2_{key}"] = R.rho2("XX", N, M, C, t)
    np.savez_compressed(os.path.join(HERE, "operators.npz"), **ops)

    N, M = 5, 11
    t = R.tables(N, M)
    nc = R.nc(N, M)
    C0 = O.perf_inputs(N, M)[0]
    E = []
    for g in LIEB_G:
        Ho, Hint = R.lieb(M, g)
        E.append(R.ground(N, M, Ho, Hint, C0, nc // 8, t)[0])
    np.savez_compressed(os.path.join(HERE, "lieb.npz"), g=np.array(LIEB_G), E0=np.array(E),
                        N=N, M=M, niter=nc // 8,
                        published_g=np.array(list(LIEB_PUBLISHED)),
                        published_E0_per_N=np.array(list(LIEB_PUBLISHED.values())))
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
