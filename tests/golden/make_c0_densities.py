"""Generate tests/golden/c0_densities.npz from the reference itself.

N=10 bosons in M=10 orbitals (nc = 92,378), the state of
oracle.random_inputs(10, 10, SEED) (a normalised complex-normal vector from
numpy.random.default_rng(SEED)). The reference's own OBrho_XM
(onebodyMatrix.h:190-251) and TBrho_XX (twobodyMatrix.h:991-1487), compiled
unmodified into oracle/_ref/libmcpi_ref.so (oracle/Makefile), with its own
int32 maps (setupFocks, OneOneMap, OneTwoMap, TwoTwoMap), give rho1 and rho2.
The state itself is not stored: the tests regenerate it from the seed and
check it against the stored sum and first entries.

    python tests/golden/make_c0_densities.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
import oracle  # noqa: E402

N, M, SEED = 10, 10, 2027


def main():
    oracle.build(ref=True)
    R = oracle.Ref()
    C = oracle.random_inputs(N, M, SEED)[0]
    t = R.tables(N, M)
    rho1 = R.rho1("XM", N, M, C, t)
    rho2 = R.rho2("XX", N, M, C, t)
    np.savez_compressed(os.path.join(HERE, "c0_densities.npz"), N=N, M=M, seed=SEED, C_sum=C.sum(),
                        C_head=C[:8], rho1=rho1, rho2=rho2)
    print("c0 densities written to", HERE, "trace rho1", np.trace(rho1))


if __name__ == "__main__":
    main()
