import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA path")


@pytest.fixture(scope="session")
def orc():
    import oracle
    return oracle.Orc()


@pytest.fixture(scope="session")
def golden_tables():
    return dict(np.load(os.path.join(GOLDEN, "tables.npz")))


@pytest.fixture(scope="session")
def golden_ops():
    return dict(np.load(os.path.join(GOLDEN, "operators.npz")))


@pytest.fixture(scope="session")
def golden_lieb():
    return dict(np.load(os.path.join(GOLDEN, "lieb.npz")))


def rel(a, b):
    """Relative Frobenius error |a - b| / |b| (|a - b| when b = 0)."""
    a = np.asarray(a)
    b = np.asarray(b)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def case_keys(golden, prefix):
    """(kind, N, M) triples present in the operator fixture."""
    out = []
    for k in golden:
        if k.startswith(prefix + "_"):
            kind, N, M = k[len(prefix) + 1:].split("_")
            out.append((kind, int(N), int(M)))
    return sorted(out)


def complex_momentum_integrals(M, seed):
    """Random complex integrals that conserve momentum: Hint[k,s,q,l] = 0 unless
    k + s = q + l, with the bosonic 8-fold symmetry; diagonal one-body part."""
    import mcpi_b200 as mc
    rng = np.random.default_rng(seed)
    Ho = np.diag(rng.standard_normal(M)).astype(np.complex128)
    H = mc.symmetrize_hint(rng.standard_normal(M ** 4) + 1j * rng.standard_normal(M ** 4), M)
    l, q, s, k = np.indices((M, M, M, M))            # flat index k + s M + q M^2 + l M^3
    H[(k + s != q + l).reshape(-1)] = 0.0
    return Ho, H
