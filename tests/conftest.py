import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build(ref=True)
    return O


@pytest.fixture(scope="session")
def qkx():
    import qkxtm_mpi_b200 as Q
    Q.lib()  # raises if the CUDA library is missing
    return Q


def rel(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (nb if nb > 0 else 1.0))


def site_index(L, x) -> int:
    return int(x[0] + L[0] * (x[1] + L[1] * (x[2] + L[2] * x[3])))


def oracle_propagator(O, L, U_op, U_smear, kappa, mu, nsmear, alpha, x_src, tol=1e-12, maxIter=2000):
    """The propagator loop of the reference's bin/test_invert_prop.cpp:83-97 composed from
    oracle pieces: point source -> Gaussian smearing -> tmDag -> CG -> smearing -> absorbVector."""
    V = O.volume(L)
    prop = np.zeros((V, 4, 4, 3, 3, 2))
    for sp in range(4):
        for ic in range(3):
            b = O.spinor_point(L, x_src, sp, ic)
            if nsmear > 0:
                b = O.gaussian_smear(L, U_smear, b, nsmear, alpha)
            rhs = O.apply("tm_dag", L, U_op, b, kappa, mu)
            x, _, _ = O.cg(L, U_op, rhs, kappa, mu, tol=tol, maxIter=maxIter)
            if nsmear > 0:
                x = O.gaussian_smear(L, U_smear, x, nsmear, alpha)
            O.absorb_vector(x, sp, ic, prop)
    return prop
