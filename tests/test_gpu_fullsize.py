"""GPU parity at the bench size, 32^3x64 (kappa 0.1615, mu 0.0015, links exp(i 0.3 H)):
the FP64 operator against the oracle on one random field, size-independent identities
of the operator (adjointness, gamma5-hermiticity, linearity), and a mixed-precision
solve whose true residual the oracle's own operator recomputes.  Tolerances: 1e-13
relative for FP64 operators, 1e-10 for the FP64 true residual of a solve."""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

L = (32, 32, 32, 64)
KAPPA, MU = 0.1615, 0.0015


@pytest.fixture(scope="module")
def big(qkx, oracle):
    U = oracle.apply_bc(L, oracle.gauge_random(L, 0.3, 1234), -1)
    lat = qkx.Lattice(qkx.LatticeInfo(L=L, kappa=KAPPA, mu=MU, twistSign=1))
    lat.load_gauge(U, qkx.LINKS_AS_GIVEN)
    yield U, lat
    lat.close()


def cdot(a, b) -> complex:
    """<a, b> = sum conj(a) b over fields in the [V][4][3][2] real layout."""
    a = a.reshape(-1, 2)
    b = b.reshape(-1, 2)
    return complex(np.dot(a[:, 0], b[:, 0]) + np.dot(a[:, 1], b[:, 1]),
                   np.dot(a[:, 0], b[:, 1]) - np.dot(a[:, 1], b[:, 0]))


def test_tm_matches_oracle_at_full_size(qkx, oracle, big):
    U, lat = big
    psi = oracle.spinor_gaussian(L, 77)
    assert rel(lat.apply("tm", psi), oracle.apply("tm", L, U, psi, KAPPA, MU)) < 1e-13


def test_operator_identities_at_full_size(qkx, oracle, big):
    U, lat = big
    x = oracle.spinor_gaussian(L, 78)
    y = oracle.spinor_gaussian(L, 79)
    Mx, My, Mdx = lat.apply("tm", x), lat.apply("tm", y), lat.apply("tm_dag", x)
    # <x, M y> = <M^+ x, y>: the sums run over 5e7 terms, so the bound is relative to |x| |M y|
    scale = np.linalg.norm(x) * np.linalg.norm(My)
    assert abs(cdot(x, My) - cdot(Mdx, y)) <= 1e-12 * scale
    # M^+ = g5 M(-mu) g5 (a flipped twist sign is M at -mu)
    lat.set_params(kappa=KAPPA, mu=MU, twistSign=-1)
    try:
        g5Mg5x = lat.apply("gamma5", lat.apply("tm", lat.apply("gamma5", x)))
    finally:
        lat.set_params(kappa=KAPPA, mu=MU, twistSign=1)
    assert rel(g5Mg5x, Mdx) < 1e-13
    # linearity
    assert rel(lat.apply("tm", 2.0 * x - 3.0 * y), 2.0 * Mx - 3.0 * My) < 1e-13


def test_mixed_solve_at_full_size(qkx, oracle, big):
    U, lat = big
    bs = [oracle.spinor_gaussian(L, 80), oracle.spinor_gaussian(L, 81)]
    xs, info = lat.invert(bs, method=qkx.SOLVER_CG_EO_MIXED, precision=qkx.PREC_HALF, tol=1e-10)
    assert info.converged == 1 and info.true_residual <= 1e-10
    r = bs[0] - oracle.apply("tm", L, U, xs[0], KAPPA, MU)
    assert np.sqrt(np.sum(r * r) / np.sum(bs[0] * bs[0])) <= 1e-10
