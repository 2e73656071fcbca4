"""CPU tests of the oracle: pinned to the reference's golden vectors (made by
tests/golden/make_golden.py from the reference's own compiled sources), to the
live reference build when it is present, and to analytic properties."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel

def _load(name):
    return np.load(os.path.join(GOLDEN, name))


def _inputs(O, L, eps, seed_u, seed_psi, bc=True):
    U = O.gauge_random(L, eps, seed_u)
    if bc:
        U = O.apply_bc(L, U, -1)
    return U, O.spinor_gaussian(L, seed_psi)


def _checksum(a):
    w = np.linspace(0.5, 1.5, a.size).reshape(a.shape)
    return np.array([a.sum(), (a * w).sum(), (a * a).sum()])


def test_generator_reproduces_golden_inputs(oracle):
    g = _load("ref_ops_small.npz")
    L = tuple(int(v) for v in g["L"])
    U, psi = _inputs(oracle, L, float(g["eps"]), int(g["seed_u"]), int(g["seed_psi"]))
    np.testing.assert_allclose(np.concatenate([_checksum(U), _checksum(psi)]), g["in_checksum"],
                               rtol=1e-12, atol=1e-12)


def test_oracle_matches_reference_golden_small(oracle):
    """Every operator, full output, 4x2x2x4, twistSign +1 and -1: FP64, 1e-13."""
    g = _load("ref_ops_small.npz")
    L = tuple(int(v) for v in g["L"])
    U, psi = _inputs(oracle, L, float(g["eps"]), int(g["seed_u"]), int(g["seed_psi"]))
    n = 0
    for key in g.files:
        if "@" not in key:
            continue
        op, ts = key.split("@")
        out = oracle.apply(op, L, U, psi, float(g["kappa"]), float(g["mu"]), int(ts))
        assert rel(out, g[key]) < 1e-13, key
        n += 1
    assert n >= 28


def test_oracle_matches_reference_golden_probe(oracle):
    g = _load("ref_ops_probe.npz")
    L = tuple(int(v) for v in g["L"])
    U, psi = _inputs(oracle, L, float(g["eps"]), int(g["seed_u"]), int(g["seed_psi"]))
    W = [oracle.spinor_gaussian(L, int(g["probe_seed"]) + k) for k in range(3)]
    sites = g["sites"]
    for op in oracle.REF_OPS:
        out = oracle.apply(op, L, U, psi, float(g["kappa"]), float(g["mu"]), 1)
        np.testing.assert_allclose(np.sum(out * out), g[f"{op}:norm2"][0], rtol=1e-13)
        np.testing.assert_allclose([np.sum(w * out) for w in W], g[f"{op}:probe"], rtol=1e-11,
                                   atol=1e-11 * np.sqrt(g[f"{op}:norm2"][0]))
        assert rel(out[sites], g[f"{op}:sites"]) < 1e-13, op


def test_oracle_blas_matches_reference_golden(oracle):
    g = _load("ref_ops_probe.npz")
    L = tuple(int(v) for v in g["L"])
    _, x = _inputs(oracle, L, float(g["eps"]), int(g["seed_u"]), int(g["seed_psi"]))
    y = oracle.spinor_gaussian(L, 23)
    np.testing.assert_allclose(oracle.re_dot(x, y), g["blas:redot"][0], rtol=1e-12)
    np.testing.assert_allclose(oracle.norm2(x), g["blas:norm2"][0], rtol=1e-13)
    x1 = x.copy()
    oracle.axpy(0.37, y, x1)
    assert rel(x1[g["sites"]], g["blas:axpy:sites"]) == 0.0
    x2 = x.copy()
    oracle.xpay(-0.41, y, x2)
    assert rel(x2[g["sites"]], g["blas:xpay:sites"]) == 0.0


@pytest.mark.parametrize("tag", ["4x4x4x8", "8x8x8x16"])
def test_oracle_cg_matches_reference_golden(oracle, tag):
    g = _load("ref_cg.npz")
    L = tuple(int(v) for v in g[f"{tag}:L"])
    su, sb = (int(v) for v in g[f"{tag}:seeds"])
    U, b = _inputs(oracle, L, float(g["eps"]), su, sb)
    np.testing.assert_allclose(np.concatenate([_checksum(U), _checksum(b)]), g[f"{tag}:in_checksum"],
                               rtol=1e-12, atol=1e-12)
    k, mu = float(g["kappa"]), float(g["mu"])
    Mdb = oracle.apply("tm_dag", L, U, b, k, mu)
    x, iters, trace = oracle.cg(L, U, Mdb, k, mu, tol=1e-10, maxIter=1000)
    assert iters == int(g[f"{tag}:iters_oracle"][0])
    np.testing.assert_allclose(np.sum(x * x), g[f"{tag}:x_norm2"][0], rtol=1e-10)
    sites = np.unique(np.linspace(0, oracle.volume(L) - 1, 16).astype(np.int64))
    assert rel(x[sites], g[f"{tag}:x_sites"]) < 1e-9
    r = b - oracle.apply("tm", L, U, x, k, mu)
    tr = np.sqrt(np.sum(r * r) / np.sum(b * b))
    np.testing.assert_allclose(tr, g[f"{tag}:true_residual"][0], rtol=1e-3)
    assert tr < 2e-10


def test_oracle_vs_live_reference(oracle):
    """All operators against the reference compiled from its sources (when present)."""
    if not oracle.ref_available():
        pytest.skip("reference build not present")
    for L, seed in (((4, 4, 4, 8), 5), ((6, 4, 2, 4), 6), ((2, 2, 2, 2), 7)):
        U, psi = _inputs(oracle, L, 0.25, seed, seed + 100, bc=(seed % 2 == 1))
        for ts in (1, -1):
            for op in oracle.REF_OPS:
                a = oracle.apply(op, L, U, psi, 0.1615, 0.004, ts)
                b = oracle.ref_apply(op, L, U, psi, 0.1615, 0.004, ts)
                assert rel(a, b) < 1e-13, (L, op, ts)


def test_oracle_cg_vs_live_reference(oracle):
    if not oracle.ref_available():
        pytest.skip("reference build not present")
    L = (4, 4, 4, 8)
    U, b = _inputs(oracle, L, 0.3, 77, 78)
    x, it, _ = oracle.cg(L, U, b, 0.1615, 0.0015, -1, tol=1e-8, maxIter=500)
    xr = oracle.ref_cg(L, U, b, 0.1615, 0.0015, -1, tol=1e-8, maxIter=500)
    assert rel(x, xr) < 1e-12


def test_gamma5_hermiticity(oracle):
    """M(s)^+ = g5 M(-s) g5 and <x, M y> = <M^+ x, y> (UKQCD and chiral)."""
    L = (4, 4, 2, 6)
    U, x = _inputs(oracle, L, 0.3, 3, 4)
    y = oracle.spinor_gaussian(L, 5)
    lhs = oracle.apply("tm_dag", L, U, x, 0.16, 0.02, 1)
    rhs = oracle.apply("gamma5", L, U,
                       oracle.apply("tm", L, U, oracle.apply("gamma5", L, U, x), 0.16, 0.02, -1))
    assert rel(lhs, rhs) < 1e-14
    for basis, g5 in (("", "gamma5"), ("_chiral", "gamma5_chiral")):
        My = oracle.apply("tm" + basis, L, U, y, 0.16, 0.02, 1)
        # M^+ x through the gamma5 trick, in either basis
        Mdx = oracle.apply(g5, L, U,
                           oracle.apply("tm" + basis, L, U, oracle.apply(g5, L, U, x), 0.16, 0.02, -1))
        c = lambda v: (v[..., 0] + 1j * v[..., 1]).ravel()  # noqa: E731
        a = np.vdot(c(x), c(My))
        b = np.vdot(c(Mdx), c(y))
        assert abs(a - b) < 1e-12 * abs(a)


def test_free_field_plane_wave(oracle):
    """U = 1, periodic: M e^{ipx} u = [(1 - 2k sum cos p) + 2ik sum g_mu sin p + i c g5] e^{ipx} u."""
    L = (4, 6, 2, 8)
    U = oracle.gauge_unit(L)
    V = oracle.volume(L)
    n = (1, 2, 1, 3)
    p = [2 * np.pi * n[m] / L[m] for m in range(4)]
    coords = np.array(np.unravel_index(np.arange(V), (L[3], L[2], L[1], L[0]))[::-1]).T  # x,y,z,t
    phase = np.exp(1j * (coords @ np.array(p)))
    u = (np.arange(12) + 1.0).reshape(4, 3) * (1 + 0.5j)
    psi_c = phase[:, None, None] * u[None]
    psi = np.stack([psi_c.real, psi_c.imag], -1)
    k, mu = 0.13, 0.05
    out = oracle.apply("tm", L, U, psi, k, mu, 1)
    g = _ukqcd_gammas()
    Mmat = (1 - 2 * k * sum(np.cos(pp) for pp in p)) * np.eye(4) + 2j * k * sum(
        g[m] * np.sin(p[m]) for m in range(4)) + 1j * 2 * k * mu * g[4]
    exp = phase[:, None, None] * (Mmat @ u)[None]
    assert rel(out, np.stack([exp.real, exp.imag], -1)) < 1e-13


def _ukqcd_gammas():
    g = np.zeros((5, 4, 4), complex)
    g[0][0, 3] = g[0][1, 2] = 1j; g[0][2, 1] = g[0][3, 0] = -1j
    g[1][0, 3] = g[1][3, 0] = 1; g[1][1, 2] = g[1][2, 1] = -1
    g[2][0, 2] = g[2][3, 1] = 1j; g[2][1, 3] = g[2][2, 0] = -1j
    g[3] = np.diag([1, 1, -1, -1])
    g[4][0, 2] = g[4][1, 3] = g[4][2, 0] = g[4][3, 1] = 1
    return g


def test_gauge_generator_properties(oracle):
    L = (8, 8, 8, 16)
    U = oracle.gauge_random(L, 0.3, 1234)
    u = U[..., 0] + 1j * U[..., 1]
    I = np.einsum("vdab,vdcb->vdac", u, u.conj())
    assert np.abs(I - np.eye(3)).max() < 1e-14
    assert np.abs(np.linalg.det(u) - 1).max() < 1e-14
    assert abs(oracle.plaquette(L, U) - 0.7832) < 0.003
