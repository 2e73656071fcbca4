"""CPU tests of the smearing / propagator part of the oracle (plaquette, SU(3)
projection, APE and Gaussian smearing, absorbVector, the propagator loop),
pinned to the golden vectors that tests/golden/make_golden.py made from the
reference's own compiled sources, and to the live reference build when present.

Tolerances.  The reference's SU(3) projection finds the eigenvectors of
H = M^+ M from a closed-form cubic; on APE-smeared links the singular values
of M are close together (spread ~1e-3 of their size), so differences of one
rounding in M come out ~1e-13 in the projected link and grow over the APE
iterations (~1e-11 after 20).  Gaussian smearing and the operators do not
amplify rounding."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, oracle_propagator, rel, site_index


def _g():
    return np.load(os.path.join(GOLDEN, "ref_smear.npz"))


def _inputs(O, g):
    L = tuple(int(v) for v in g["L"])
    U = O.gauge_random(L, float(g["eps"]), int(g["seed_u"]))
    psi = O.spinor_gaussian(L, int(g["seed_psi"]))
    return L, U, psi


def _checksum(a):
    w = np.linspace(0.5, 1.5, a.size).reshape(a.shape)
    return np.array([a.sum(), (a * w).sum(), (a * a).sum()])


def _perturbed(O, L, U, scale, seed):
    g = np.concatenate([O.spinor_gaussian(L, seed + k).reshape(-1, 24) for k in range(3)], axis=1)
    return U + scale * g.reshape(U.shape)


def test_smear_golden_inputs(oracle):
    g = _g()
    L, U, psi = _inputs(oracle, g)
    np.testing.assert_allclose(np.concatenate([_checksum(U), _checksum(psi)]), g["in_checksum"], rtol=1e-12)


def test_plaquette_and_projection_golden(oracle):
    g = _g()
    L, U, _ = _inputs(oracle, g)
    np.testing.assert_allclose(oracle.plaquette_ref(L, U), g["plaq"][0], rtol=1e-14)
    np.testing.assert_allclose(oracle.plaquette_ref(L, oracle.apply_bc(L, U, -1)), g["plaq_bc"][0], rtol=1e-14)
    # the oracle's plaquette of the generator tests agrees too
    np.testing.assert_allclose(oracle.plaquette(L, U), g["plaq"][0], rtol=1e-13)
    M = _perturbed(oracle, L, U, 0.3, int(g["seed_pert"]))
    P = M.copy()
    P[:, :3] = oracle.su3_project(M[:, :3])
    sites = g["sites"]
    np.testing.assert_allclose(P[sites], g["proj:sites"], rtol=0, atol=1e-13)
    # the projected links are SU(3) (to 3e-13 for an M with a singular value near 0.03,
    # the accuracy of the reference's closed-form eigen-decomposition)
    Pc = (P[..., 0] + 1j * P[..., 1])[:, :3].reshape(-1, 3, 3)
    assert np.abs(Pc @ np.conj(np.swapaxes(Pc, 1, 2)) - np.eye(3)).max() < 1e-12
    assert np.abs(np.linalg.det(Pc) - 1).max() < 1e-12


def test_ape_golden(oracle):
    g = _g()
    L, U, _ = _inputs(oracle, g)
    sites = g["sites"]
    alpha = float(g["ape_alpha"])
    for n, tol in ((1, 1e-12), (2, 1e-11)):
        A = oracle.ape_smear(L, U, n, alpha)
        np.testing.assert_allclose(A[sites], g[f"ape{n}:sites"], rtol=0, atol=tol)
    A = oracle.ape_smear(L, U, int(g["ape_n"]), alpha)
    np.testing.assert_allclose(A[sites], g["ape:sites"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(oracle.plaquette_ref(L, A), g["ape:plaq"][0], rtol=1e-12)
    # t-links are those of the input
    assert np.array_equal(A[:, 3], U[:, 3])


def test_gaussian_smearing_golden(oracle):
    g = _g()
    L, U, psi = _inputs(oracle, g)
    A = oracle.ape_smear(L, U, int(g["ape_n"]), float(g["ape_alpha"]))
    W = [oracle.spinor_gaussian(L, 9000 + k) for k in range(3)]
    for n in (1, int(g["gauss_n"])):
        s = oracle.gaussian_smear(L, A, psi, n, float(g["gauss_alpha"]))
        np.testing.assert_allclose(s[g["sites"]], g[f"gauss{n}:sites"], rtol=0,
                                   atol=1e-10 * np.abs(g[f"gauss{n}:sites"]).max())
        np.testing.assert_allclose(np.sum(s * s), g[f"gauss{n}:norm2"][0], rtol=1e-10)
        np.testing.assert_allclose([np.sum(w * s) for w in W], g[f"gauss{n}:probe"], rtol=1e-9)


def test_propagator_golden(oracle):
    """Oracle composition of the propagator loop vs the reference's own loop."""
    g = _g()
    L, U, _ = _inputs(oracle, g)
    A = oracle.ape_smear(L, U, int(g["ape_n"]), float(g["ape_alpha"]))
    Ubc = oracle.apply_bc(L, U, -1)
    src = tuple(int(v) for v in g["prop_src"])
    prop = oracle_propagator(oracle, L, Ubc, A, float(g["kappa"]), float(g["mu"]), int(g["prop_n"]),
                             float(g["prop_alpha"]), src, tol=float(g["prop_tol"]))
    assert rel(prop[g["sites"]], g["prop:sites"]) < 1e-9
    np.testing.assert_allclose(np.sum(prop * prop), g["prop:norm2"][0], rtol=1e-9)


def test_absorb_vector(oracle):
    L = (4, 2, 2, 4)
    V = oracle.volume(L)
    prop = np.arange(V * 288, dtype=np.float64).reshape(V, 4, 4, 3, 3, 2)
    before = prop.copy()
    phi = oracle.spinor_gaussian(L, 3)
    oracle.absorb_vector(phi, 2, 1, prop)
    assert np.array_equal(prop[:, :, 2, :, 1], phi)
    mask = np.ones(prop.shape, bool)
    mask[:, :, 2, :, 1] = False
    assert np.array_equal(prop[mask], before[mask])


def test_smearing_vs_live_reference(oracle):
    """Plaquette, projection, APE, Gaussian smearing and absorbVector against the
    reference compiled from its sources, on cubic and non-cubic lattices."""
    if not oracle.ref_available():
        pytest.skip("reference build not present")
    for L, seed in (((4, 4, 4, 4), 61), ((6, 4, 2, 4), 62), ((2, 4, 6, 2), 63)):
        U = oracle.gauge_random(L, 0.3, seed)
        psi = oracle.spinor_gaussian(L, seed + 1)
        assert abs(oracle.plaquette_ref(L, U) - oracle.ref_plaquette(L, U)) < 1e-14
        M = _perturbed(oracle, L, U, 0.5, seed + 2)
        P = M.copy()
        P[:, :3] = oracle.su3_project(M[:, :3])
        assert np.abs(P - oracle.ref_project_su3(L, M)).max() < 1e-13
        for n in (0, 1, 3):
            init = oracle.gauge_random(L, 0.1, seed + 3)  # nsmear 0 leaves the output as it was
            a = oracle.ape_smear(L, U, n, 0.45, out=init)
            b = oracle.ref_ape_smear(L, U, n, 0.45, out=init)
            assert np.abs(a - b).max() < 1e-11, (L, n)
        A = oracle.ref_ape_smear(L, U, 5, 0.5)
        for n in (0, 1, 2, 7):
            init = oracle.spinor_gaussian(L, seed + 4)
            a = oracle.gaussian_smear(L, A, psi, n, 3.0, out=init)
            b = oracle.ref_gaussian_smear(L, A, psi, n, 3.0, out=init)
            assert rel(a, b) < 1e-14, (L, n)
        V = oracle.volume(L)
        p1 = oracle.spinor_gaussian(L, 5).repeat(12, axis=0).reshape(V, 4, 4, 3, 3, 2)
        p2 = p1.copy()
        oracle.absorb_vector(psi, 3, 2, p1)
        oracle.ref_absorb_vector(L, psi, 3, 2, p2)
        assert np.array_equal(p1, p2)


def test_propagator_vs_live_reference(oracle):
    if not oracle.ref_available():
        pytest.skip("reference build not present")
    L = (4, 2, 4, 4)
    U = oracle.gauge_random(L, 0.3, 71)
    A = oracle.ref_ape_smear(L, U, 3, 0.5)
    Ubc = oracle.apply_bc(L, U, -1)
    src = (3, 1, 0, 2)
    for nsmear in (0, 4):
        a = oracle_propagator(oracle, L, Ubc, A, 0.1615, 0.004, nsmear, 4.0, src, tol=1e-12)
        b = oracle.ref_propagator(L, Ubc, A, 0.1615, 0.004, nsmear, 4.0, src=site_index(L, src), tol=1e-12,
                                  maxIter=2000)
        if nsmear == 0:
            # the reference's Gaussian_smearing returns at once for nsmear 0 and leaves the zeroed
            # output in place, so its loop produces a zero propagator
            assert not b.any()
        else:
            assert rel(a, b) < 1e-9
