"""GPU parity of the gauge-side stencils and the propagator workflow through the
C ABI: plaquette, SU(3) projection, APE smearing, Gaussian smearing (batched),
absorbVector and the smeared-source propagator, against the oracle and the
golden vectors made from the reference.

Tolerances (FP64): plaquette 1e-13 relative; Gaussian smearing 1e-13
relative; absorbVector exact.  The SU(3) projection follows the reference's
closed-form eigen-decomposition, which is ill-conditioned when the singular
values of M are close (APE-smeared links: spread ~1e-3 of their size) or one
is small: a difference of one rounding in M (FMA contraction on the GPU, the
order of the staple sums) comes out as up to ~1e-13 in the projected link
after one APE step and up to ~1e-11 after 20, the same size as the
oracle-vs-reference differences.  The propagator is compared at the solver
tolerance."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, oracle_propagator, rel

pytestmark = pytest.mark.gpu


def _golden():
    return np.load(os.path.join(GOLDEN, "ref_smear.npz"))


def _perturbed(O, L, U, scale, seed):
    g = np.concatenate([O.spinor_gaussian(L, seed + k).reshape(-1, 24) for k in range(3)], axis=1)
    return U + scale * g.reshape(U.shape)


@pytest.fixture(scope="module")
def lat48(qkx):
    lat = qkx.Lattice(qkx.LatticeInfo(L=(4, 4, 4, 8), kappa=0.16, mu=0.01))
    yield lat
    lat.close()


@pytest.mark.parametrize("L", [(4, 4, 4, 8), (6, 4, 2, 10), (8, 8, 8, 16)])
def test_plaquette(qkx, oracle, L):
    U = oracle.gauge_random(L, 0.3, 300 + L[3])
    Ubc = oracle.apply_bc(L, U, -1)
    with qkx.Lattice(qkx.LatticeInfo(L=L)) as lat:
        assert rel(lat.plaquette(U), oracle.plaquette_ref(L, U)) < 1e-13
        lat.load_gauge(U, qkx.LINKS_APPLY_BC)
        assert rel(lat.plaquette(), oracle.plaquette_ref(L, Ubc)) < 1e-13
        with pytest.raises(qkx.QkxError) as e:
            lat.plaquette(which=qkx.LINKS_SMEARING)
        assert e.value.code == qkx.ERR_NOGAUGE


def test_plaquette_golden(qkx, oracle, lat48):
    g = _golden()
    L = (4, 4, 4, 8)
    U = oracle.gauge_random(L, float(g["eps"]), int(g["seed_u"]))
    assert rel(lat48.plaquette(U), g["plaq"][0]) < 1e-13
    assert rel(lat48.plaquette(oracle.apply_bc(L, U, -1)), g["plaq_bc"][0]) < 1e-13
    # unit links: plaquette exactly 1
    assert lat48.plaquette(oracle.gauge_unit(L)) == pytest.approx(1.0, abs=1e-15)


def test_project_su3(qkx, oracle, lat48):
    g = _golden()
    L = (4, 4, 4, 8)
    U = oracle.gauge_random(L, float(g["eps"]), int(g["seed_u"]))
    M = _perturbed(oracle, L, U, 0.3, int(g["seed_pert"]))
    P = lat48.project_su3(M)
    exp = M.copy()
    exp[:, :3] = oracle.su3_project(M[:, :3])
    assert np.array_equal(P[:, 3], M[:, 3])
    assert np.abs(P - exp).max() < 1e-12
    assert np.abs(P[g["sites"]] - g["proj:sites"]).max() < 1e-12
    # unit links and an already diagonal H go through the reference's shortcut
    D = oracle.gauge_unit(L) * 2.5
    assert np.abs(lat48.project_su3(D)[:, :3] - oracle.gauge_unit(L)[:, :3]).max() < 1e-15


def test_ape_smearing(qkx, oracle, lat48):
    g = _golden()
    L = (4, 4, 4, 8)
    U = oracle.gauge_random(L, float(g["eps"]), int(g["seed_u"]))
    sites = g["sites"]
    alpha = float(g["ape_alpha"])
    for n, tol in ((1, 1e-13), (2, 1e-12)):
        A = lat48.APE_smearing(U, n, alpha)
        assert np.abs(A - oracle.ape_smear(L, U, n, alpha)).max() < tol, n
        assert np.abs(A[sites] - g[f"ape{n}:sites"]).max() < tol, n
    A = lat48.APE_smearing(U, int(g["ape_n"]), alpha)
    assert np.array_equal(A[:, 3], U[:, 3])
    assert np.abs(A - oracle.ape_smear(L, U, int(g["ape_n"]), alpha)).max() < 1e-10
    assert np.abs(A[sites] - g["ape:sites"]).max() < 1e-10
    # the result is kept as the smearing links
    assert rel(lat48.plaquette(which=qkx.LINKS_SMEARING), g["ape:plaq"][0]) < 1e-12
    # nsmear 0 leaves the output untouched (as the reference leaves *this)
    keep = np.full_like(U, 7.0)
    lat48.APE_smearing(U, 0, alpha, out=keep)
    assert (keep == 7.0).all()


@pytest.mark.parametrize("L,nrhs", [((4, 4, 4, 8), 1), ((6, 4, 2, 10), 3), ((8, 8, 8, 16), 5)])
def test_gaussian_smearing(qkx, oracle, L, nrhs):
    U = oracle.gauge_random(L, 0.3, 400 + L[3])
    A = oracle.ape_smear(L, U, 3, 0.5)
    psis = [oracle.spinor_gaussian(L, 500 + k) for k in range(nrhs)]
    with qkx.Lattice(qkx.LatticeInfo(L=L)) as lat:
        with pytest.raises(qkx.QkxError) as e:
            lat.Gaussian_smearing(psis, 2, 4.0)
        assert e.value.code == qkx.ERR_NOGAUGE
        lat.load_smearing_gauge(A)
        for n in (1, 2, 7):
            outs = lat.Gaussian_smearing(psis, n, 4.0)
            for p, o in zip(psis, outs):
                assert rel(o, oracle.gaussian_smear(L, A, p, n, 4.0)) < 1e-13, (L, n)
        keep = [np.full_like(p, 3.0) for p in psis]
        lat.Gaussian_smearing(psis, 0, 4.0, out=keep)
        assert all((k == 3.0).all() for k in keep)


def test_gaussian_smearing_golden(qkx, oracle, lat48):
    g = _golden()
    L = (4, 4, 4, 8)
    U = oracle.gauge_random(L, float(g["eps"]), int(g["seed_u"]))
    psi = oracle.spinor_gaussian(L, int(g["seed_psi"]))
    lat48.APE_smearing(U, int(g["ape_n"]), float(g["ape_alpha"]))
    W = [oracle.spinor_gaussian(L, 9000 + k) for k in range(3)]
    for n in (1, int(g["gauss_n"])):
        (s,) = lat48.Gaussian_smearing([psi], n, float(g["gauss_alpha"]))
        assert rel(s[g["sites"]], g[f"gauss{n}:sites"]) < 1e-11
        np.testing.assert_allclose([np.sum(w * s) for w in W], g[f"gauss{n}:probe"], rtol=1e-9)


def test_gaussian_smearing_dev_rejects_aliasing(qkx, oracle, lat48):
    L = (4, 4, 4, 8)
    lat48.load_smearing_gauge(oracle.gauge_random(L, 0.3, 1))
    f = lat48.field(oracle.spinor_gaussian(L, 2))
    h = lat48.field()
    with pytest.raises(qkx.QkxError) as e:
        lat48.Gaussian_smearing_dev([f], [f], 2, 4.0)
    assert e.value.code == qkx.ERR_INVALID
    lat48.Gaussian_smearing_dev([f], [h], 3, 4.0)
    lat48.sync()
    exp = oracle.gaussian_smear(L, oracle.gauge_random(L, 0.3, 1), oracle.spinor_gaussian(L, 2), 3, 4.0)
    assert rel(h.download(), exp) < 1e-13


def test_absorb_vector(qkx, oracle, lat48):
    L = (4, 4, 4, 8)
    V = oracle.volume(L)
    prop = np.random.default_rng(5).standard_normal((V, 4, 4, 3, 3, 2))
    exp = prop.copy()
    for nu, c2 in ((0, 0), (3, 2), (1, 2)):
        phi = oracle.spinor_gaussian(L, 10 * nu + c2)
        lat48.absorbVector(prop, phi, nu, c2)
        oracle.absorb_vector(phi, nu, c2, exp)
    assert np.array_equal(prop, exp)


@pytest.mark.parametrize("method,prec", [(0, 0), (1, 2), (1, 1)])
def test_propagator_golden(qkx, oracle, method, prec):
    """The propagator of the reference's loop (golden, 4x4x4x8): FP64 CG, and the
    even-odd mixed solver in half and single precision, all to tol 1e-12."""
    g = _golden()
    L = (4, 4, 4, 8)
    U = oracle.gauge_random(L, float(g["eps"]), int(g["seed_u"]))
    src = tuple(int(v) for v in g["prop_src"])
    with qkx.Lattice(qkx.LatticeInfo(L=L, kappa=float(g["kappa"]), mu=float(g["mu"]))) as lat:
        lat.load_gauge(U, qkx.LINKS_APPLY_BC)
        lat.APE_smearing(U, int(g["ape_n"]), float(g["ape_alpha"]))
        prop, info = lat.propagator(src, int(g["prop_n"]), float(g["prop_alpha"]), method=method,
                                    precision=prec, tol=1e-12)
        assert info.converged == 1 and info.true_residual <= 1e-12
        assert rel(prop[g["sites"]], g["prop:sites"]) < 1e-9
        np.testing.assert_allclose(np.sum(prop * prop), g["prop:norm2"][0], rtol=1e-9)


@pytest.mark.parametrize("L,src", [((4, 2, 4, 4), (3, 1, 0, 2)), ((6, 4, 4, 8), (5, 3, 2, 7))])
def test_propagator_vs_oracle(qkx, oracle, L, src):
    U = oracle.gauge_random(L, 0.3, 700 + L[3])
    Ubc = oracle.apply_bc(L, U, -1)
    A = oracle.ape_smear(L, U, 4, 0.5)
    with qkx.Lattice(qkx.LatticeInfo(L=L, kappa=0.1615, mu=0.004)) as lat:
        lat.load_gauge(Ubc, qkx.LINKS_AS_GIVEN)
        with pytest.raises(qkx.QkxError) as e:
            lat.propagator(src, 3, 4.0)
        assert e.value.code == qkx.ERR_NOGAUGE
        lat.load_smearing_gauge(A)
        for nsmear in (0, 3):
            prop, info = lat.propagator(src, nsmear, 4.0, tol=1e-12)
            exp = oracle_propagator(oracle, L, Ubc, A, 0.1615, 0.004, nsmear, 4.0, src, tol=1e-12)
            assert rel(prop, exp) < 1e-9, (L, nsmear, rel(prop, exp))


def test_propagator_argument_checks(qkx, lat48):
    with pytest.raises(qkx.QkxError) as e:
        lat48.propagator((4, 0, 0, 0), 0, 4.0)
    assert e.value.code == qkx.ERR_INVALID
    with pytest.raises(qkx.QkxError) as e:
        lat48.propagator((0, 0, 0, 0), -1, 4.0)
    assert e.value.code == qkx.ERR_INVALID
