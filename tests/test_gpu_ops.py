"""GPU parity of the FP64 operators, BLAS, link generator and the reference CG
against the oracle and the reference's golden vectors, through the C ABI.
FP64 tolerance: 1e-13 relative (the parity bar for the FP64 operators)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel

pytestmark = pytest.mark.gpu

TOL = 1e-13
LATTICES = [(4, 4, 4, 8), (8, 8, 8, 16), (6, 4, 2, 10), (2, 2, 2, 2)]


def _inputs(O, L, eps, seed_u, seed_psi, bc=True):
    U = O.gauge_random(L, eps, seed_u)
    if bc:
        U = O.apply_bc(L, U, -1)
    return U, O.spinor_gaussian(L, seed_psi)


@pytest.fixture(scope="module")
def lattices(qkx):
    made = {}

    def get(L, kappa=0.16, mu=0.01, ts=1):
        key = tuple(L)
        if key not in made:
            made[key] = qkx.Lattice(qkx.LatticeInfo(L=L, kappa=kappa, mu=mu, twistSign=ts))
        lat = made[key]
        lat.set_params(kappa=kappa, mu=mu, twistSign=ts)
        return lat

    yield get
    for lat in made.values():
        lat.close()


@pytest.mark.parametrize("L", LATTICES)
def test_all_operators_match_oracle(qkx, oracle, lattices, L):
    U, psi = _inputs(oracle, L, 0.3, 100 + L[3], 200 + L[3])
    for ts in (1, -1):
        lat = lattices(L, 0.1615, 0.004, ts)
        lat.load_gauge(U, qkx.LINKS_AS_GIVEN)
        for op in oracle.REF_OPS:
            got = lat.apply(op, psi)
            exp = oracle.apply(op, L, U, psi, 0.1615, 0.004, ts)
            assert rel(got, exp) < TOL, (L, op, ts, rel(got, exp))


def test_chiral_extras_match_gamma5_trick(qkx, oracle, lattices):
    """tm_dag_chiral / tm_dagtm_chiral (no reference member) equal g5 M(-s) g5 (M)."""
    L = (4, 4, 4, 8)
    U, psi = _inputs(oracle, L, 0.3, 5, 6)
    lat = lattices(L, 0.16, 0.02, 1)
    lat.load_gauge(U)
    exp = oracle.apply("gamma5_chiral", L, U, oracle.apply(
        "tm_chiral", L, U, oracle.apply("gamma5_chiral", L, U, psi), 0.16, 0.02, -1))
    assert rel(lat.apply("tm_dag_chiral", psi), exp) < TOL
    exp2 = oracle.apply("gamma5_chiral", L, U, oracle.apply(
        "tm_chiral", L, U, oracle.apply("gamma5_chiral", L, U, oracle.apply("tm_chiral", L, U, psi, 0.16, 0.02, 1)),
        0.16, 0.02, -1))
    assert rel(lat.apply("tm_dagtm_chiral", psi), exp2) < TOL


def test_operators_match_reference_golden(qkx, oracle, lattices):
    """Straight against the outputs of the reference's own code (tests/golden)."""
    g = np.load(os.path.join(GOLDEN, "ref_ops_small.npz"))
    L = tuple(int(v) for v in g["L"])
    U, psi = _inputs(oracle, L, float(g["eps"]), int(g["seed_u"]), int(g["seed_psi"]))
    for key in g.files:
        if "@" not in key:
            continue
        op, ts = key.split("@")
        lat = lattices(L, float(g["kappa"]), float(g["mu"]), int(ts))
        lat.load_gauge(U)
        assert rel(lat.apply(op, psi), g[key]) < TOL, key


def test_boundary_modes(qkx, oracle, lattices):
    """APPLY_BC on raw links == AS_GIVEN on links that carry the sign, and the
    links the library reports are the reference's applyBoundaryCondition output."""
    L = (4, 4, 4, 8)
    Uraw = oracle.gauge_random(L, 0.3, 9)
    Ubc = oracle.apply_bc(L, Uraw, -1)
    psi = oracle.spinor_gaussian(L, 10)
    lat = lattices(L)
    lat.load_gauge(Uraw, qkx.LINKS_APPLY_BC)
    a = lat.apply("tm", psi)
    assert np.array_equal(lat.download_gauge(), Ubc)
    assert lat.compressible()
    lat.load_gauge(Ubc, qkx.LINKS_AS_GIVEN)
    b = lat.apply("tm", psi)
    assert lat.compressible()
    assert rel(a, b) == 0.0
    assert rel(b, oracle.apply("tm", L, Ubc, psi)) < TOL
    # periodic operator when the links carry no sign
    lat.load_gauge(Uraw, qkx.LINKS_AS_GIVEN)
    assert rel(lat.apply("tm", psi), oracle.apply("tm", L, Uraw, psi)) < TOL


def test_non_su3_links_are_not_compressed(qkx, oracle, lattices):
    L = (4, 4, 4, 8)
    U = oracle.gauge_random(L, 0.3, 12) * 1.01
    lat = lattices(L)
    lat.load_gauge(U)
    assert not lat.compressible()
    psi = oracle.spinor_gaussian(L, 13)
    assert rel(lat.apply("tm", psi), oracle.apply("tm", L, U, psi)) < TOL


def test_device_generator_matches_oracle(qkx, oracle, lattices):
    L = (4, 4, 4, 8)
    lat = lattices(L)
    lat.generate_gauge(0.3, 1234, qkx.LINKS_AS_GIVEN)
    Ud = lat.download_gauge()
    Uo = oracle.gauge_random(L, 0.3, 1234)
    assert np.abs(Ud - Uo).max() < 1e-13
    lat.generate_gauge(0.3, 1234, qkx.LINKS_APPLY_BC)
    assert np.abs(lat.download_gauge() - oracle.apply_bc(L, Uo, -1)).max() < 1e-13


def test_blas_match_oracle(qkx, oracle, lattices):
    L = (8, 8, 8, 16)
    lat = lattices(L)
    x = oracle.spinor_gaussian(L, 1)
    y = oracle.spinor_gaussian(L, 2)
    dx, dy = lat.field(x), lat.field(y)
    np.testing.assert_allclose(lat.reCdotXdagY(dx, dy), oracle.re_dot(x, y), rtol=1e-12)
    np.testing.assert_allclose(lat.norm2(dx), oracle.norm2(x), rtol=1e-13)
    lat.X_eq_X_p_aY(dx, 0.37, dy)
    x1 = x.copy()
    oracle.axpy(0.37, y, x1)
    assert rel(dx.download(), x1) < 1e-15
    lat.X_eq_aX_p_Y(dx, -0.41, dy)
    oracle.xpay(-0.41, y, x1)
    assert rel(dx.download(), x1) < 1e-15
    # device-resident operator equals the host-buffer one
    dz = lat.field()
    U, _ = _inputs(oracle, L, 0.3, 3, 4)
    lat.load_gauge(U)
    lat.apply_dev("tm_dagtm", dy, dz)
    assert rel(dz.download(), lat.apply("tm_dagtm", y)) == 0.0
    for f in (dx, dy, dz):
        f.close()


def test_blas_reduction_is_deterministic(qkx, oracle, lattices):
    L = (8, 8, 8, 16)
    lat = lattices(L)
    x = lat.field(oracle.spinor_gaussian(L, 7))
    y = lat.field(oracle.spinor_gaussian(L, 8))
    vals = {lat.reCdotXdagY(x, y) for _ in range(5)}
    assert len(vals) == 1


@pytest.mark.parametrize("tag", ["4x4x4x8", "8x8x8x16"])
def test_reference_cg_replica(qkx, oracle, lattices, tag):
    """qkx_cg reproduces CG::operator(): same iteration count, same solution to
    rounding, same r2 stopping rule (golden from the reference)."""
    g = np.load(os.path.join(GOLDEN, "ref_cg.npz"))
    L = tuple(int(v) for v in g[f"{tag}:L"])
    su, sb = (int(v) for v in g[f"{tag}:seeds"])
    U, b = _inputs(oracle, L, float(g["eps"]), su, sb)
    k, mu = float(g["kappa"]), float(g["mu"])
    lat = lattices(L, k, mu, 1)
    lat.set_params(tol=1e-10, maxIter=1000)
    lat.load_gauge(U)
    Mdb = lat.tmDag(b)
    x, info = lat.cg(Mdb)
    assert info.converged == 1
    assert abs(info.iterations - int(g[f"{tag}:iters_oracle"][0])) <= 1
    sites = np.unique(np.linspace(0, oracle.volume(L) - 1, 16).astype(np.int64))
    assert rel(x[sites], g[f"{tag}:x_sites"]) < 1e-9
    np.testing.assert_allclose(np.sum(x * x), g[f"{tag}:x_norm2"][0], rtol=1e-9)


def test_cg_accumulates_into_x(qkx, oracle, lattices):
    """Like the reference, CG adds the solution to the incoming x."""
    L = (4, 4, 4, 8)
    U, b = _inputs(oracle, L, 0.3, 50, 51)
    lat = lattices(L, 0.16, 0.01, 1)
    lat.set_params(tol=1e-8, maxIter=500)
    lat.load_gauge(U)
    x0 = oracle.spinor_gaussian(L, 52)
    x1, _ = lat.cg(b)
    x2, _ = lat.cg(b, x0)
    assert rel(x2 - x0, x1) < 1e-12


def test_invert_fp64_true_residual(qkx, oracle, lattices):
    L = (8, 8, 8, 16)
    U, b = _inputs(oracle, L, 0.3, 60, 61)
    lat = lattices(L, 0.16, 0.01, 1)
    lat.load_gauge(U)
    xs, info = lat.invert([b], method=qkx.SOLVER_CG_FP64, tol=1e-10)
    r = b - oracle.apply("tm", L, U, xs[0], 0.16, 0.01)
    tr = np.sqrt(np.sum(r * r) / np.sum(b * b))
    assert tr <= 1e-10
    assert info.true_residual <= 1e-10
    np.testing.assert_allclose(info.true_residual, tr, rtol=1e-3)


def test_errors_are_status_codes(qkx, oracle):
    L = (4, 4, 4, 4)
    with qkx.Lattice(qkx.LatticeInfo(L=L)) as lat:
        with pytest.raises(qkx.QkxError) as e:
            lat.apply("tm", oracle.spinor_gaussian(L, 1))
        assert e.value.code == qkx.ERR_NOGAUGE
        import ctypes as C
        psi = oracle.spinor_gaussian(L, 1)
        out = np.empty_like(psi)
        assert qkx.lib().qkx_apply(lat.ctx, 999, psi.ctypes.data, out.ctypes.data) == qkx.ERR_INVALID
        assert qkx.lib().qkx_set_params(lat.ctx, C.byref(qkx.LatticeInfo(L=(4, 4, 4, 8)).to_c())) == \
            qkx.ERR_INVALID


# Row widths W = L0/2 from 1 to 16 (12W threads a block: 12, 48, 72, 144 leave the last warp
# partial), y extents that are multiples of the four-row tile, extents of 2 in z and t (the
# +-z and +-t planes coincide)
TILED = [(2, 4, 2, 2), (4, 4, 4, 8), (6, 4, 2, 10), (8, 8, 8, 16), (12, 4, 2, 4), (16, 4, 4, 4),
         (24, 4, 2, 2), (32, 4, 2, 2)]


@pytest.mark.parametrize("L", TILED)
def test_tiled_fp64_hop_matches_direct_kernel(qkx, oracle, monkeypatch, L):
    """The FP64 hop on TMA-staged row tiles (QKX_FP64_TILED=1, where L0 <= 32 and Ly % 4 == 0)
    against the direct kernel (the default) and the oracle, every operator."""
    U, psi = _inputs(oracle, L, 0.3, 300 + L[0], 400 + L[3])
    monkeypatch.setenv("QKX_FP64_TILED", "0")
    direct = qkx.Lattice(qkx.LatticeInfo(L=L, kappa=0.1615, mu=0.004, twistSign=1))
    monkeypatch.setenv("QKX_FP64_TILED", "1")
    tiled = qkx.Lattice(qkx.LatticeInfo(L=L, kappa=0.1615, mu=0.004, twistSign=1))
    try:
        for lat in (direct, tiled):
            lat.load_gauge(U, qkx.LINKS_AS_GIVEN)
        for op in oracle.REF_OPS:
            a, b = tiled.apply(op, psi), direct.apply(op, psi)
            assert rel(a, b) <= 1e-15, (L, op, rel(a, b))
            assert rel(a, oracle.apply(op, L, U, psi, 0.1615, 0.004, 1)) < TOL, (L, op)
    finally:
        direct.close()
        tiled.close()


@pytest.mark.parametrize("prec", ["half", "double"])
def test_tiled_fp64_hop_in_the_mixed_solver(qkx, oracle, monkeypatch, prec):
    """Batched right-hand sides through the reliable updates and the final reconstruction
    (FP64 hops with residual and norm epilogues): tiled and direct kernels give the same
    solutions to the solver's accuracy, each to 1e-10 in the true residual."""
    L = (16, 8, 4, 8)
    U = oracle.apply_bc(L, oracle.gauge_random(L, 0.3, 777), -1)
    bs = [oracle.spinor_gaussian(L, 30 + i) for i in range(3)]
    p = {"half": qkx.PREC_HALF, "double": qkx.PREC_DOUBLE}[prec]
    out = {}
    for mode in ("0", "1"):
        monkeypatch.setenv("QKX_FP64_TILED", mode)
        with qkx.Lattice(qkx.LatticeInfo(L=L, kappa=0.1615, mu=0.004, twistSign=1)) as lat:
            lat.load_gauge(U)
            xs, info = lat.invert(bs, method=qkx.SOLVER_CG_EO_MIXED, precision=p, tol=1e-10)
        assert info.converged == 1
        for x, b in zip(xs, bs):
            r = b - oracle.apply("tm", L, U, x, 0.1615, 0.004, 1)
            assert np.sqrt(np.sum(r * r) / np.sum(b * b)) <= 1e-10
        out[mode] = xs
    for a, b in zip(out["0"], out["1"]):
        assert rel(a, b) < 1e-8
