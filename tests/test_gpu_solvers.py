"""GPU tests of the solvers: every solve must reach ||b - M x|| / ||b|| <= 1e-10
recomputed in FP64 by the oracle, for the plain FP64 method and the even-odd
mixed-precision method (half, single, double sloppy), batched right-hand
sides, several twisted masses in one batch, and the error paths."""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

TOL = 1e-10


def true_res(O, L, U, x, b, kappa, mu, ts=1):
    r = b - O.apply("tm", L, U, x, kappa, mu, ts)
    return float(np.sqrt(np.sum(r * r) / np.sum(b * b)))


@pytest.fixture(scope="module")
def setup8(qkx, oracle):
    L = (8, 8, 8, 16)
    U = oracle.apply_bc(L, oracle.gauge_random(L, 0.3, 4321), -1)
    lat = qkx.Lattice(qkx.LatticeInfo(L=L, kappa=0.1615, mu=0.004, twistSign=1))
    lat.load_gauge(U)
    yield L, U, lat
    lat.close()


@pytest.mark.parametrize("prec", ["half", "single", "double"])
def test_eo_mixed_reaches_true_residual(qkx, oracle, setup8, prec):
    L, U, lat = setup8
    p = {"half": qkx.PREC_HALF, "single": qkx.PREC_SINGLE, "double": qkx.PREC_DOUBLE}[prec]
    b = oracle.spinor_gaussian(L, 11)
    xs, info = lat.invert([b], method=qkx.SOLVER_CG_EO_MIXED, precision=p, tol=TOL)
    tr = true_res(oracle, L, U, xs[0], b, 0.1615, 0.004)
    assert tr <= TOL, tr
    assert info.converged == 1 and info.true_residual <= TOL
    np.testing.assert_allclose(info.true_residual, tr, rtol=1e-2)
    # same solution as the reference's own method (oracle FP64 CG on M^+M)
    Mdb = oracle.apply("tm_dag", L, U, b, 0.1615, 0.004)
    x_ref, _, _ = oracle.cg(L, U, Mdb, 0.1615, 0.004, tol=1e-12, maxIter=2000)
    assert rel(xs[0], x_ref) < 1e-8


def test_eo_mixed_matches_fp64_method(qkx, oracle, setup8):
    L, U, lat = setup8
    b = oracle.spinor_gaussian(L, 12)
    x1, i1 = lat.invert([b], method=qkx.SOLVER_CG_FP64, tol=TOL)
    x2, i2 = lat.invert([b], method=qkx.SOLVER_CG_EO_MIXED, precision=qkx.PREC_HALF, tol=TOL)
    assert rel(x2[0], x1[0]) < 1e-8
    # the even-odd system converges in fewer iterations than the full normal equations
    assert i2.iterations < i1.iterations


def test_multi_rhs_batch_point_sources(qkx, oracle, setup8):
    """12 spin-colour point sources in one batch; each one to 1e-10."""
    L, U, lat = setup8
    bs = [oracle.spinor_point(L, (0, 0, 0, 0), s, c) for s in range(4) for c in range(3)]
    xs, info = lat.invert(bs, method=qkx.SOLVER_CG_EO_MIXED, precision=qkx.PREC_HALF, tol=TOL)
    assert info.converged == 1
    for b, x in zip(bs, xs):
        assert true_res(oracle, L, U, x, b, 0.1615, 0.004) <= TOL


def test_batch_equals_single_solves(qkx, oracle, setup8):
    L, U, lat = setup8
    bs = [oracle.spinor_gaussian(L, 20 + i) for i in range(3)]
    xb, _ = lat.invert(bs, method=qkx.SOLVER_CG_EO_MIXED, precision=qkx.PREC_SINGLE, tol=TOL)
    for b, x in zip(bs, xb):
        xs, _ = lat.invert([b], method=qkx.SOLVER_CG_EO_MIXED, precision=qkx.PREC_SINGLE, tol=TOL)
        assert rel(x, xs[0]) < 1e-8


def test_multi_mass_batch(qkx, oracle, setup8):
    """Several twisted masses in one batch: each RHS solves its own M(mu_i)."""
    import ctypes as C
    L, U, lat = setup8
    mus = [0.0015, 0.004, 0.01]
    bs = [oracle.spinor_gaussian(L, 30 + i) for i in range(3)]
    xs = [np.empty_like(b) for b in bs]
    n = len(bs)
    arr = (C.c_double * n)(*mus)
    sp = qkx.SolverParams(qkx.SOLVER_CG_EO_MIXED, qkx.PREC_HALF, TOL, 10000, 0.0, 1,
                          C.cast(arr, C.POINTER(C.c_double)))
    info = qkx.SolveInfo()
    bp = (C.c_void_p * n)(*[b.ctypes.data for b in bs])
    xp = (C.c_void_p * n)(*[x.ctypes.data for x in xs])
    qkx.check(qkx.lib().qkx_invert(lat.ctx, C.byref(sp), n, bp, xp, C.byref(info)))
    for mu, b, x in zip(mus, bs, xs):
        assert true_res(oracle, L, U, x, b, 0.1615, mu) <= TOL


@pytest.mark.parametrize("prec", ["half", "double"])
def test_device_loop_host_loop_and_eager_agree_bitwise(qkx, oracle, setup8, prec):
    """The three drivers of the mixed solve take the same decisions from the same scalars and
    launch the same kernels in the same order: the whole loop as one graph with conditional
    nodes (the default), one graph per iteration with the decisions on the host (taken while
    the hop kernels are timed), and eager launches.  Same iterations, reliable updates and
    restarts, bit-identical solutions, for a batch with a twisted mass per right-hand side."""
    L, U, lat = setup8
    P = {"half": qkx.PREC_HALF, "double": qkx.PREC_DOUBLE}[prec]
    bs = [oracle.spinor_gaussian(L, 40 + i) for i in range(3)]
    runs = []
    for graphs, prof in ((1, False), (1, True), (0, False)):
        lat.profile(prof)
        try:
            xs, info = lat.invert(bs, precision=P, tol=TOL, use_graphs=graphs)
        finally:
            lat.profile(False)
        runs.append((xs, info))
    (xd, idv), (xh, ih), (xe, ie) = runs
    for i in (ih, ie):
        assert (i.iterations, i.reliable_updates, i.restarts) == (idv.iterations, idv.reliable_updates, idv.restarts)
    for k in range(len(bs)):
        assert np.array_equal(xd[k], xh[k]) and np.array_equal(xd[k], xe[k])
    assert idv.converged == 1 and idv.true_residual <= TOL
    assert idv.seconds_reliable > 0 and idv.seconds_setup > 0 and idv.seconds_final > 0


def test_twist_sign_and_periodic_links(qkx, oracle):
    L = (4, 4, 4, 8)
    Uraw = oracle.gauge_random(L, 0.3, 99)
    b = oracle.spinor_gaussian(L, 98)
    for ts, bc in ((-1, -1), (1, 1)):
        with qkx.Lattice(qkx.LatticeInfo(L=L, kappa=0.16, mu=0.01, twistSign=ts, boundaryT=bc)) as lat:
            lat.load_gauge(Uraw, qkx.LINKS_APPLY_BC)
            Uop = oracle.apply_bc(L, Uraw, bc)
            xs, _ = lat.invert([b], precision=qkx.PREC_HALF, tol=TOL)
            assert true_res(oracle, L, Uop, xs[0], b, 0.16, 0.01, ts) <= TOL


def test_zero_source_gives_zero_solution(qkx, oracle, setup8):
    L, U, lat = setup8
    b = np.zeros((oracle.volume(L), 4, 3, 2))
    xs, info = lat.invert([b], precision=qkx.PREC_HALF, tol=TOL)
    assert not np.any(xs[0])
    assert info.converged == 1


def test_non_su3_links_refuse_mixed_precision(qkx, oracle):
    L = (4, 4, 4, 8)
    U = oracle.gauge_random(L, 0.3, 5) * 1.01
    with qkx.Lattice(qkx.LatticeInfo(L=L, kappa=0.16, mu=0.01)) as lat:
        lat.load_gauge(U)
        with pytest.raises(qkx.QkxError) as e:
            lat.invert([oracle.spinor_gaussian(L, 1)], precision=qkx.PREC_HALF, tol=TOL)
        assert e.value.code == qkx.ERR_UNSUPPORTED
        # the FP64 methods still work on them
        xs, _ = lat.invert([oracle.spinor_gaussian(L, 1)], precision=qkx.PREC_DOUBLE, tol=TOL)
        assert true_res(oracle, L, U, xs[0], oracle.spinor_gaussian(L, 1), 0.16, 0.01) <= TOL


def test_maxiter_reports_not_converged(qkx, oracle, setup8):
    L, U, lat = setup8
    b = oracle.spinor_gaussian(L, 50)
    xs, info = lat.invert([b], precision=qkx.PREC_HALF, tol=TOL, maxIter=5, strict=False)
    assert info.converged == 0
    with pytest.raises(qkx.QkxError) as e:
        lat.invert([b], precision=qkx.PREC_HALF, tol=TOL, maxIter=5)
    assert e.value.code == qkx.ERR_NOT_CONVERGED


def test_autotuner_picks_a_tile_and_results_are_unchanged(qkx, oracle, setup8):
    """Every tile computes the same operator: the solve with the tuned tile
    matches a solve with the tile forced to one RHS per thread."""
    L, U, lat = setup8
    nr, nt, ms = lat.tune(qkx.PREC_SINGLE, 5)
    assert nr in (1, 2, 3, 4) and nt in (64, 128, 256) and ms > 0
    bs = [oracle.spinor_gaussian(L, 60 + i) for i in range(5)]
    xa, ia = lat.invert(bs, precision=qkx.PREC_SINGLE, tol=TOL)
    for b, x in zip(bs, xa):
        assert true_res(oracle, L, U, x, b, 0.1615, 0.004) <= TOL


TILES = [(nr, nt, 0) for nr in (1, 2, 3, 4) for nt in (64, 128, 256)]
# FP16 only: two right-hand sides a thread; loads pipelined through registers or shared
# memory, with several register bounds
TILES_F16 = ([(2, nt, k) for k in (1, 2, 4) for nt in (64, 128, 256)] + [(2, 64, 3), (2, 128, 3)] +
             [(2, 64, 5), (2, 128, 5), (2, 64, 6), (2, 64, 7), (2, 128, 7), (2, 64, 8), (2, 128, 8),
              (2, 64, 9), (2, 128, 9), (2, 64, 10), (2, 128, 10), (2, 64, 11), (2, 128, 11)])


@pytest.mark.parametrize("prec,tol", [("half", 1e-2), ("single", 1e-5), ("double", 1e-12)])
def test_sloppy_normal_operator_every_tile(qkx, oracle, setup8, prec, tol):
    """Each hop tile computes tm_xxDagTm_xx(EE) (the mixed solver's A p): the scalar
    kernels for any number of right-hand sides per thread and, in half precision, the
    packed-pair kernels for an even number.  Five right-hand sides, so the last group
    has lanes outside the batch.  Tolerances: input and three intermediate fields
    rounded to FP16 (2^-11 of the site maximum) or FP32; FP64 arithmetic throughout."""
    L, U, lat = setup8
    p = {"half": qkx.PREC_HALF, "single": qkx.PREC_SINGLE, "double": qkx.PREC_DOUBLE}[prec]
    bs = [oracle.spinor_gaussian(L, 80 + i) for i in range(5)]
    exp = [oracle.apply("tm_xx_dagtm_xx_ee", L, U, b, 0.1615, 0.004) for b in bs]
    first = None
    for tile in TILES + (TILES_F16 if prec == "half" else []):
        got = lat.sloppy_normal(bs, p, tile)
        for g, e in zip(got, exp):
            assert rel(g, e) < tol, (prec, tile, rel(g, e))
        if first is None:
            first = got
        else:  # the tiles differ only in the order of the FP rounding
            for g, f in zip(got, first):
                assert rel(g, f) < tol
    for bad in [(5, 64, 0)] + ([] if prec == "half" else [(2, 128, 1)]):
        with pytest.raises(qkx.QkxError) as e:
            lat.sloppy_normal(bs, p, bad)
        assert e.value.code == qkx.ERR_INVALID


@pytest.mark.parametrize("prec,tile", [("half", t) for t in (
    (1, 128, 0), (2, 64, 0), (2, 256, 0), (3, 64, 0), (4, 128, 0), (2, 128, 1), (2, 256, 2), (2, 64, 3), (2, 128, 4),
    (2, 128, 5), (2, 64, 6), (2, 64, 7), (2, 64, 8), (2, 128, 9), (2, 64, 10), (2, 128, 11))] + [
    ("single", (1, 64, 0)), ("single", (2, 128, 0))])
def test_every_tile_solves_a_multi_mass_batch(qkx, oracle, setup8, prec, tile):
    """Solves with the tile forced: three masses in a batch of five, so right-hand sides
    leave the batch at different iterations (the per-RHS active mask) and the last
    group of the tile is partly outside the batch."""
    import ctypes as C
    L, U, lat = setup8
    p = {"half": qkx.PREC_HALF, "single": qkx.PREC_SINGLE}[prec]
    mus = [0.0015, 0.01, 0.004, 0.02, 0.0015]
    bs = [oracle.spinor_gaussian(L, 90 + i) for i in range(5)]
    xs = [np.empty_like(b) for b in bs]
    n = len(bs)
    lat.set_tile(p, n, tile)
    arr = (C.c_double * n)(*mus)
    sp = qkx.SolverParams(qkx.SOLVER_CG_EO_MIXED, p, TOL, 10000, 0.0, 1,
                          C.cast(arr, C.POINTER(C.c_double)))
    info = qkx.SolveInfo()
    bp = (C.c_void_p * n)(*[b.ctypes.data for b in bs])
    xp = (C.c_void_p * n)(*[x.ctypes.data for x in xs])
    qkx.check(qkx.lib().qkx_invert(lat.ctx, C.byref(sp), n, bp, xp, C.byref(info)))
    assert info.converged == 1
    for mu, b, x in zip(mus, bs, xs):
        assert true_res(oracle, L, U, x, b, 0.1615, mu) <= TOL
    with pytest.raises(qkx.QkxError) as e:
        lat.set_tile(qkx.PREC_HALF, n, (2, 100, 0))
    assert e.value.code == qkx.ERR_INVALID


def test_reliable_delta_below_the_half_precision_limit_is_clamped(qkx, oracle, setup8):
    """A reliable_delta too small for FP16 storage (1e-3 made a 32^3x64 batch diverge) is
    raised to the half-precision minimum: the solve converges like the default one."""
    L, U, lat = setup8
    bs = [oracle.spinor_gaussian(L, 700 + i) for i in range(2)]
    xs, info = lat.invert(bs, method=qkx.SOLVER_CG_EO_MIXED, precision=qkx.PREC_HALF, tol=TOL,
                          reliable_delta=1e-6)
    for b, x in zip(bs, xs):
        assert true_res(oracle, L, U, x, b, 0.1615, 0.004) <= TOL
    assert info.converged == 1 and info.true_residual <= TOL


def test_solve_info_phases(qkx, oracle, setup8):
    """CG_EO_MIXED reports the device time of its set-up, reliable updates and final residual,
    each inside the solve's total; the plain FP64 method leaves them zero."""
    L, U, lat = setup8
    bs = [oracle.spinor_gaussian(L, 800 + i) for i in range(3)]
    _, info = lat.invert(bs, method=qkx.SOLVER_CG_EO_MIXED, precision=qkx.PREC_HALF, tol=TOL)
    parts = (info.seconds_setup, info.seconds_reliable, info.seconds_final)
    assert all(t > 0 for t in parts), parts
    assert sum(parts) < info.seconds
    assert info.reliable_updates >= 1 and info.restarts >= 0
    _, info64 = lat.invert(bs[:1], method=qkx.SOLVER_CG_FP64, tol=TOL)
    assert (info64.seconds_setup, info64.seconds_reliable, info64.seconds_final) == (0.0, 0.0, 0.0)
    assert info64.seconds > 0
