"""GPU parity at the sizes of the benchmark configurations, every solution's true
residual ||b - M x|| / ||b|| recomputed by the oracle's FP64 operator (the
reference's Vector::tm, lib/lattice_util.cpp:1925) unless stated otherwise.

  mixed EO   24^3x48, kappa 0.1615, mu 0.004, one Gaussian source: the mixed
             even-odd solver (FP16 and FP32 sloppy) and the plain FP64 CG of the
             reference's algorithm (lib/solvers.cpp:16-81) both reach 1e-10, and
             their solutions agree to 1e-6 relative (condition number x 1e-10)
  12 sources 32^3x64, kappa 0.1615, mu 0.0015, the 12 spin-colour point sources
             in one batch; three of the twelve solutions checked by the oracle
  uneven     one job of 4 Gaussian sources on each of 16^3x32, 20^3x40, 24^3x48,
             32^3x64 (own links, eps in [0.2, 0.35], mu in {0.0015, 0.004, 0.01});
             every job's FP64 true residual as the library reports it, and the
             16^3x32 job's solutions by the oracle
  learned    32^3x64 with the learned preconditioner after a short training run,
             flexible CG on two point sources

Tolerance: 1e-10 on every true residual, as the solves are asked for."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10


def true_residual(O, L, U, b, x, kappa, mu):
    r = b - O.apply("tm", L, U, x, kappa, mu, 1)
    return float(np.linalg.norm(r) / np.linalg.norm(b))


def point_source(L, spin, colour):
    V = L[0] * L[1] * L[2] * L[3]
    b = np.zeros((V, 4, 3, 2))
    b[0, spin, colour, 0] = 1.0
    return b


def test_mixed_eo_against_plain_fp64_at_24x48(qkx, oracle):
    L, kappa, mu = (24, 24, 24, 48), 0.1615, 0.004
    U = oracle.apply_bc(L, oracle.gauge_random(L, 0.3, 1234), -1)
    b = oracle.spinor_gaussian(L, 2402)
    with qkx.Lattice(qkx.LatticeInfo(L=L, kappa=kappa, mu=mu, twistSign=1)) as lat:
        lat.load_gauge(U, qkx.LINKS_AS_GIVEN)
        (x64,), i64 = lat.invert([b], method=qkx.SOLVER_CG_FP64, tol=TOL, maxIter=5000)
        assert i64.converged == 1 and i64.true_residual <= TOL
        assert true_residual(oracle, L, U, b, x64, kappa, mu) <= TOL
        for prec in (qkx.PREC_HALF, qkx.PREC_SINGLE):
            (xm,), im = lat.invert([b], method=qkx.SOLVER_CG_EO_MIXED, precision=prec, tol=TOL)
            assert im.converged == 1 and im.true_residual <= TOL
            assert im.reliable_updates >= 1
            assert true_residual(oracle, L, U, b, xm, kappa, mu) <= TOL
            # both solve the same system to 1e-10; the solutions differ by at most the condition
            # number of M times that (about 1e3 here)
            assert np.linalg.norm(xm - x64) / np.linalg.norm(x64) < 1e-6


def test_twelve_point_sources_at_32x64(qkx, oracle):
    L, kappa, mu = (32, 32, 32, 64), 0.1615, 0.0015
    U = oracle.apply_bc(L, oracle.gauge_random(L, 0.3, 1234), -1)
    bs = [point_source(L, s, c) for s in range(4) for c in range(3)]
    with qkx.Lattice(qkx.LatticeInfo(L=L, kappa=kappa, mu=mu, twistSign=1)) as lat:
        lat.load_gauge(U, qkx.LINKS_AS_GIVEN)
        xs, info = lat.invert(bs, method=qkx.SOLVER_CG_EO_MIXED, precision=qkx.PREC_HALF, tol=TOL)
        assert info.converged == 1 and info.true_residual <= TOL
        for k in (0, 5, 11):  # spin 0 colour 0, spin 1 colour 2, spin 3 colour 2
            assert true_residual(oracle, L, U, bs[k], xs[k], kappa, mu) <= TOL, k


def test_uneven_instances_at_benchmark_sizes(qkx, oracle):
    rng = np.random.default_rng(4040)
    shapes = [(16, 16, 16, 32), (20, 20, 20, 40), (24, 24, 24, 48), (32, 32, 32, 64)]
    mus = [0.0015, 0.004, 0.01]
    kappa = 0.1615
    lats, jobs, checks = [], [], None
    try:
        for i, L in enumerate(shapes):
            eps = float(rng.uniform(0.2, 0.35))
            U = oracle.apply_bc(L, oracle.gauge_random(L, eps, 500 + i), -1)
            lat = qkx.Lattice(qkx.LatticeInfo(L=L, kappa=kappa, mu=0.01))
            lat.load_gauge(U, qkx.LINKS_AS_GIVEN)
            lats.append(lat)
            bs = [oracle.spinor_gaussian(L, 600 + 10 * i + k) for k in range(4)]
            bd = [lat.field(b) for b in bs]
            xd = [lat.field() for _ in bs]
            mu = [mus[(i + k) % 3] for k in range(4)]
            jobs.append((lat, bd, xd, mu))
            if i == 0:
                checks = (L, U, bs, xd, mu)
        res = qkx.invert_batch(jobs, tol=TOL)
        for r in res:
            assert r["status"] == qkx.OK, r["message"]
            assert r["info"]["converged"] == 1 and r["info"]["true_residual"] <= TOL
        L, U, bs, xd, mu = checks
        for b, x, m in zip(bs, xd, mu):
            assert true_residual(oracle, L, U, b, x.download(), kappa, m) <= TOL
    finally:
        for _, bd, xd, _ in jobs:
            for f in bd + xd:
                f.close()
        for lat in lats:
            lat.close()


def test_learned_preconditioner_at_32x64(qkx, oracle):
    L, kappa, mu = (32, 32, 32, 64), 0.1615, 0.0015
    U = oracle.apply_bc(L, oracle.gauge_random(L, 0.3, 1234), -1)
    bs = [point_source(L, 0, 0), point_source(L, 2, 1)]
    with qkx.Lattice(qkx.LatticeInfo(L=L, kappa=kappa, mu=mu, twistSign=1)) as lat:
        lat.load_gauge(U, qkx.LINKS_AS_GIVEN)
        net = qkx.Ptc(lat, (4, 16, 16, 16, 4), seed=3, init_scale=0.05, tensor_cores=True)
        try:
            train = net.train(n_solves=4, steps=40, lr=3e-3, solve_tol=1e-6, seed=9)
            assert train["loss_final"] < train["loss_initial"]
            xs, info = lat.invert(bs, method=qkx.SOLVER_GCR_PTC, tol=TOL, preconditioner=net)
            assert info.converged == 1 and info.true_residual <= TOL
            for b, x in zip(bs, xs):
                assert true_residual(oracle, L, U, b, x, kappa, mu) <= TOL
        finally:
            net.close()
