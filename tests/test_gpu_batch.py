"""GPU test of the batched uneven-instance solve (qkx_invert_batch): several
lattices, each with its own seeded links and twisted masses, several jobs of a
few right-hand sides each, run concurrently; every solution checked by the
oracle's FP64 operator to the true-residual target."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_uneven_batch(qkx, oracle):
    specs = [((4, 4, 4, 8), 0.22, 11), ((6, 6, 6, 12), 0.3, 12), ((8, 8, 8, 16), 0.35, 13)]
    mus = [0.0015, 0.004, 0.01]
    lats, gauges, jobs, fields = [], [], [], []
    for L, eps, seed in specs:
        U = oracle.apply_bc(L, oracle.gauge_random(L, eps, seed), -1)
        lat = qkx.Lattice(qkx.LatticeInfo(L=L, kappa=0.16, mu=0.01))
        lat.load_gauge(U, qkx.LINKS_AS_GIVEN)
        lats.append(lat)
        gauges.append(U)
        for j in range(2):  # two jobs of 3 RHS per lattice
            bs = [oracle.spinor_gaussian(L, 100 * seed + 10 * j + k) for k in range(3)]
            bd = [lat.field(b) for b in bs]
            xd = [lat.field() for _ in bs]
            mu = [mus[(j + k) % 3] for k in range(3)]
            jobs.append((lat, bd, xd, mu))
            fields.append((len(lats) - 1, bs, xd, mu))
    res = qkx.invert_batch(jobs, tol=1e-10)
    assert all(r["status"] == qkx.OK for r in res)
    assert all(r["info"]["converged"] == 1 for r in res)
    for (li, bs, xd, mu), r in zip(fields, res):
        L = specs[li][0]
        for b, x, m in zip(bs, xd, mu):
            xv = x.download()
            rr = b - oracle.apply("tm", L, gauges[li], xv, 0.16, m)
            assert np.linalg.norm(rr) / np.linalg.norm(b) <= 1e-10
    # jobs of one lattice finish in order; every latency is positive
    for li in range(len(specs)):
        lat_res = [r["latency"] for r, f in zip(res, fields) if f[0] == li]
        assert lat_res == sorted(lat_res) and lat_res[0] > 0
    for _, _, xd, _ in fields:
        for x in xd:
            x.close()
    for lat in lats:
        lat.close()


def test_uneven_batch_one_graph_and_threaded_paths(qkx, oracle):
    """The same jobs through the one-graph path (the default for the mixed solver) and through
    the thread-per-lattice path (graphs off): both reach the target on every right-hand side,
    each job's reported residual is the worst of its own right-hand sides, and in the graph
    path the jobs of a lattice end together (one batch per lattice)."""
    specs = [((8, 8, 8, 16), 0.3, 21), ((4, 4, 4, 8), 0.25, 22)]
    lats, gauges, jobs, fields = [], [], [], []
    for L, eps, seed in specs:
        U = oracle.apply_bc(L, oracle.gauge_random(L, eps, seed), -1)
        lat = qkx.Lattice(qkx.LatticeInfo(L=L, kappa=0.1615, mu=0.004))
        lat.load_gauge(U, qkx.LINKS_AS_GIVEN)
        lats.append(lat)
        gauges.append(U)
        for j in range(2):
            bs = [oracle.spinor_gaussian(L, 1000 * seed + 10 * j + k) for k in range(2)]
            jobs.append((lat, [lat.field(b) for b in bs], [lat.field() for _ in bs], [0.004, 0.01]))
            fields.append((len(lats) - 1, bs))
    try:
        for graphs in (1, 0):
            res = qkx.invert_batch(jobs, tol=1e-10, use_graphs=graphs)
            for r, (li, bs), (_, _, xd, mu) in zip(res, fields, jobs):
                assert r["status"] == qkx.OK and r["info"]["converged"] == 1
                L = specs[li][0]
                worst = 0.0
                for b, x, m in zip(bs, xd, mu):
                    rr = b - oracle.apply("tm", L, gauges[li], x.download(), 0.1615, m)
                    worst = max(worst, np.linalg.norm(rr) / np.linalg.norm(b))
                assert worst <= 1e-10
                assert abs(r["info"]["true_residual"] - worst) <= 1e-3 * worst
            if graphs:
                for li in range(len(specs)):
                    lat_res = [r["latency"] for r, f in zip(res, fields) if f[0] == li]
                    assert len(set(lat_res)) == 1 and lat_res[0] > 0
    finally:
        for _, bd, xd, _ in jobs:
            for f in bd + xd:
                f.close()
        for lat in lats:
            lat.close()


def test_batch_reports_job_errors(qkx, oracle):
    L = (4, 4, 4, 4)
    lat = qkx.Lattice(qkx.LatticeInfo(L=L))  # no gauge field: the job fails
    b = lat.field(oracle.spinor_gaussian(L, 1))
    x = lat.field()
    with pytest.raises(qkx.QkxError) as e:
        qkx.invert_batch([(lat, [b], [x], None)])
    assert "gauge" in str(e.value)
    lat.close()
