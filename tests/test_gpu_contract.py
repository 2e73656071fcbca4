"""GPU parity of the two-point contractions (qkx_meson_2pt / qkx_baryon_2pt /
qkx_delta_2pt / qkx_nucleon_2pt: lib/contractions.cpp Meson/Baryon/Baryon_Dec::contract
+ fourier, contractNucleon of lib/lattice_util.cpp) against the oracle and
the golden vectors from the reference.  FP64; the GPU sums the Fourier
transform in a different order and contracts complex products with FMA, so the
bar is 1e-12 relative to the largest correlator entry."""
import ctypes as C
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu
sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from make_golden import seeded_propagator  # noqa: E402

TOL = 1e-12


def _close(a, b):
    return np.abs(a - b).max() <= TOL * max(np.abs(b).max(), 1e-300)


def test_golden(qkx):
    g = np.load(os.path.join(GOLDEN, "ref_contract.npz"))
    L = tuple(int(v) for v in g["L"])
    p1, p2 = seeded_propagator(L, int(g["seed1"])), seeded_propagator(L, int(g["seed2"]))
    Q, xs = int(g["Q_sq"]), tuple(int(v) for v in g["x_src"])
    assert np.array_equal(qkx.momenta(Q), g["momenta"])
    with qkx.Lattice(qkx.LatticeInfo(L=L)) as lat:
        m = lat.meson_2pt(p1, range(10), Q, xs)
        for op, name in enumerate(qkx.MESONS):
            assert _close(m[op], g[f"meson:{name}"]), name
        for op, name in enumerate(qkx.BARYONS):
            assert _close(lat.baryon_2pt(p1, p2, op, Q, xs), g[f"baryon:{name}"]), name
        for op, name in enumerate(qkx.DELTAS):
            assert _close(lat.delta_2pt(p1, p2, op, Q, xs), g[f"delta:{name}"]), name
        n = lat.nucleon_2pt(p1, p2, Q, xs)
        assert _close(n, g["baryon:NTN"])
        assert np.abs(n - g["nucleon_text"]).max() <= 1e-6 * np.abs(n).max()


@pytest.mark.parametrize("L,Q,xs", [((4, 4, 4, 8), 0, (0, 0, 0, 0)), ((6, 4, 2, 10), 1, (5, 3, 1, 9)),
                                    ((8, 8, 8, 16), 4, (2, 7, 1, 3))])
def test_vs_oracle(qkx, oracle, L, Q, xs):
    p1, p2 = seeded_propagator(L, 100 + L[3]), seeded_propagator(L, 200 + L[3])
    with qkx.Lattice(qkx.LatticeInfo(L=L)) as lat:
        ops = [1, 0, 7] if L[0] == 8 else list(range(10))
        m = lat.meson_2pt(p1, ops, Q, xs)
        for i, op in enumerate(ops):
            assert _close(m[i], oracle.meson_2pt(L, p1, op, Q, xs)), (L, op)
        for op in (range(4) if L[0] != 8 else (0, 3)):
            assert _close(lat.baryon_2pt(p1, p2, op, Q, xs), oracle.baryon_2pt(L, p1, p2, op, Q, xs)), (L, op)
        if L[0] != 8:  # the decuplet oracle is slow: 48 components x 576 colour-spin terms a site
            for op in range(2):
                assert _close(lat.delta_2pt(p1, p2, op, Q, xs), oracle.delta_2pt(L, p1, p2, op, Q, xs)), (L, op)
            assert _close(lat.nucleon_2pt(p1, p2, Q, xs), oracle.nucleon_2pt(L, p1, p2, Q, xs)), L


def test_propagator_to_correlators_on_device(qkx, oracle):
    """qkx_propagator_dev -> contractions from device memory, against the host route."""
    L = (4, 4, 4, 8)
    U = oracle.gauge_random(L, 0.3, 9)
    src = (1, 2, 3, 4)
    with qkx.Lattice(qkx.LatticeInfo(L=L, kappa=0.16, mu=0.01)) as lat:
        lat.load_gauge(U, qkx.LINKS_APPLY_BC)
        lat.APE_smearing(U, 5, 0.5)
        nbytes = lat.V * 2304
        d = qkx.lib().qkx_device_alloc(lat.ctx, nbytes)
        assert d
        try:
            lat.propagator_dev(d, src, 4, 4.0, tol=1e-12)
            lat.sync()
            prop = np.empty((lat.V, 4, 4, 3, 3, 2))
            qkx.check(qkx.lib().qkx_memcpy_d2h(lat.ctx, prop.ctypes.data, C.c_void_p(d), nbytes))
            dev = lat.meson_2pt(d, range(10), 1, src, device=True)
            host = lat.meson_2pt(prop, range(10), 1, src)
            assert np.array_equal(dev, host)
            nd = lat.baryon_2pt(d, d, 0, 1, src, device=True)
            assert _close(nd, oracle.baryon_2pt(L, prop, prop, 0, 1, src))
        finally:
            qkx.lib().qkx_device_free(lat.ctx, C.c_void_p(d))


def test_argument_checks(qkx):
    with qkx.Lattice(qkx.LatticeInfo(L=(4, 4, 4, 4))) as lat:
        p = np.zeros((lat.V, 4, 4, 3, 3, 2))
        with pytest.raises(qkx.QkxError):
            lat.meson_2pt(p, [10])
        with pytest.raises(qkx.QkxError):
            lat.baryon_2pt(p, p, 4)
        with pytest.raises(qkx.QkxError):
            lat.delta_2pt(p, p, 2)
        with pytest.raises(qkx.QkxError):
            lat.meson_2pt(p, [0], Q_sq=-1)
