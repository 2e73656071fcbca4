"""CPU tests of the contraction oracle (oracle/qkx_oracle_contract.c) against the
reference's Meson/Baryon/Baryon_Dec contractions and Fourier transforms and its
contractNucleon: golden vectors
made from the compiled reference (tests/golden/ref_contract.npz) and the live
build.  The restatement keeps the reference's term order and arithmetic, so
agreement is to the last bit on the golden lattice."""
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))


def _g():
    return np.load(os.path.join(GOLDEN, "ref_contract.npz"))


def _props(O, g):
    from make_golden import seeded_propagator
    L = tuple(int(v) for v in g["L"])
    return L, seeded_propagator(L, int(g["seed1"])), seeded_propagator(L, int(g["seed2"]))


def test_momenta(oracle):
    m = oracle.momenta(1)
    assert m.tolist() == [[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [0, 0, -1], [0, -1, 0], [-1, 0, 0]]
    assert len(oracle.momenta(2)) == 19 and len(oracle.momenta(4)) == 33
    assert np.array_equal(oracle.momenta(int(_g()["Q_sq"])), _g()["momenta"])


def test_contractions_golden(oracle):
    g = _g()
    L, p1, p2 = _props(oracle, g)
    Q, xs = int(g["Q_sq"]), tuple(int(v) for v in g["x_src"])
    for op, name in enumerate(oracle.MESONS):
        a = oracle.meson_2pt(L, p1, op, Q, xs)
        assert np.abs(a - g[f"meson:{name}"]).max() <= 1e-14 * np.abs(a).max(), name
    for op, name in enumerate(oracle.BARYONS):
        a = oracle.baryon_2pt(L, p1, p2, op, Q, xs)
        assert np.abs(a - g[f"baryon:{name}"]).max() <= 1e-14 * np.abs(a).max(), name


def test_decuplet_and_contract_nucleon_golden(oracle):
    """Baryon_Dec (both isospin operators) to the last bit; contractNucleon against the
    numbers the reference printed (7 digits) and, to rounding, against Baryon NTN."""
    g = _g()
    L, p1, p2 = _props(oracle, g)
    Q, xs = int(g["Q_sq"]), tuple(int(v) for v in g["x_src"])
    for op, name in enumerate(oracle.DELTAS):
        assert np.array_equal(oracle.delta_2pt(L, p1, p2, op, Q, xs), g[f"delta:{name}"]), name
    n = oracle.nucleon_2pt(L, p1, p2, Q, xs)
    scale = np.abs(n).max()
    assert np.abs(n - g["nucleon_text"]).max() <= 1e-6 * scale
    assert np.abs(n - g["baryon:NTN"]).max() <= 1e-14 * scale


def test_contractions_vs_live_reference(oracle):
    if not oracle.ref_available():
        pytest.skip("reference build not present")
    from make_golden import seeded_propagator
    for L, xs, Q in (((2, 2, 2, 4), (0, 0, 0, 0), 0), ((4, 4, 2, 2), (3, 1, 1, 1), 1)):
        p1, p2 = seeded_propagator(L, 5), seeded_propagator(L, 6)
        for op in range(10):
            assert np.array_equal(oracle.meson_2pt(L, p1, op, Q, xs), oracle.ref_meson_2pt(L, p1, op, Q, xs))
        for op in range(4):
            assert np.array_equal(oracle.baryon_2pt(L, p1, p2, op, Q, xs),
                                  oracle.ref_baryon_2pt(L, p1, p2, op, Q, xs))
        for op in range(2):
            assert np.array_equal(oracle.delta_2pt(L, p1, p2, op, Q, xs), oracle.ref_delta_2pt(L, p1, p2, op, Q, xs))
