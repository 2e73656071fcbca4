"""GPU tests of the ILDG/LIME reader and writer (qkxTM_MPI_getGaugeLime,
lib/read_conf_lime.cpp:111-245; qkxTM_writeGaugeLime, lib/write_conf_lime.cpp)
against the LIME restatement in oracle/lime.py and the operator oracle.
Byte-exact: the reader returns and loads the file's links unchanged."""
import numpy as np
import pytest

from conftest import rel
from oracle import lime

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("L", [(4, 4, 4, 8), (6, 4, 2, 10)])
def test_read_matches_file(qkx, oracle, tmp_path, L):
    U = oracle.apply_bc(L, oracle.gauge_random(L, 0.3, 40 + L[3]), -1)
    p = tmp_path / "conf.lime"
    lime.write_gauge(p, U, L, extra=[("ildg-data-lfn", b"lfn://x"), ("xlf-info", b"odd")])
    psi = oracle.spinor_gaussian(L, 1)
    with qkx.Lattice(qkx.LatticeInfo(L=L, kappa=0.16, mu=0.01)) as lat:
        Uh, info = lat.read_gauge_lime(str(p), qkx.LINKS_AS_GIVEN)
        assert np.array_equal(Uh, U)
        assert info["precision"] == 64 and info["L"] == L and info["records"] == 5
        assert info["data_bytes"] == U.size * 8
        # the loaded operator links are the file's
        assert rel(lat.tm(psi), oracle.apply("tm", L, U, psi, 0.16, 0.01)) < 1e-13
        assert np.array_equal(lat.download_gauge(), U)


def test_read_applies_boundary_condition(qkx, oracle, tmp_path):
    L = (4, 4, 4, 8)
    U = oracle.gauge_random(L, 0.3, 5)
    p = tmp_path / "raw.lime"
    lime.write_gauge(p, U, L)
    with qkx.Lattice(qkx.LatticeInfo(L=L)) as lat:
        Uh, _ = lat.read_gauge_lime(str(p), qkx.LINKS_APPLY_BC)
        assert np.array_equal(Uh, U)  # the returned array is the file's
        assert np.array_equal(lat.download_gauge(), oracle.apply_bc(L, U, -1))
        assert lat.compressible()


def test_read_32_bit_file(qkx, oracle, tmp_path):
    L = (4, 4, 4, 8)
    U = oracle.gauge_random(L, 0.3, 6)
    p = tmp_path / "single.lime"
    lime.write_gauge(p, U, L, precision=32)
    with qkx.Lattice(qkx.LatticeInfo(L=L)) as lat:
        Uh, info = lat.read_gauge_lime(str(p))
        assert info["precision"] == 32
        assert np.array_equal(Uh, U.astype(np.float32).astype(np.float64))


def test_write_then_read(qkx, oracle, tmp_path):
    L = (4, 4, 4, 8)
    U = oracle.apply_bc(L, oracle.gauge_random(L, 0.3, 7), -1)
    with qkx.Lattice(qkx.LatticeInfo(L=L)) as lat:
        p1 = tmp_path / "host.lime"
        lat.write_gauge_lime(str(p1), U, "written from host links")
        assert np.array_equal(lime.read_gauge(p1, L), U)
        recs = dict(lime.read_records(p1))
        assert b"<precision> 64 </precision>" in recs["ildg-format"] and recs["xlf-info"] == b"written from host links"
        lat.load_gauge(U, qkx.LINKS_AS_GIVEN)
        p2 = tmp_path / "ctx.lime"
        lat.write_gauge_lime(str(p2))
        assert np.array_equal(lime.read_gauge(p2, L), U)
        Uh, _ = lat.read_gauge_lime(str(p2))
        assert np.array_equal(Uh, U)


def test_reader_errors(qkx, oracle, tmp_path):
    L = (4, 4, 4, 8)
    U = oracle.gauge_random(L, 0.3, 8)
    with qkx.Lattice(qkx.LatticeInfo(L=L)) as lat:
        with pytest.raises(qkx.QkxError) as e:
            lat.read_gauge_lime(str(tmp_path / "missing.lime"))
        assert e.value.code == qkx.ERR_INVALID
        wrong = tmp_path / "wrong.lime"
        lime.write_gauge(wrong, oracle.gauge_random((4, 4, 4, 4), 0.3, 1), (4, 4, 4, 4))
        with pytest.raises(qkx.QkxError):
            lat.read_gauge_lime(str(wrong))
        nobin = tmp_path / "nobin.lime"
        with open(nobin, "wb") as f:
            lime.write_record(f, "ildg-format", lime.ildg_xml(L))
        with pytest.raises(qkx.QkxError) as e:
            lat.read_gauge_lime(str(nobin))
        assert "ildg-binary-data" in str(e.value)
        good = tmp_path / "good.lime"
        lime.write_gauge(good, U, L)
        raw = good.read_bytes()
        trunc = tmp_path / "trunc.lime"
        trunc.write_bytes(raw[:-1000])
        with pytest.raises(qkx.QkxError):
            lat.read_gauge_lime(str(trunc))
        badmagic = tmp_path / "badmagic.lime"
        badmagic.write_bytes(b"\0\0\0\0" + raw[4:])
        with pytest.raises(qkx.QkxError):
            lat.read_gauge_lime(str(badmagic))
        # a failed read leaves no gauge field behind
        with pytest.raises(qkx.QkxError):
            lat.tm(oracle.spinor_gaussian(L, 1))


def test_reader_and_writer_pinned_to_reference_written_file(qkx, oracle, tmp_path):
    """tests/golden/ref_conf_4x2x2x4.lime was written by the reference's qkxTM_writeGaugeLime:
    the library reads exactly its links (as the reference's reader does) and writes the same
    bytes from them, from host links and from the links a context holds."""
    import os
    L = (4, 2, 2, 4)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_conf_4x2x2x4.lime")
    U = oracle.apply_bc(L, oracle.gauge_random(L, 0.3, 77), -1)
    golden = open(path, "rb").read()
    msg = "written by the reference's qkxTM_writeGaugeLime"
    with qkx.Lattice(qkx.LatticeInfo(L=L)) as lat:
        Uh, info = lat.read_gauge_lime(path, qkx.LINKS_AS_GIVEN)
        assert np.array_equal(Uh, U) and np.array_equal(lat.download_gauge(), U)
        if oracle.ref_available():
            assert np.array_equal(Uh, oracle.ref_read_gauge_lime(path, L))
        p1 = tmp_path / "host.lime"
        lat.write_gauge_lime(str(p1), U, msg)
        assert p1.read_bytes() == golden
        p2 = tmp_path / "ctx.lime"
        lat.write_gauge_lime(str(p2), None, msg)
        assert p2.read_bytes() == golden
