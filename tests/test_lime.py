"""CPU tests of the LIME/ILDG restatement used as the checker for the library's
reader and writer (oracle/lime.py): record framing, padding, the Gauge::M order
of the binary record, and its pin to the reference's own reader and writer
(compiled with project-written LIME and MPI-IO stand-ins) and to a file that
the reference wrote."""
import struct

import numpy as np

from oracle import lime


def test_record_framing_and_padding(tmp_path):
    p = tmp_path / "r.lime"
    with open(p, "wb") as f:
        lime.write_record(f, "a-type", b"12345", mb=True)
        lime.write_record(f, "b-type", b"", me=True)
    raw = p.read_bytes()
    assert len(raw) == 144 + 8 + 144
    magic, ver, flags, n = struct.unpack(">IHHQ", raw[:16])
    assert (magic, ver, flags, n) == (0x456789AB, 1, 0x8000, 5)
    assert raw[16:22] == b"a-type" and raw[144 + 5:152] == b"\0\0\0"
    assert lime.read_records(p) == [("a-type", b"12345"), ("b-type", b"")]


def test_gauge_round_trip_and_order(tmp_path, oracle):
    L = (4, 2, 2, 4)
    U = oracle.gauge_random(L, 0.3, 3)
    p = tmp_path / "g.lime"
    lime.write_gauge(p, U, L, extra=[("xlf-info", b"odd length!")])
    assert np.array_equal(lime.read_gauge(p, L), U)
    # the binary record is big-endian in Gauge::M order: site (x fastest), mu, c1, c2, re/im
    rec = dict(lime.read_records(p))["ildg-binary-data"]
    first = struct.unpack(">d", rec[:8])[0]
    mu1 = struct.unpack(">d", rec[18 * 8:19 * 8])[0]
    assert first == U[0, 0, 0, 0, 0] and mu1 == U[0, 1, 0, 0, 0]
    p32 = tmp_path / "g32.lime"
    lime.write_gauge(p32, U, L, precision=32)
    assert np.array_equal(lime.read_gauge(p32, L), U.astype(np.float32).astype(np.float64))


GOLDEN_L = (4, 2, 2, 4)
GOLDEN_MESSAGE = b"written by the reference's qkxTM_writeGaugeLime"


def golden_path():
    import os
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_conf_4x2x2x4.lime")


def golden_links(oracle):
    return oracle.apply_bc(GOLDEN_L, oracle.gauge_random(GOLDEN_L, 0.3, 77), -1)


def test_restatement_pinned_to_reference_written_file(tmp_path, oracle):
    """tests/golden/ref_conf_4x2x2x4.lime was written by the reference's own writer
    (tests/golden/make_golden.py): the restatement reads its links exactly and writes the
    same bytes from the same links and message."""
    U = golden_links(oracle)
    assert np.array_equal(lime.read_gauge(golden_path(), GOLDEN_L), U)
    p = tmp_path / "ours.lime"
    lime.write_gauge(p, U, GOLDEN_L, message=GOLDEN_MESSAGE)
    assert p.read_bytes() == open(golden_path(), "rb").read()


def test_restatement_against_live_reference(tmp_path, oracle):
    """The reference's reader and writer (read_conf_lime.cpp, write_conf_lime.cpp compiled
    unmodified) against the restatement in both directions, with records the reader must
    skip and a message whose length needs padding."""
    import pytest
    if not oracle.ref_available():
        pytest.skip("reference build absent")
    for L, seed in (((4, 2, 2, 4), 5), ((2, 4, 6, 2), 6)):
        U = oracle.apply_bc(L, oracle.gauge_random(L, 0.3, seed), -1)
        ours = tmp_path / f"ours{seed}.lime"
        lime.write_gauge(ours, U, L, message=b"odd-length message", extra=[("ildg-data-lfn", b"lfn://abc")])
        assert np.array_equal(oracle.ref_read_gauge_lime(ours, L), U)
        theirs = tmp_path / f"ref{seed}.lime"
        oracle.ref_write_gauge_lime(theirs, L, U, b"odd-length message")
        assert np.array_equal(lime.read_gauge(theirs, L), U)
        plain = tmp_path / f"plain{seed}.lime"
        lime.write_gauge(plain, U, L, message=b"odd-length message")
        assert plain.read_bytes() == theirs.read_bytes()
