"""CPU tests of the LIME/ILDG restatement used as the checker for the library's
reader and writer (oracle/lime.py): record framing, padding, and the Gauge::M
order of the binary record."""
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
