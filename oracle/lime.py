"""LIME / ILDG files for the tests -- TEST INFRASTRUCTURE ONLY.

A restatement, in numpy, of the reference's gauge reader and writer
(lib/read_conf_lime.cpp:111-245, lib/write_conf_lime.cpp:49-199) over the
published LIME record format (the c-lime library is not part of the reference
tree).  Each record: a 144-byte big-endian header -- magic 0x456789ab (4
bytes), version (2), flags (2: bit 15 message begin, bit 14 message end),
data length (8), type (128, NUL-padded) -- then the data padded to 8 bytes.
An ILDG configuration: "ildg-format" XML with <precision>, <lx>..<lt>, and
"ildg-binary-data" holding the links big-endian in the Gauge::M order (sites
x fastest, t slowest; directions x y z t; 3x3 row-major complex).
"""
from __future__ import annotations

import re
import struct

import numpy as np

MAGIC = 0x456789AB


def write_record(f, rtype: str, data: bytes, mb: bool = False, me: bool = False) -> None:
    flags = (0x8000 if mb else 0) | (0x4000 if me else 0)
    hdr = struct.pack(">IHHQ", MAGIC, 1, flags, len(data)) + rtype.encode().ljust(128, b"\0")
    f.write(hdr)
    f.write(data)
    f.write(b"\0" * ((8 - len(data) % 8) % 8))


def ildg_xml(L, precision=64) -> bytes:
    """The ildg-format text of lib/write_conf_lime.cpp:84, character for character (a
    writer that is to produce the reference's bytes has to write this exact text)."""
    return ("<?xml version=\"1.0\" encoding=\"UTF-8\"?>\n<ildgFormat xmlns=\"http://www.lqkxTM.org/ildg\"\n"
            "            xmlns:xsi=\"http://www.w3.org/2001/XMLSchema-instance\"\n"
            "            xsi:schemaLocation=\"http://www.lqkxTM.org/ildg filefmt.xsd\">\n"
            f"  <version> 1.0 </version>\n  <field> su3gauge </field>\n  <precision> {precision} </precision>\n"
            f"  <lx> {L[0]} </lx>\n  <ly> {L[1]} </ly>\n  <lz> {L[2]} </lz>\n  <lt> {L[3]} </lt>\n</ildgFormat>"
            ).encode()


def write_gauge(path, U: np.ndarray, L, precision=64, message=b"test configuration", extra=()) -> None:
    """Records as lib/write_conf_lime.cpp writes them (ildg-format, xlf-info, ildg-binary-data);
    `extra` (type, bytes) records are written first."""
    dt = ">f8" if precision == 64 else ">f4"
    with open(path, "wb") as f:
        for t, d in extra:
            write_record(f, t, d)
        write_record(f, "ildg-format", ildg_xml(L, precision), mb=True)
        write_record(f, "xlf-info", message)
        write_record(f, "ildg-binary-data", np.ascontiguousarray(U, dtype=np.float64).astype(dt).tobytes(), me=True)


def read_records(path):
    out = []
    with open(path, "rb") as f:
        data = f.read()
    pos = 0
    while pos + 144 <= len(data):
        magic, ver, flags, n = struct.unpack(">IHHQ", data[pos:pos + 16])
        if magic != MAGIC:
            raise ValueError("bad LIME magic number")
        rtype = data[pos + 16:pos + 144].split(b"\0")[0].decode()
        out.append((rtype, data[pos + 144:pos + 144 + n]))
        pos += 144 + n + (8 - n % 8) % 8
    return out


def read_gauge(path, L) -> np.ndarray:
    """The links of the first ildg-binary-data record as Gauge::M [V, 4, 3, 3, 2]."""
    prec = 64
    for rtype, d in read_records(path):
        if rtype == "ildg-format":
            m = re.search(rb"<precision>\s*(\d+)", d)
            prec = int(m.group(1)) if m else 64
        if rtype == "ildg-binary-data":
            a = np.frombuffer(d, dtype=">f8" if prec == 64 else ">f4").astype(np.float64)
            return a.reshape(int(np.prod(L)), 4, 3, 3, 2)
    raise ValueError("no ildg-binary-data record")
