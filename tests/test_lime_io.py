"""LIME / SciDAC / ILDG I/O (cvc_b200.lime over lime_io.cpp).

The reference's readers and writers need c-lime, which is not here, so the
files are checked against an independent Python reading of the published
formats (LIME record headers, big-endian numbers, the site and direction
orders of io.c:282-322 and propagator_io.c:363-366, CVC order for
contractions), and the SciDAC checksum is pinned against the reference's own
dml.c / DML_crc32.c (compiled into oracle/_ref)."""
import ctypes
import os
import struct
import zlib

import numpy as np
import pytest

from conftest import seeded

DIMS = (4, 2, 4, 6)  # T, LX, LY, LZ: all distinct orders show up
T, LX, LY, LZ = DIMS
V = T * LX * LY * LZ


def parse(path):
    """[(type, mb, me, data)] of a LIME file."""
    out = []
    with open(path, "rb") as f:
        while True:
            h = f.read(144)
            if not h:
                return out
            magic, version, flags, n = struct.unpack(">IHHQ", h[:16])
            assert magic == 0x456789AB and version == 1
            typ = h[16:144].split(b"\0")[0].decode()
            data = f.read(n)
            pad = f.read((8 - n % 8) % 8)
            assert pad == b"\0" * len(pad)
            out.append((typ, bool(flags & 0x8000), bool(flags & 0x4000), data))


def record(typ, data, mb=False, me=False):
    h = struct.pack(">IHHQ", 0x456789AB, 1, (0x8000 if mb else 0) | (0x4000 if me else 0),
                    len(data)) + typ.encode().ljust(128, b"\0")
    return h + data + b"\0" * ((8 - len(data) % 8) % 8)


def rotl(w, r):
    return ((w << r) | (w >> (32 - r))) & 0xFFFFFFFF if r else w


def scidac_sums(site_bytes_by_rank):
    a = b = 0
    for rank, buf in site_bytes_by_rank:
        w = zlib.crc32(buf)
        a ^= rotl(w, rank % 29)
        b ^= rotl(w, rank % 31)
    return a, b


def ildg_order(gauge, dtype):
    """CVC gauge (72 V) -> per file site (t, z, y, x) the 72 reals with the
    directions in the order x, y, z, t."""
    g = gauge.reshape(T, LX, LY, LZ, 4, 18)[..., [1, 2, 3, 0], :]
    return np.ascontiguousarray(g.transpose(0, 3, 2, 1, 4, 5)).astype(dtype)


def test_crc32_matches_zlib_and_reference(cb):
    from cvc_b200 import lime
    import oracle_bind
    for n in (0, 1, 7, 64, 1000):
        data = bytes((np.arange(n) * 37 % 251).astype(np.uint8))
        assert lime.crc32(data) == zlib.crc32(data)
        assert lime.crc32(data[n // 2:], lime.crc32(data[:n // 2])) == zlib.crc32(data)
    if oracle_bind.reference_available():
        ref = ctypes.CDLL(oracle_bind.REF_LIB)
        ref.ref_dml_crc32.restype = ctypes.c_uint
        ref.ref_dml_crc32.argtypes = [ctypes.c_uint, ctypes.c_void_p, ctypes.c_size_t]
        data = bytes(range(256)) * 3
        assert lime.crc32(data) == ref.ref_dml_crc32(0, data, len(data))


def test_dml_checksum_matches_reference(cb):
    from cvc_b200 import lime
    import oracle_bind
    if not oracle_bind.reference_available():
        pytest.skip("reference library not built")
    ref = ctypes.CDLL(oracle_bind.REF_LIB)
    ref.ref_dml_checksum_accum.restype = None
    ref.ref_dml_checksum_accum.argtypes = [ctypes.POINTER(ctypes.c_uint), ctypes.c_uint,
                                           ctypes.c_void_p, ctypes.c_size_t]
    ours = (0, 0)
    theirs = (ctypes.c_uint * 2)(0, 0)
    for rank in list(range(70)) + [29 * 31, 29 * 31 * 7 + 3, 2 ** 32 - 1]:
        buf = np.float64(seeded(rank + 1, 9)).astype(">f8").tobytes()
        ours = lime.dml_checksum_accum(ours, rank, buf)
        ref.ref_dml_checksum_accum(theirs, rank, buf, len(buf))
        assert ours == (theirs[0], theirs[1]), rank


@pytest.mark.parametrize("prec", [64, 32])
def test_gauge_read_of_independent_ildg_file(cb, tmp_path, prec):
    from cvc_b200 import lime
    gauge = seeded(5, 72 * V)
    dt = ">f8" if prec == 64 else ">f4"
    sites = ildg_order(gauge, dt).reshape(V, 72)
    fn = tmp_path / "conf.0000"
    fn.write_bytes(record("ildg-format", b"<ildgFormat/>", mb=True) +
                   record("ildg-binary-data", sites.tobytes()) +
                   record("scidac-checksum", b"x", me=True))
    g, sums = lime.read_lime_gauge_field(fn, DIMS)
    want = gauge if prec == 64 else gauge.astype(np.float32).astype(np.float64)
    assert np.array_equal(g, want)
    # rank of file site (t, z, y, x) is its position in the file
    assert sums == scidac_sums((r, sites[r].tobytes()) for r in range(V))


@pytest.mark.parametrize("prec", [64, 32])
def test_gauge_write_format_and_round_trip(cb, tmp_path, prec):
    from cvc_b200 import lime
    gauge = seeded(6, 72 * V)
    fn = tmp_path / "g.lime"
    sums = lime.write_lime_gauge_field(fn, gauge, DIMS, prec)
    recs = parse(fn)
    assert [r[0] for r in recs] == ["ildg-format", "ildg-binary-data", "scidac-checksum"]
    assert recs[0][1] and recs[-1][2]
    assert b"<precision> %d </precision>" % prec in recs[0][3]
    assert b"<lt> %d </lt>" % T in recs[0][3] and b"<lz> %d </lz>" % LZ in recs[0][3]
    dt = ">f8" if prec == 64 else ">f4"
    assert recs[1][3] == ildg_order(gauge, dt).tobytes()
    assert (b"<suma>%#010x</suma>" % sums[0]) in recs[2][3]
    g, sums2 = lime.read_lime_gauge_field(fn, DIMS)
    assert sums2 == sums
    want = gauge if prec == 64 else gauge.astype(np.float32).astype(np.float64)
    assert np.array_equal(g, want)


def test_spinor_files(cb, tmp_path):
    from cvc_b200 import lime
    a, b = seeded(7, 24 * V), seeded(8, 24 * V)
    fn = tmp_path / "source.0000.00.inverted"
    s_a = lime.write_propagator(fn, a, DIMS, 64)
    s_b = lime.write_lime_spinor(fn, b, DIMS, append=True, prec=32)
    recs = parse(fn)
    assert [r[0] for r in recs] == ["etmc-propagator-format", "scidac-binary-data",
                                    "scidac-checksum", "scidac-binary-data", "scidac-checksum"]
    assert b"<field>diracFermion</field>" in recs[0][3]
    # file order t, z, y, x with 24 reals per site in CVC's within-site order
    order = a.reshape(T, LX, LY, LZ, 24).transpose(0, 3, 2, 1, 4)
    assert recs[1][3] == np.ascontiguousarray(order).astype(">f8").tobytes()
    ra, sa = lime.read_lime_spinor(fn, DIMS, 0)
    rb, sb = lime.read_lime_spinor(fn, DIMS, 1)
    assert np.array_equal(ra, a) and sa == s_a
    assert np.array_equal(rb, b.astype(np.float32).astype(np.float64)) and sb == s_b
    with pytest.raises(cb.CvcbError):
        lime.read_lime_spinor(fn, DIMS, 2)
    with pytest.raises(cb.CvcbError):
        lime.read_lime_spinor(fn, (T, LX, LY, LZ + 2), 0)
    with pytest.raises(cb.CvcbError):
        lime.read_lime_spinor(tmp_path / "missing", DIMS, 0)


def test_contraction_files(cb, tmp_path):
    from cvc_b200 import lime
    conn = seeded(9, 32 * V)
    fn = tmp_path / "cvc_v_x.0000"
    sums = lime.write_lime_contraction(fn, conn, DIMS, 64, 16, "cvc", 4, 7)
    recs = parse(fn)
    assert [r[0] for r in recs] == ["cvc_contraction-format", "scidac-binary-data",
                                    "scidac-checksum"]
    fmt = recs[0][3]
    for tag in (b"<type>cvc</type>", b"<components>16</components>", b"<nconf>4</nconf>",
                b"<source>7</source>", b"<lt>%d</lt>" % T, b"<lx>%d</lx>" % LX):
        assert tag in fmt
    # CVC site order and layout: the record is conn itself, big-endian
    assert recs[1][3] == conn.astype(">f8").tobytes()
    site = 32 * 8
    assert sums == scidac_sums((r, recs[1][3][r * site:(r + 1) * site]) for r in range(V))
    assert (b"<suma>%08x</suma>" % sums[0]) in recs[2][3]
    c, s2 = lime.read_lime_contraction(fn, DIMS, 16, 0)
    assert np.array_equal(c, conn) and s2 == sums
    lime.write_lime_contraction(fn, conn, DIMS, 32)
    c32, _ = lime.read_lime_contraction(fn, DIMS, 16, 0)
    assert np.array_equal(c32, conn.astype(np.float32).astype(np.float64))


def test_gauge_read_errors(cb, tmp_path):
    """Wrong lattice, a truncated record and a file that is not LIME are
    errors with a message, never a partial field."""
    from cvc_b200 import lime
    g = cb.gauge_random(*DIMS, 0.3, 5)
    fn = tmp_path / "conf.0001"
    lime.write_lime_gauge_field(fn, g, DIMS)
    with pytest.raises(cb.CvcbError):
        lime.read_lime_gauge_field(fn, (T, LX, LY, LZ + 2))
    data = fn.read_bytes()
    cut = tmp_path / "conf.cut"
    cut.write_bytes(data[:len(data) // 2])
    with pytest.raises(cb.CvcbError):
        lime.read_lime_gauge_field(cut, DIMS)
    junk = tmp_path / "conf.txt"
    junk.write_bytes(b"plain text, not a LIME file\n" * 8)
    with pytest.raises(cb.CvcbError, match="not a LIME file"):
        lime.read_lime_gauge_field(junk, DIMS)
    with pytest.raises(cb.CvcbError, match="cannot open"):
        lime.read_lime_gauge_field(tmp_path / "missing", DIMS)
