"""LIME / SciDAC / ILDG files for gauge fields, propagators and contractions
(the reference's io.c, gauge_io.c, propagator_io.c, contractions_io.c), over
the host-side functions of libcvcb200.so.  Arrays are float64 numpy arrays in
CVC's layouts; every function also returns the SciDAC checksum (suma, sumb)
of the binary record."""
import ctypes

import numpy as np

from . import _lib
from .lattice import _check


def _sums():
    return (ctypes.c_uint32 * 2)()


def _dims(dims):
    T, LX, LY, LZ = (int(d) for d in dims)
    return T, LX, LY, LZ, T * LX * LY * LZ


def crc32(data, crc=0):
    """CRC-32 of `data` (bytes) continuing from `crc`, as DML_crc32."""
    out = ctypes.c_uint32()
    buf = bytes(data)
    _check("cvcb_crc32", _lib.load().cvcb_crc32(crc, buf, len(buf), ctypes.byref(out)))
    return out.value


def dml_checksum_accum(sums, rank, data):
    """One DML_checksum_accum step: returns the new (suma, sumb)."""
    s = (ctypes.c_uint32 * 2)(*sums)
    buf = bytes(data)
    _check("cvcb_dml_checksum_accum",
           _lib.load().cvcb_dml_checksum_accum(s, rank, buf, len(buf)))
    return s[0], s[1]


def read_lime_gauge_field(filename, dims):
    """Gauge field (72*V) from an ILDG file, 64- or 32-bit."""
    T, LX, LY, LZ, V = _dims(dims)
    g = np.zeros(72 * V)
    s = _sums()
    _check("read_lime_gauge_field", _lib.load().cvcb_read_lime_gauge_field_doubleprec(
        str(filename).encode(), g.ctypes.data, T, LX, LY, LZ, s))
    return g, (s[0], s[1])


def write_lime_gauge_field(filename, gauge, dims, prec=64):
    T, LX, LY, LZ, _ = _dims(dims)
    g = np.ascontiguousarray(gauge, np.float64)
    s = _sums()
    _check("write_lime_gauge_field", _lib.load().cvcb_write_lime_gauge_field(
        str(filename).encode(), g.ctypes.data, T, LX, LY, LZ, int(prec), s))
    return s[0], s[1]


def read_lime_spinor(filename, dims, position=0):
    """Dirac field (24*V) from the position-th scidac-binary-data record."""
    T, LX, LY, LZ, V = _dims(dims)
    f = np.zeros(24 * V)
    s = _sums()
    _check("read_lime_spinor", _lib.load().cvcb_read_lime_spinor(
        f.ctypes.data, str(filename).encode(), int(position), T, LX, LY, LZ, s))
    return f, (s[0], s[1])


def write_lime_spinor(filename, field, dims, append=False, prec=64):
    T, LX, LY, LZ, _ = _dims(dims)
    f = np.ascontiguousarray(field, np.float64)
    s = _sums()
    _check("write_lime_spinor", _lib.load().cvcb_write_lime_spinor(
        f.ctypes.data, str(filename).encode(), int(bool(append)), int(prec), T, LX, LY, LZ, s))
    return s[0], s[1]


def write_propagator(filename, field, dims, prec=64):
    T, LX, LY, LZ, _ = _dims(dims)
    f = np.ascontiguousarray(field, np.float64)
    s = _sums()
    _check("write_propagator", _lib.load().cvcb_write_propagator(
        f.ctypes.data, str(filename).encode(), int(prec), T, LX, LY, LZ, s))
    return s[0], s[1]


def write_lime_contraction(filename, conn, dims, prec=64, N=16, ctype="cvc", gid=0, sid=0):
    T, LX, LY, LZ, _ = _dims(dims)
    c = np.ascontiguousarray(conn, np.float64)
    s = _sums()
    _check("write_lime_contraction", _lib.load().cvcb_write_lime_contraction(
        c.ctypes.data, str(filename).encode(), int(prec), int(N), ctype.encode(), int(gid),
        int(sid), T, LX, LY, LZ, s))
    return s[0], s[1]


def read_lime_contraction(filename, dims, N=16, position=0):
    T, LX, LY, LZ, V = _dims(dims)
    c = np.zeros(2 * N * V)
    s = _sums()
    _check("read_lime_contraction", _lib.load().cvcb_read_lime_contraction(
        c.ctypes.data, str(filename).encode(), int(N), int(position), T, LX, LY, LZ, s))
    return c, (s[0], s[1])
