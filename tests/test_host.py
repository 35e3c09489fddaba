"""Host-side parts of the product that need no GPU: geometry tables, gamma
tables, boundary phases, RANLUX, the gauge generator, propagator file
names, and the C ABI's symbol table."""
import ctypes
import os
import re

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
FIX = np.load(os.path.join(HERE, "golden", "reference_fixtures.npz"))


@pytest.mark.parametrize("dims", [(8, 4, 4, 4), (6, 4, 2, 4)])
def test_geometry_bit_exact(cb, dims):
    t = cb.geometry_tables(*dims)
    tag = "x".join(map(str, dims))
    for k, v in t.items():
        assert np.array_equal(v, FIX[f"geom_{tag}_{k}"]), k


def test_geometry_properties(cb):
    T, LX, LY, LZ = 6, 4, 8, 2
    t = cb.geometry_tables(T, LX, LY, LZ)
    V = T * LX * LY * LZ
    iup, idn = t["g_iup"].reshape(V, 4), t["g_idn"].reshape(V, 4)
    for mu in range(4):
        assert np.array_equal(idn[iup[:, mu], mu], np.arange(V))
    assert sorted(t["g_eo2lexic"]) == list(range(V))
    assert np.array_equal(t["g_lexic2eo"][t["g_eo2lexic"]], np.arange(V))


def test_gamma_tables(cb):
    perm, sign = cb.gamma_tables()
    assert np.array_equal(perm, FIX["gamma_perm"])
    assert np.array_equal(sign, FIX["gamma_sign"])


@pytest.mark.parametrize("bc", [(1.0, 0.0, 0.0, 0.0), (1.0, 0.5, 0.0, 0.25)])
def test_phases(cb, bc):
    ph = cb.boundary_phases(8, 6, 4, 2, bc)
    ref = FIX["phase_8x6x4x2_" + "_".join(str(b) for b in bc)]
    assert np.array_equal(np.stack([ph.real, ph.imag], 1).ravel(), ref)


@pytest.mark.parametrize("seed,level", [(1234, 1), (7, 2), (11, 1), (3, 1), (21, 1), (1, 1)])
def test_ranlxd_bit_exact(cb, seed, level):
    ref = FIX[f"ranlxd_{seed}_{level}"]
    assert np.array_equal(cb.ranlxd(ref.size, seed, level), ref)


def test_gauge_generator(cb):
    g = cb.gauge_random(4, 2, 2, 4, 0.3, 1234)
    u = (g[0::2] + 1j * g[1::2]).reshape(-1, 3, 3)
    eye = np.eye(3)
    assert np.max(np.abs(u @ np.conj(np.transpose(u, (0, 2, 1))) - eye)) < 1e-14
    assert np.max(np.abs(np.linalg.det(u) - 1)) < 1e-14
    assert np.array_equal(g, cb.gauge_random(4, 2, 2, 4, 0.3, 1234))
    assert not np.array_equal(g, cb.gauge_random(4, 2, 2, 4, 0.3, 1235))
    # small eps: close to the identity, with the first links drawn from
    # ranlxd seed 1234 through Box-Muller (H traceless hermitian)
    s = cb.gauge_random(2, 2, 2, 2, 1e-6, 1234)
    us = (s[0::2] + 1j * s[1::2]).reshape(-1, 3, 3)
    H = (us - eye) / 1e-6 / 1j
    assert np.max(np.abs(H - np.conj(np.transpose(H, (0, 2, 1))))) < 1e-5
    assert np.max(np.abs(np.trace(H, axis1=1, axis2=2))) < 1e-5
    r = cb.ranlxd(8, 1234)
    w0 = np.sqrt(-2 * np.log(r[0])) * np.cos(2 * np.pi * r[1])  # lambda_1 weight
    assert abs(H[0, 0, 1].real - w0 / 2) < 1e-5


def test_get_filename(cb):
    from cvc_b200.files import get_filename
    cases = [(0, 4, 7, 1), (0, 2, 11, -1), (0, 1, 0, 0), (2, 3, 5, 1), (3, 0, 9, -1), (4, 4, 2, 1)]
    for (fmt, nu, sc, sign), want in zip(cases, FIX["filenames"]):
        got = get_filename(nu, sc, sign, filename_prefix="source", filename_prefix2="dnprop",
                           Nconf=17, format=fmt, source_location=37, T_global=8, LX_global=4,
                           LY_global=4, LZ_global=4)
        assert got == str(want)


def _declared_symbols():
    text = open(os.path.join(ROOT, "include", "cvcb.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cvcb_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol(cb):
    from cvc_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    declared = _declared_symbols()
    assert len(declared) >= 30
    for name in declared:
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, name
    assert set(_lib.SIGNATURES) == set(declared)


def test_no_gpu_needed_for_host_api(cb):
    # geometry and generators work without touching a device
    assert cb.geometry_tables(2, 2, 2, 2)["g_iup"].size == 64
    assert cb.last_error() is not None


def test_stencil_timing_algorithmic_bytes():
    """Byte counts the profiles and the bench roofline use (24^3x48, 12 rhs)."""
    from cvc_b200.stencil_timing import algorithmic_bytes
    dims = (48, 24, 24, 24)
    assert algorithmic_bytes(1, 1, 12, 12, dims) == 891_813_888
    assert algorithmic_bytes(2, 1, 12, 12, dims) == 2 * 891_813_888 + 2 * 1_274_019_840
    # the fused |M p|^2 of a CG iteration reads no field: same bytes as M^+M alone
    assert algorithmic_bytes(3, 1, 12, 12, dims) == algorithmic_bytes(2, 1, 12, 12, dims)
    assert algorithmic_bytes(0, 0, 18, 1, dims) == 663_552 * 960
    # no-reuse counts: 3072 B per site for the FP64 operator; the packed FP32 sweep
    # reads 8 x 96 + 8 x 48 / 2 + 96 (+ 96 with the diagonal term) per site and rhs
    from cvc_b200.stencil_timing import flops, no_reuse_bytes
    assert flops(2, 12, dims) == 4 * 12 * 331_776 * 1392 and flops(0, 1, dims) == 663_552 * 1392
    assert no_reuse_bytes(0, 0, 18, 1, dims) == 663_552 * 3072
    assert no_reuse_bytes(1, 1, 12, 12, dims) == 12 * 331_776 * 1056
    assert no_reuse_bytes(2, 1, 12, 12, dims) == 12 * 331_776 * (2 * 1056 + 2 * 1152)


def test_tmlqcd_library_exports_the_wrapper_abi(cb):
    """libcvcb200_tmlqcd.so exports every function of the tmLQCD wrapper
    header (include/cvcb_tmlqcd.h, tmLQCD.h:46-54 of the reference)."""
    from cvc_b200 import _lib
    path = os.path.join(os.path.dirname(_lib.LIB_PATH), "libcvcb200_tmlqcd.so")
    lib = ctypes.CDLL(path)
    hdr = open(os.path.join(os.path.dirname(os.path.dirname(_lib.LIB_PATH)), "include",
                            "cvcb_tmlqcd.h")).read()
    names = set(re.findall(r"\bint\s+(tmLQCD_\w+)\s*\(", hdr))
    assert len(names) == 7
    for n in names:
        assert hasattr(lib, n), n


def test_host_api_error_convention(cb):
    """Host-only calls return the status codes of include/cvcb.h and set the
    thread's error text; none of them needs a device."""
    from cvc_b200 import _lib
    lib = _lib.load()
    perm = np.zeros(16 * 24, np.int32)
    assert lib.cvcb_gamma_tables(None, perm.ctypes.data) == _lib.CVCB_ERR_NULL
    ph = np.zeros(8)
    bc = np.array([1.0, 0.0, 0.0, 0.0])
    assert lib.cvcb_boundary_phases(8, 4, 4, 4, None, ph.ctypes.data) == _lib.CVCB_ERR_NULL
    assert lib.cvcb_boundary_phases(8, 0, 4, 4, bc.ctypes.data, ph.ctypes.data) == _lib.CVCB_ERR_ARG
    assert "extents" in cb.last_error()
    assert lib.cvcb_geometry_tables(0, 4, 4, 4, *([None] * 9)) == _lib.CVCB_ERR_ARG
    r = np.zeros(4)
    assert lib.cvcb_ranlxd(3, 1, r.ctypes.data, 4) == _lib.CVCB_ERR_ARG     # level 1 or 2
    assert lib.cvcb_ranlxd(1, 0, r.ctypes.data, 4) == _lib.CVCB_ERR_ARG     # seed > 0
    assert lib.cvcb_gauge_random(None, 2, 2, 2, 2, 0.3, 1) == _lib.CVCB_ERR_ARG
    out = ctypes.c_uint32()
    assert lib.cvcb_crc32(0, None, 4, ctypes.byref(out)) == _lib.CVCB_ERR_NULL
    assert lib.cvcb_crc32(0, None, 0, ctypes.byref(out)) == _lib.CVCB_OK and out.value == 0


def test_tmlqcd_wrapper_before_and_without_init(cb, tmp_path):
    """The tmLQCD wrapper's status codes on the paths that touch no device:
    every call before tmLQCD_invert_init is refused with 1, and init fails
    with 1 on a missing input file, one without the lattice extents or one
    with an operator block that is not closed
    (tmLQCD.h:46-54 of the reference; no exit() inside the library)."""
    from cvc_b200 import _lib
    lib = ctypes.CDLL(os.path.join(os.path.dirname(_lib.LIB_PATH), "libcvcb200_tmlqcd.so"))
    assert lib.tmLQCD_finalise() == 0
    buf = (ctypes.c_double * 24)()
    assert lib.tmLQCD_invert(buf, buf, 0, 0) == 1
    assert lib.tmLQCD_read_gauge(0) == 1
    gf = ctypes.c_void_p()
    assert lib.tmLQCD_get_gauge_field_pointer(ctypes.byref(gf)) == 1
    params = (ctypes.c_uint * 16)()
    assert lib.tmLQCD_get_lat_params(params) == 1
    assert lib.tmLQCD_get_mpi_params(params) == 1

    def init(path):
        argv = (ctypes.c_char_p * 3)(b"prog", b"-f", str(path).encode())
        return lib.tmLQCD_invert_init(3, argv, 0)

    assert init(tmp_path / "missing.input") == 1
    no_extents = tmp_path / "invert.input"
    no_extents.write_text("# no T or L\nkappa = 0.15\n2KappaMu = 0.01\n")
    assert init(no_extents) == 1
    open_block = tmp_path / "open.input"
    open_block.write_text("T = 8\nL = 4\nBeginOperator TMWILSON\n  kappa = 0.15\n")
    assert init(open_block) == 1
    assert lib.tmLQCD_read_gauge(0) == 1     # still not initialised
    assert lib.tmLQCD_finalise() == 0


def test_gauge_recipe_restatement(cb):
    """The numpy restatement of the gauge recipe (used where the CUDA library
    must not be loaded: the reference arm of bench.py) agrees with the
    library's generator to rounding."""
    import sys
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import gauge_recipe
    for dims, eps, seed in [((8, 4, 4, 4), 0.3, 1234), ((4, 6, 2, 4), 0.25, 11)]:
        a = cb.gauge_random(*dims, eps, seed)
        b = gauge_recipe.gauge_random(*dims, eps, seed, cb.ranlxd)
        assert np.max(np.abs(a - b)) < 1e-14
