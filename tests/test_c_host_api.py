"""The host-only part of the C ABI called from a C99 program
(tests/compat/host_api_driver.c, compiled here with -std=c99 -pedantic
against include/cvcb.h): its results must equal the same calls made from
Python, and the LIME files it writes must read back bit for bit.  No GPU."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT

DIMS = (8, 4, 4, 2)


def weighted_int(a, m=7):
    a = np.asarray(a, np.int64).reshape(-1)
    return int(np.sum((np.arange(a.size) % m + 1) * a))


def weighted_float(a, m=5):
    """The driver's left-to-right double sum with weights i % m + 1."""
    s = 0.0
    for i, v in enumerate(np.asarray(a, np.float64).reshape(-1)):
        s += float(i % m + 1) * float(v)
    return s


def test_c_program_matches_python(cb, tmp_path):
    from cvc_b200 import lime
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    exe = tmp_path / "host_api_driver"
    libdir = os.path.join(ROOT, "cvc_b200")
    subprocess.run([cc, "-std=c99", "-pedantic", "-Wall", "-Werror", "-O2", "-o", str(exe),
                    os.path.join(ROOT, "tests/compat/host_api_driver.c"),
                    "-I" + os.path.join(ROOT, "include"), "-L" + libdir, "-lcvcb200",
                    "-Wl,-rpath," + libdir], check=True)
    out = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    tok = out.stdout.split()
    got = {}
    i = 0
    while i < len(tok):
        key = tok[i]
        n = 4 if key.endswith("_sums") else 1
        got[key] = tok[i + 1:i + 1 + n]
        i += 1 + n

    tabs = cb.geometry_tables(*DIMS)
    assert int(got["ipt"][0]) == weighted_int(tabs["g_ipt"])
    assert int(got["iup"][0]) == weighted_int(tabs["g_iup"])
    assert int(got["idn"][0]) == weighted_int(tabs["g_idn"])
    assert int(got["lexic2eo"][0]) == weighted_int(tabs["g_lexic2eo"])
    perm, sign = cb.gamma_tables()
    assert int(got["perm"][0]) == weighted_int(perm) and int(got["sign"][0]) == weighted_int(sign)
    ph = cb.boundary_phases(*DIMS, (1.0, 0.5, 0.0, 0.25))
    assert float(got["ph"][0]) == weighted_float(np.stack([ph.real, ph.imag], -1))
    r = cb.ranlxd(1000, 17, level=1)
    assert float(got["ranlxd"][0]) == weighted_float(r)
    g = cb.gauge_random(*DIMS, 0.3, 1234)
    assert float(got["gauge"][0]) == weighted_float(g)
    assert int(got["crc"][0]) == lime.crc32(b"cvc-b200")

    # files written from C read back from Python, with the same checksums
    g2, gsums = lime.read_lime_gauge_field(tmp_path / "gauge.ildg", DIMS)
    assert np.array_equal(g2, g)
    assert [int(v) for v in got["gauge_sums"]] == [*gsums, *gsums]
    s = np.resize(r - 0.5, 24 * int(np.prod(DIMS)))
    s2, ssums = lime.read_lime_spinor(tmp_path / "spinor.lime", DIMS)
    assert np.array_equal(s2, s)
    assert [int(v) for v in got["spinor_sums"]] == [*ssums, *ssums]
    assert got["gauge_same"] == ["1"] and got["spinor_same"] == ["1"]
