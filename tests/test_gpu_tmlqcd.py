"""The tmLQCD library-wrapper ABI (libcvcb200_tmlqcd.so) driven by a C
program that makes the calls of cvc_exact2_xspace.c's tmLQCD branch: input
file with two operators (+2 kappa mu and -2 kappa mu), an ILDG gauge file
written by cvc_b200.lime, 2 x 12 point-source inversions.  Propagators must
equal the oracle's FP64 solutions of Q x = b divided by 2 kappa (tmLQCD's
normalisation) to 1e-8, the gauge field pointer must hold the file's field,
the propagator written with write_prop must read back, and SolverPrecision
is an absolute squared residual as in tmLQCD."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT, rel_err

pytestmark = pytest.mark.gpu

DIMS = (8, 4, 4, 4)
V = 512
KAPPA, TWO_KAPPA_MU = 0.150, 0.01
SRC = (1, 2, 3, 0)


def test_tmlqcd_abi(cb, oracle_mod, tmp_path):
    from cvc_b200 import lime
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    exe = tmp_path / "tmlqcd_driver"
    libdir = os.path.join(ROOT, "cvc_b200")
    subprocess.run([cc, "-O2", "-o", str(exe), os.path.join(ROOT, "tests/compat/tmlqcd_driver.c"),
                    "-I" + os.path.join(ROOT, "include"), "-L" + libdir, "-lcvcb200_tmlqcd",
                    "-Wl,-rpath," + libdir], check=True)
    g = cb.gauge_random(*DIMS, 0.3, 1234)
    lime.write_lime_gauge_field(tmp_path / "conf.0005", g, DIMS)
    (tmp_path / "invert.input").write_text(
        "T = 8\nL = 4\nInitialStoreCounter = 5\nGaugeConfigInputFile = conf\n"
        "ThetaT = 1.0\nPropagatorFilePrefix = source\nGPUPrecision = single\n"
        f"BeginOperator TMWILSON\n  2KappaMu = {TWO_KAPPA_MU}\n  kappa = {KAPPA}\n"
        "  SolverPrecision = 1e-24\nEndOperator\n"
        f"BeginOperator TMWILSON\n  2KappaMu = {-TWO_KAPPA_MU}\n  kappa = {KAPPA}\n"
        "  SolverPrecision = 1e-24\nEndOperator\n")
    out = subprocess.run([str(exe), "-f", "invert.input", *map(str, SRC), str(tmp_path)],
                         cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    assert np.array_equal(np.fromfile(tmp_path / "gauge.raw"), g)
    mu = TWO_KAPPA_MU / (2 * KAPPA)
    orc = oracle_mod.Oracle(*DIMS, KAPPA, mu)
    orc.set_gauge(g)
    ix = ((SRC[0] * 4 + SRC[1]) * 4 + SRC[2]) * 4 + SRC[3]
    for op, m in enumerate((mu, -mu)):
        orc.set_params(KAPPA, m)
        for ia in range(12):
            b = np.zeros(24 * V)
            b[24 * ix + 2 * ia] = 1.0
            _, x, _ = orc.invert(b, 1e-26, 5000, her=True)
            p = np.fromfile(tmp_path / f"prop.{op}.{ia:02d}.raw")
            assert rel_err(p, x / (2 * KAPPA)) < 1e-8, (op, ia)
    # SolverPrecision 1e-24 is absolute: for a source of norm 1e-3 the solve
    # reaches |b - Q x|^2 <= 1e-24, i.e. a relative 1e-9 (not 1e-12)
    orc.set_params(KAPPA, mu)
    b = np.zeros(24 * V)
    b[24 * ix] = 1e-3
    p = np.fromfile(tmp_path / "prop.scaled.raw")
    r = b - orc.Q_phi_tbc(2 * KAPPA * p)
    assert np.dot(r, r) <= 1e-24
    _, x, _ = orc.invert(b, 1e-26, 5000, her=True)
    assert rel_err(p, x / (2 * KAPPA)) < 1e-5
    written, _ = lime.read_lime_spinor(tmp_path / "source.0005.00.inverted", DIMS, 0)
    assert np.array_equal(written, np.fromfile(tmp_path / "prop.0.00.raw"))
