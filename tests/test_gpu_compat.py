"""Link-level drop-in: a program built from the unmodified reference
objects (geometry, utilities) and libcvcb200_cvc.so in place of Q_phi.o and
invert_Qtm.o (tests/compat/compat_driver.cpp, built by `make -C oracle
compat` where the reference tree is present).  Its outputs are compared
with the oracle; the reference's own check_source, which calls Q_phi and
spinor_scalar_product_re, runs through the GPU library too."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT, rel_err, seeded

pytestmark = pytest.mark.gpu

DRIVER = os.path.join(ROOT, "oracle", "_ref", "compat_driver")


def test_reference_program_links_and_runs_on_gpu(cb, oracle_mod):
    if not os.path.exists(DRIVER):
        pytest.skip("compat driver not built (needs the reference tree at build time)")
    dims, kappa, mu = (8, 4, 4, 4), 0.15, 0.01 / 0.3
    V = 8 * 64
    g = cb.gauge_random(*dims, 0.3, 1234)
    phi = seeded(21, 24 * V)
    orc = oracle_mod.Oracle(*dims, kappa, mu)
    orc.set_gauge(g)
    with tempfile.TemporaryDirectory() as d:
        g.tofile(os.path.join(d, "g.bin"))
        phi.tofile(os.path.join(d, "phi.bin"))
        out = subprocess.run([DRIVER, *map(str, dims), repr(kappa), repr(mu),
                              os.path.join(d, "g.bin"), os.path.join(d, "phi.bin"),
                              os.path.join(d, "out")], capture_output=True, text=True,
                             timeout=300)
        assert out.returncode == 0, out.stderr[-2000:]
        q = np.fromfile(os.path.join(d, "out.Q_phi_tbc"))
        f5 = np.fromfile(os.path.join(d, "out.Qf5_minus"))
        x = np.fromfile(os.path.join(d, "out.x"))
        q_edit = np.fromfile(os.path.join(d, "out.Q_phi_tbc_edit"))
    assert rel_err(q, orc.Q_phi_tbc(phi)) < 1e-14
    qf5 = orc.Qf5(phi, -mu)
    assert rel_err(f5, qf5) < 1e-14
    lines = out.stdout.splitlines()
    dot = [l for l in lines if l.startswith("dot")][0].split()
    ref = orc.scalar_product_co(phi, qf5, V)
    assert abs(complex(float(dot[1]), float(dot[2])) - ref) < 1e-12 * abs(ref)
    niter = int([l for l in lines if l.startswith("niter")][0].split()[1])
    b = np.zeros(24 * V)
    b[8] = 1.0
    n2, xo, _ = orc.invert(b, 1e-20, 2000, her=True)
    assert niter > 0 and abs(niter - n2) <= max(3, n2 // 10)
    assert rel_err(x, xo) < 1e-8
    # the reference's check_source printed |Q x - delta|^2 via the GPU Q_phi
    res = [l for l in lines if "norm of A x - delta" in l][0]
    assert float(res.split("=")[1]) < 1e-18
    # the point-source breakdown keeps the reference's return value
    assert int([l for l in lines if l.startswith("breakdown")][0].split()[1]) == -3
    # one link edited in place (site 37, mu 2, times e^{0.7 i}) is picked up
    ge = g.copy()
    u = ge[18 * (4 * 37 + 2):18 * (4 * 37 + 2) + 18].view(np.complex128)
    u *= np.exp(0.7j)
    orc.set_gauge(ge)
    want = orc.Q_phi_tbc(phi)
    assert rel_err(q_edit, want) < 1e-14
    orc.set_gauge(g)
    assert rel_err(q_edit, orc.Q_phi_tbc(phi)) > 1e-6
