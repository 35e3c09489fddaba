"""Pi_mu_nu contraction (cvc_exact2_xspace.c:577-861), Ward identity
(:928-1008) and the p2gg sequential source (p2gg_xspace.c:525-539) on the
GPU against the oracle.  FP64: 1e-12 relative to the largest |Pi| (the GPU
restructures the 4608 sweeps into 24 hop-and-dot passes, so the summation
order differs)."""
import numpy as np
import pytest

from conftest import rel_err, seeded

pytestmark = pytest.mark.gpu

DIMS = (8, 4, 4, 4)
KAPPA, MU = 0.15, 0.01 / 0.3


@pytest.fixture(scope="module")
def env(cb, oracle_mod):
    lat = cb.Lattice(*DIMS, kappa=KAPPA, mu=MU)
    g = cb.gauge_random(*DIMS, 0.3, 1234)
    lat.upload_gauge(g)
    orc = oracle_mod.Oracle(*DIMS, KAPPA, MU)
    orc.set_gauge(g)
    yield lat, orc, g
    lat.close()


@pytest.mark.parametrize("src", [0, 37, 511])
def test_contract_random_fields(env, src):
    lat, orc, _ = env
    V = lat.VOLUME
    fields = [seeded(1000 + i, 24 * V) for i in range(120)]
    conn, contact = lat.cvc_contract(fields, src)
    oconn, ocontact = orc.cvc_contract(fields, src)
    assert rel_err(conn, oconn) < 1e-12
    assert np.max(np.abs(contact - ocontact)) < 1e-12 * np.max(np.abs(ocontact))


def test_ward_identity_with_solved_propagators(cb, env):
    """With propagators that solve Q x = delta_{y+mu}, the conserved current
    is conserved: the divergence vanishes except at y and y+nu, where it is
    +/- the contact term the reference prints."""
    lat, orc, g = env
    V = lat.VOLUME
    T, LX, LY, LZ = DIMS
    src = 0  # y = (0,0,0,0)
    shifted = [LX * LY * LZ, LY * LZ, LZ, 1, 0]  # y + mu for mu = 0..3, then y
    bs = []
    for m in range(5):
        for sc in range(12):
            b = np.zeros(24 * V)
            b[24 * shifted[m] + 2 * sc] = 1.0
            bs.append(b)
    p = cb.solver_defaults()
    p.tol = 1e-13
    up = [np.zeros(24 * V) for _ in range(60)]
    st = lat.solve(up, bs, p)
    assert st.converged == 60
    # dn flavour: mu -> -mu
    lat.set_params(KAPPA, -MU)
    dn = [np.zeros(24 * V) for _ in range(60)]
    st = lat.solve(dn, bs, p)
    assert st.converged == 60
    lat.set_params(KAPPA, MU)
    conn, contact = lat.cvc_contract(up + dn, src)
    wi = lat.cvc_ward(conn).reshape(V, 4, 2)
    owi = orc.cvc_ward(conn).reshape(V, 4, 2)
    assert np.max(np.abs(wi - owi)) < 1e-13
    scale = np.max(np.abs(conn))
    for nu in range(4):
        w = wi[:, nu, 0] + 1j * wi[:, nu, 1]
        ct = contact[2 * nu] + 1j * contact[2 * nu + 1]
        nb = shifted[nu]
        assert abs(ct) > 1e-3
        assert abs(w[src] - ct) < 1e-9 * scale
        assert abs(w[nb] + ct) < 1e-9 * scale
        others = np.delete(np.abs(w), [src, nb])
        assert np.max(others) < 1e-9 * scale
    # and the GPU contraction equals the oracle's on these propagators
    oconn, ocontact = orc.cvc_contract(up + dn, src)
    assert rel_err(conn, oconn) < 1e-12


@pytest.mark.parametrize("t,mom,gid,pos", [(3, (1, 0, 2), 5, 0), (7, (0, 1, 1), 4, 1),
                                           (0, (2, 3, 1), 6, 0)])
def test_seq_source(env, t, mom, gid, pos):
    lat, orc, _ = env
    V = lat.VOLUME
    prop = seeded(77, 24 * V)
    src = np.zeros(24 * V)
    lat.p2gg_seq_source(src, prop, t, mom, gid, pos)
    ref = orc.seq_source(prop, t, mom, gid, pos)
    assert rel_err(src, ref) < 1e-14


VARIANT_CHILD = r"""
import sys
import numpy as np
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[1] + "/tests")
import cvc_b200 as cb
from conftest import seeded
dims = (8, 4, 4, 6)
lat = cb.Lattice(*dims, kappa=0.15, mu=0.01 / 0.3)
lat.upload_gauge(cb.gauge_random(*dims, 0.3, 1234))
V = lat.VOLUME
fields = [seeded(3000 + i, 24 * V) for i in range(120)]
conn, contact = lat.cvc_contract(fields, 41)
np.save(sys.argv[2], conn)
"""


def test_pi_kernel_variants_agree(tmp_path):
    """Every Pi kernel the contraction times on first use (one thread per
    site at three register caps, one thread per site and mu at three),
    pinned by CVCB_CVC_PI in a child process: the same Pi to the last bit
    (the same terms, accumulated in the same order)."""
    import os
    import subprocess
    import sys
    from conftest import ROOT
    out = {}
    for v in range(6):
        f = tmp_path / f"pi{v}.npy"
        env = dict(os.environ, CVCB_CVC_PI=str(v))
        r = subprocess.run([sys.executable, "-c", VARIANT_CHILD, str(ROOT), str(f)], env=env,
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        out[v] = np.load(f)
    for v in range(1, 6):
        assert np.array_equal(out[v], out[0]), (v, float(np.max(np.abs(out[v] - out[0]))))
