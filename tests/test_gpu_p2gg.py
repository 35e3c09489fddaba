"""The P -> gamma gamma pipeline (cvc_b200.p2gg: forward solves of both
flavours for the source and its four forward neighbours, sequential sources
of p2gg_xspace.c:525-539, sequential solves, conserved-current contraction
of p2gg_xspace.c:615-899) against the same pipeline run by the oracle on
the CPU.  Tolerances: both sides solve to a relative residual of about
1e-12, so Pi agrees to about cond(Q) * 1e-12; asserted at 1e-9 for FP64
inner iterations and at 1e-7 for FP32 (solver tolerance 1e-10)."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

DIMS = (8, 4, 4, 4)
V = 512
KAPPA, MU = 0.156, 0.004 / 0.312
SRC, DT, MOM, GID = 37, 4, (1, 0, 2), 5


@pytest.fixture(scope="module")
def oracle_pi(oracle_mod, cb):
    from cvc_b200.p2gg import shifted_sites
    g = cb.gauge_random(*DIMS, 0.3, 21)
    orc = oracle_mod.Oracle(*DIMS, KAPPA, MU)
    orc.set_gauge(g)
    bs = []
    for s in shifted_sites(DIMS, SRC):
        for sc in range(12):
            b = np.zeros(24 * V)
            b[24 * s + 2 * sc] = 1.0
            bs.append(b)

    def solve(m):
        orc.set_params(KAPPA, m)
        out = []
        for b in bs_now:
            rc, x, _ = orc.invert(b, 1e-26, 5000, her=True)
            assert rc > 0
            out.append(x)
        return out

    out = {}
    for pos in (0, 1):
        bs_now = bs
        up, dn = solve(MU), solve(-MU)
        t_seq = (SRC // 64 + DT) % DIMS[0]
        bs_now = [orc.seq_source(u, t_seq, MOM, GID, pos) for u in up]
        seq = solve(MU if pos == 0 else -MU)
        orc.set_params(KAPPA, MU)
        out[pos] = orc.cvc_contract(seq + dn, SRC)
    return g, out


@pytest.mark.parametrize("pos", [0, 1])
@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "fp32"])
def test_p2gg_pipeline(cb, oracle_pi, pos, prec):
    torch = pytest.importorskip("torch")
    from cvc_b200.p2gg import p2gg
    g, ref = oracle_pi
    lat = cb.Lattice(*DIMS, kappa=KAPPA, mu=MU)
    lat.upload_gauge(g)
    p = cb.solver_defaults()
    p.precision = prec
    p.link_recon = 18 if prec == 0 else 12
    p.tol = 1e-12 if prec == 0 else 1e-10
    conn, contact, st = p2gg(lat, SRC, DT, MOM, GID, pos, p)
    assert st["solves"] == 180
    oconn, ocontact = ref[pos]
    tol = 1e-9 if prec == 0 else 1e-7
    assert rel_err(conn.cpu().numpy(), oconn) < tol
    assert rel_err(contact, ocontact) < tol
    lat.close()
