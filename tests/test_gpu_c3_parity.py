"""Parity at the solver benchmark's configuration: 24^3x48, kappa 0.155,
2 kappa mu 0.005, gauge U = exp(i 0.25 H) of ranlxd seed 11, antiperiodic in
time.

* The gauge field is the fixture's: its plaquette equals the one the
  reference computed (tests/golden/reference_c3.npz, made by
  tests/golden/make_golden_configs.py from the unmodified reference).
* Q_phi_tbc, Qf5(+-mu) and Hopping on the full lattice against the oracle
  (Q_phi.c:38-188, :789-934, :399-528): 1e-14 relative to the largest
  component.
* Two point-source columns of the benchmark's first source, solved by the
  batched mixed-precision solver (FP32 and FP16+norm inner iterations, FP64
  reliable updates) and by the FP64 mirror of invert_Qtm_her, against the
  reference's invert_Qtm_her solutions at 2,057 sites (the source, its
  neighbours, 2,048 more) and their norms: 1e-8 (both sides reach a
  relative residual of 1e-12; solutions differ by up to cond(Q) times
  that).  The benchmark's own criterion, |b - Q x| / |b| <= 1e-10, is
  recomputed with the oracle's operator, and the mirror's iteration count
  is the reference's within 10 %.
* Pi_mu_nu of the 120 columns of that source (cvc_exact2_xspace.c:577-861),
  solved and contracted on the GPU, against the oracle's contraction of the
  same propagators at 521 sites including the source and its neighbours:
  1e-12 relative to the largest |Pi| there; the contact term to 1e-12.
"""
import os

import numpy as np
import pytest

from conftest import ROOT, rel_err, seeded

pytestmark = pytest.mark.gpu

DIMS = (48, 24, 24, 24)
KAPPA = 0.155
MU = 0.005 / (2 * KAPPA)
FIX = os.path.join(ROOT, "tests", "golden", "reference_c3.npz")


@pytest.fixture(scope="module")
def c3(cb, oracle_mod):
    fix = np.load(FIX)
    g = cb.gauge_random(*DIMS, 0.25, 11)
    lat = cb.Lattice(*DIMS, kappa=KAPPA, mu=MU)
    lat.upload_gauge(g)
    orc = oracle_mod.Oracle(*DIMS, KAPPA, MU)
    orc.set_gauge(g)
    yield lat, orc, fix
    lat.close()


def point_source(site, sc):
    V = int(np.prod(DIMS))
    b = np.zeros(24 * V)
    b[24 * site + 2 * sc] = 1.0
    return b


def test_c3_gauge_matches_fixture(c3):
    lat, orc, fix = c3
    pl, _ = orc.plaquette()
    assert abs(pl - float(fix["plaquette"])) < 1e-14
    assert abs(lat.plaquette()[0] - float(fix["plaquette"])) < 1e-13


def test_c3_operators(c3):
    lat, orc, _ = c3
    V = lat.VOLUME
    phi = seeded(31, 24 * V)
    out = np.zeros(24 * V)
    lat.Q_phi_tbc(out, phi)
    assert rel_err(out, orc.Q_phi_tbc(phi)) < 1e-14
    for m in (MU, -MU):
        lat.Qf5(out, phi, m)
        assert rel_err(out, orc.Qf5(phi, m)) < 1e-14
    lat.Hopping(out, phi)
    assert rel_err(out, orc.Hopping(phi)) < 1e-14


@pytest.mark.parametrize("prec", [1, 2], ids=["fp32-inner", "fp16-inner"])
def test_c3_batched_solutions_against_reference(cb, c3, prec):
    lat, orc, fix = c3
    site = int(fix["source_site"])
    sites = fix["sites"]
    cols = [int(c) for c in fix["cfg_columns"]]
    bs = [point_source(site, sc) for sc in cols]
    xs = [np.zeros_like(b) for b in bs]
    p = cb.solver_defaults()
    p.precision, p.link_recon, p.tol = prec, 12, 1e-12
    st = lat.solve(xs, bs, p)
    assert st.converged == len(cols) and st.max_true_res <= 1e-12
    for k, (x, b) in enumerate(zip(xs, bs)):
        xr = fix["x_sites"][k]
        assert rel_err(x.reshape(-1, 24)[sites], xr) < 1e-8
        assert abs(np.dot(x, x) / fix["x_norm2"][k] - 1) < 1e-8
    # the benchmark's criterion with the oracle's operator, at its tolerance
    p.tol = 1e-10
    x = np.zeros_like(bs[0])
    st = lat.solve([x], [bs[0]], p)
    assert st.converged == 1
    r = bs[0] - orc.Q_phi_tbc(x)
    assert np.linalg.norm(r) <= 1.02e-10 * np.linalg.norm(bs[0])


def test_c3_fp64_mirror_against_reference(c3):
    lat, orc, fix = c3
    site = int(fix["source_site"])
    sc = int(fix["cfg_columns"][0])
    b = point_source(site, sc)
    x = np.zeros_like(b)
    n, tr2 = lat.invert_Qtm_her(x, b, float(fix["cfg_precision"]), 20000, return_residual=True)
    nref = int(fix["iterations"][0])
    assert n > 0 and abs(n - nref) <= max(3, nref // 10), (n, nref)
    assert tr2 < 1e-23
    assert rel_err(x.reshape(-1, 24)[fix["sites"]], fix["x_sites"][0]) < 1e-8


def test_c3_pi_against_oracle_contraction(cb, c3):
    torch = pytest.importorskip("torch")
    from cvc_b200.p2gg import shifted_sites
    lat, orc, fix = c3
    V = lat.VOLUME
    site = int(fix["source_site"])
    sample = fix["sites"][:521]
    dev = torch.device("cuda", 0)
    p = cb.solver_defaults()
    cols = {}
    for flav, m in (("up", MU), ("dn", -MU)):
        bs, xs = [], []
        for s in shifted_sites(DIMS, site):
            for sc in range(12):
                b = torch.zeros(24 * V, dtype=torch.float64, device=dev)
                b[24 * s + 2 * sc] = 1.0
                bs.append(b)
                xs.append(torch.zeros_like(b))
        lat.set_params(KAPPA, m, (1.0, 0.0, 0.0, 0.0))
        st = lat.solve(xs, bs, p)
        assert st.converged == 60
        cols[flav] = xs
        del bs
    lat.set_params(KAPPA, MU, (1.0, 0.0, 0.0, 0.0))
    fields = cols["up"] + cols["dn"]
    conn = torch.zeros(32 * V, dtype=torch.float64, device=dev)
    conn, contact = lat.cvc_contract(fields, site, conn=conn)
    got = conn.view(-1, 32)[torch.as_tensor(sample, device=dev)].cpu().numpy()

    def fetch(idx):
        it = torch.as_tensor(idx, device=dev)
        return [f.view(-1, 24)[it].cpu().numpy() for f in fields]

    want, ocontact = orc.cvc_contract_sites(sample, site, fetch)
    assert rel_err(got, want) < 1e-12
    assert np.max(np.abs(contact - ocontact)) < 1e-12 * np.max(np.abs(ocontact))
