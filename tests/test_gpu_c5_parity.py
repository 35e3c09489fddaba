"""Parity of the P -> gamma gamma pipeline at its benchmark configuration:
32^3x64, kappa 0.156, 2 kappa mu 0.004, gauge U = exp(i 0.3 H) of ranlxd
seed 21, source-sink separation 16, the first source position of the
ranlxd stream of seed 21, zero momentum, pseudoscalar insertion (gamma 5),
FP32 inner iterations (cvc_b200.p2gg: 120 forward and 60 sequential solves,
the conserved-current contraction of p2gg_xspace.c:615-899).

Checked against the oracle on the same inputs:
* the sequential source of the first forward column on the sink timeslice
  (p2gg_xspace.c:525-539): 1e-14;
* that sequential propagator solves Q x = source with the oracle's operator
  to the solver tolerance 1e-10 (Q_phi.c:38-188);
* Pi_mu_nu with the up columns replaced by the sequential propagators, at
  521 sites (the source, its neighbours and random sites) against the
  oracle's contraction of the same columns: 1e-12 relative to the largest
  |Pi| there; the contact term to 1e-12.
The pipeline holds 180 columns of 403 MB on the device (about 105 GB with
the solver's work space)."""
import os
import sys

import numpy as np
import pytest

from conftest import ROOT, rel_err

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

pytestmark = pytest.mark.gpu

DIMS = (64, 32, 32, 32)
KAPPA, MU2K = 0.156, 0.004
MU = MU2K / (2 * KAPPA)
EPS, SEED, DT, MOM, GID = 0.3, 21, 16, (0, 0, 0), 5


def test_c5_p2gg_against_oracle(cb, oracle_mod):
    torch = pytest.importorskip("torch")
    from cvc_b200.p2gg import p2gg
    import inputs
    free, _ = torch.cuda.mem_get_info()
    if free < 120e9:
        pytest.skip(f"needs about 120 GB of free device memory ({free / 1e9:.0f} GB free)")
    T, LX, LY, LZ = DIMS
    V = T * LX * LY * LZ
    r = cb.ranlxd(4, SEED)
    c = [int(r[i] * n) % n for i, n in enumerate(DIMS)]
    site = ((c[0] * LX + c[1]) * LY + c[2]) * LZ + c[3]
    g = cb.gauge_random(*DIMS, EPS, SEED)
    lat = cb.Lattice(*DIMS, kappa=KAPPA, mu=MU)
    lat.upload_gauge(g)
    p = cb.solver_defaults()
    p.block_rhs = 12
    keep = {}
    conn, contact, st = p2gg(lat, site, DT, MOM, GID, 0, p, keep=keep)
    assert st["solves"] == 180 and st["max_true_res"] <= 1e-10
    orc = oracle_mod.Oracle(*DIMS, KAPPA, MU)
    orc.set_gauge(g)
    # sequential source of the first forward column
    up0 = keep["up0"].cpu().numpy()
    src0 = keep["seq_source0"].cpu().numpy()
    want = orc.seq_source(up0, keep["t_seq"], MOM, GID, 0)
    assert rel_err(src0, want) < 1e-14
    del up0, want
    # its sequential propagator solves Q x = source (the oracle's operator)
    fields = keep["fields"]
    x0 = fields[0].cpu().numpy()
    res = src0 - orc.Q_phi_tbc(x0)
    assert np.linalg.norm(res) <= 1.02e-10 * np.linalg.norm(src0)
    del x0, res, src0
    # Pi at sample sites against the oracle's contraction of the same columns
    sample = inputs.sample_sites(DIMS, site, 512)
    dev = conn.device
    got = conn.view(-1, 32)[torch.as_tensor(sample, device=dev)].cpu().numpy()

    def fetch(idx):
        it = torch.as_tensor(idx, device=dev)
        return [f.view(-1, 24)[it].cpu().numpy() for f in fields]

    want, ocontact = orc.cvc_contract_sites(sample, site, fetch)
    assert rel_err(got, want) < 1e-12
    assert np.max(np.abs(contact - ocontact)) < 1e-12 * np.max(np.abs(ocontact))
    keep.clear()
    lat.close()
