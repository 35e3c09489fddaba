"""Every launch variant of the batched stencil, pinned by CVCB_SHAPE in a
child process (the autotuner caches one shape per configuration and
process): one rhs per thread with per-thread links, shared-memory links
for several rows, 2 and 4 rhs per thread, packed FP32x2 rhs pairs, and
(FP32 only, CVCB_PAIRS=1) the pair-tiled fields with 12- and 18-real
links, with plain neighbour loads, with the t and x neighbours staged in
shared memory by bulk copies (4th shape field 2) and with the accumulator in
tensor memory at both register budgets (4th shape field 3, 4).
A wrong sloppy operator would still be corrected by the FP64 reliable
updates, so each variant must also converge in the same number of inner
iterations as the plain one (the arithmetic differs only in rounding)."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import cvc_b200 as cb
prec = int(sys.argv[2])
recon = int(sys.argv[3])
dims = (16, 8, 8, 8)
V = 16 * 8 ** 3
lat = cb.Lattice(*dims, kappa=0.155, mu=0.005 / 0.31)
lat.upload_gauge(cb.gauge_random(*dims, 0.25, 11))
bs = []
for i in range(11):                       # odd count: a lone last rhs in pair kernels
    b = np.zeros(24 * V); b[24 * (37 * i) + 2 * (i % 12)] = 1.0; bs.append(b)
xs = [np.zeros(24 * V) for _ in bs]
p = cb.solver_defaults(); p.precision = prec; p.block_rhs = 11; p.link_recon = recon
st = lat.solve(xs, bs, p)
r = np.zeros(24 * V); lat.Q_phi_tbc(r, xs[4])
print(json.dumps({"iters": st.iterations, "conv": st.converged, "res": st.max_true_res,
                  "chk": float(np.linalg.norm(r - bs[4]) / np.linalg.norm(bs[4])),
                  "x4": float(np.abs(xs[4]).sum())}))
"""

VARIANTS = ["64,1,1", "32,4,1", "64,1,2", "32,1,4", "64,1,2,1", "32,2,2,1"]
# (shape, CVCB_PAIRS, link reals) of the pair-tiled fields
PAIR_VARIANTS = [("64,1,2,1", 1, 12), ("32,2,2,1", 1, 12), ("64,1,2,1", 1, 18),
                 ("128,1,2,1", 1, 18), ("128,1,2,2", 1, 12), ("128,1,2,2", 1, 18),
                 ("128,1,2,3", 1, 12), ("128,1,2,3", 1, 18), ("128,1,2,4", 1, 12),
                 ("128,1,2,4", 1, 18)]


def run(prec, shape, pairs=0, recon=12):
    env = dict(os.environ, CVCB_SHAPE=shape, CVCB_PAIRS=str(pairs))
    out = subprocess.run([sys.executable, "-c", CHILD, str(ROOT), str(prec), str(recon)],
                         env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    return json.loads(out.stdout.strip().splitlines()[-1])


@pytest.mark.parametrize("prec", [1, 2], ids=["fp32", "fp16"])
def test_stencil_variants_agree(prec):
    res = {v: run(prec, v) for v in VARIANTS}
    if prec == 1:
        res.update({f"pairs {v} {r}": run(prec, v, pt, r) for v, pt, r in PAIR_VARIANTS})
    base = res["64,1,1"]
    print({v: r["iters"] for v, r in res.items()})
    for v, r in res.items():
        assert r["conv"] == 11, (v, r)
        assert r["res"] <= 1e-10 and r["chk"] <= 1e-10, (v, r)
        assert abs(r["iters"] - base["iters"]) <= 0.1 * base["iters"], (v, r, base)
        assert abs(r["x4"] - base["x4"]) <= 1e-8 * base["x4"], (v, r, base)
