"""Error of Pi_mu_nu(x) computed from mixed-precision propagators against
the FP64 one (16^3x32, kappa 0.150, 2 kappa mu 0.01, gauge eps 0.3 seed 7,
source at the origin: 120 columns per flavour pair and shift).

Each mixed solve meets |b - Q x| / |b| <= 1e-10 in FP64, so each column
differs from its FP64 solution by about cond(Q) * 1e-10; Pi is bilinear in
the columns, so its relative error is of that size too.  Stated per output:
the whole field, each (mu, nu) component, and the contact term; asserted at
1e-8 relative (L2) and printed with -s."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DIMS = (32, 16, 16, 16)
KAPPA, MU = 0.150, 0.01 / 0.3


@pytest.fixture(scope="module")
def pis(cb):
    lat = cb.Lattice(*DIMS, kappa=KAPPA, mu=MU)
    lat.upload_gauge(cb.gauge_random(*DIMS, 0.3, 7))
    out = {}
    for name, prec, recon, tol in [("fp64", cb.PREC_DOUBLE, 18, 1e-12),
                                   ("fp32", cb.PREC_SINGLE, 12, 1e-10),
                                   ("fp16", cb.PREC_HALF, 12, 1e-10)]:
        p = cb.solver_defaults()
        p.precision, p.link_recon, p.tol = prec, recon, tol
        conn, contact = lat.pi_forward(0, p, keep_bytes=0)
        out[name] = (conn.copy(), contact.copy())
    lat.close()
    return out


@pytest.mark.parametrize("name", ["fp32", "fp16"])
def test_mixed_pi_error(pis, name):
    c64, k64 = pis["fp64"]
    c, k = pis[name]
    z64 = (c64[0::2] + 1j * c64[1::2]).reshape(-1, 4, 4)
    z = (c[0::2] + 1j * c[1::2]).reshape(-1, 4, 4)
    total = np.linalg.norm(z - z64) / np.linalg.norm(z64)
    worst = np.max(np.abs(z - z64)) / np.max(np.abs(z64))
    comp = np.array([[np.linalg.norm(z[:, m, n] - z64[:, m, n]) / np.linalg.norm(z64[:, m, n])
                      for n in range(4)] for m in range(4)])
    contact = np.linalg.norm(k - k64) / np.linalg.norm(k64)
    print(f"\n{name}: Pi rel L2 {total:.3e}, max|dPi|/max|Pi| {worst:.3e}, "
          f"contact {contact:.3e}, per (mu,nu) max {comp.max():.3e} min {comp.min():.3e}")
    assert total < 1e-8
    assert comp.max() < 1e-8
    assert contact < 1e-8
