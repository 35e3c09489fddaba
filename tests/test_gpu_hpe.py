"""Hopping-parameter-expansion helpers (Q_phi.c:536-781) on the GPU against
the reference's own functions (compiled from its sources into oracle/_ref),
including what they leave in phi and work.  Each BH step is one Hopping
(summation order differs from the reference's) and one site-diagonal
multiplication, so results agree to about 1e-15 per step; asserted at
1e-13 relative."""
import numpy as np
import pytest

from conftest import rel_err, seeded

pytestmark = pytest.mark.gpu

DIMS = (8, 4, 4, 4)
V = 512
KAPPA, MU = 0.15, 0.01 / 0.3


@pytest.fixture(scope="module")
def env(cb):
    import oracle_bind
    if not oracle_bind.reference_available():
        pytest.skip("reference library not built")
    g = cb.gauge_random(*DIMS, 0.3, 77)
    lat = cb.Lattice(*DIMS, kappa=KAPPA, mu=MU)
    lat.upload_gauge(g)
    ref = oracle_bind.Reference(*DIMS, KAPPA, MU)
    ref.set_gauge(g)
    yield lat, ref
    lat.close()


@pytest.mark.parametrize("name,n", [("BHn", 0), ("BHn", 1), ("BHn", 2), ("BHn", 5), ("BHn", 6),
                                    ("BH", None), ("BH2", None), ("BH3", None), ("BH5", None),
                                    ("BH7", None)])
def test_bh(env, name, n):
    lat, ref = env
    phi0 = seeded(11, 24 * V)
    extra = () if n is None else (n,)
    rxi, rphi = ref.hpe(name, phi0, *extra)
    xi = np.zeros(24 * V)
    phi = phi0.copy()
    getattr(lat, name)(xi, phi, *extra)
    assert rel_err(xi, rxi) < 1e-13
    assert rel_err(phi, rphi) < 1e-13


def test_gamma5_BdagH4_gamma5(env):
    lat, ref = env
    phi0 = seeded(12, 24 * V)
    rxi, rphi, rwork = ref.gamma5_BdagH4_gamma5(phi0)
    xi, work = np.zeros(24 * V), np.zeros(24 * V)
    phi = phi0.copy()
    lat.gamma5_BdagH4_gamma5(xi, phi, work)
    assert rel_err(xi, rxi) < 1e-13
    assert rel_err(work, rwork) < 1e-13
    assert np.array_equal(phi, phi0) and np.array_equal(rphi, phi0)


def test_bhn_negative(env, cb):
    lat, _ = env
    with pytest.raises(cb.CvcbError):
        lat.BHn(np.zeros(24 * V), np.zeros(24 * V), -1)
