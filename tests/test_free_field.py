"""Free-field known-answer tests of the oracle (unit links): plane waves
through Q_phi_tbc and point-source propagators from invert_Qtm_her against
the analytic momentum-space results of free_field.py, with antiperiodic
time and twisted spatial boundary phases."""
import numpy as np
import pytest

import free_field as ff

DIMS = (8, 4, 4, 4)
KAPPA, MU = 0.15, 0.01 / 0.3
BCS = [(1.0, 0.0, 0.0, 0.0), (1.0, 0.5, 0.0, 0.25)]


@pytest.fixture(scope="module", params=BCS, ids=["apbc-t", "twisted"])
def setup(request, cb, oracle_mod):
    bc = request.param
    V = int(np.prod(DIMS))
    orc = oracle_mod.Oracle(*DIMS, KAPPA, MU, bc)
    orc.set_gauge(ff.unit_gauge(V))
    perm, sign = cb.gamma_tables()
    return orc, cb.boundary_phases(*DIMS, bc), perm, sign


@pytest.mark.parametrize("n", [(0, 0, 0, 0), (1, 2, 0, 3), (7, 1, 3, 2), (4, 2, 2, 2)])
def test_plane_waves(setup, n):
    orc, ph, perm, sign = setup
    rng = np.random.default_rng(sum(n))
    u = rng.standard_normal(12) + 1j * rng.standard_normal(12)
    got = ff.to_complex(orc.Q_phi_tbc(ff.to_reals(ff.plane_wave(DIMS, n, u))))
    want = ff.apply_free(DIMS, n, u, ph, KAPPA, MU, perm, sign)
    assert np.max(np.abs(got - want)) <= 1e-13 * np.max(np.abs(want))


@pytest.mark.parametrize("y0,sc", [((0, 0, 0, 0), 0), ((3, 1, 2, 3), 7)])
def test_point_source_propagator(setup, y0, sc):
    orc, ph, perm, sign = setup
    T, LX, LY, LZ = DIMS
    b = np.zeros(24 * int(np.prod(DIMS)))
    ix = ((y0[0] * LX + y0[1]) * LY + y0[2]) * LZ + y0[3]
    b[24 * ix + 2 * sc] = 1.0
    rc, x, _ = orc.invert(b, 1e-26, 2000)   # squared relative residual (invert_Qtm.c:276-478)
    assert rc > 0
    want = ff.free_propagator(DIMS, y0, sc, ph, KAPPA, MU, perm, sign)
    got = ff.to_complex(x)
    assert np.max(np.abs(got - want)) <= 1e-10 * np.max(np.abs(want))
