"""Free-field known-answer tests on the GPU (unit links): the FP64 operator
on plane waves and the batched mixed-precision solver on point sources,
against the analytic momentum-space results of free_field.py (no oracle
involved), with antiperiodic time and twisted spatial boundary phases."""
import numpy as np
import pytest

import free_field as ff

pytestmark = pytest.mark.gpu

DIMS = (8, 4, 4, 4)
KAPPA, MU = 0.15, 0.01 / 0.3
BCS = [(1.0, 0.0, 0.0, 0.0), (1.0, 0.5, 0.0, 0.25)]


@pytest.fixture(scope="module", params=BCS, ids=["apbc-t", "twisted"])
def setup(request, cb):
    bc = request.param
    lat = cb.Lattice(*DIMS, kappa=KAPPA, mu=MU, bc_angle=bc)
    lat.upload_gauge(ff.unit_gauge(lat.VOLUME))
    perm, sign = cb.gamma_tables()
    yield lat, cb.boundary_phases(*DIMS, bc), perm, sign
    lat.close()


@pytest.mark.parametrize("n", [(0, 0, 0, 0), (1, 2, 0, 3), (7, 1, 3, 2)])
def test_plane_waves(setup, n):
    lat, ph, perm, sign = setup
    rng = np.random.default_rng(sum(n))
    u = rng.standard_normal(12) + 1j * rng.standard_normal(12)
    xi = np.zeros(24 * lat.VOLUME)
    lat.Q_phi_tbc(xi, ff.to_reals(ff.plane_wave(DIMS, n, u)))
    want = ff.apply_free(DIMS, n, u, ph, KAPPA, MU, perm, sign)
    assert np.max(np.abs(ff.to_complex(xi) - want)) <= 1e-13 * np.max(np.abs(want))


@pytest.mark.parametrize("prec", ["single", "half"])
def test_batched_solver_point_sources(setup, cb, prec):
    """Twelve spin-colour columns of one point source at the default true
    residual 1e-10.  |x - x_exact|_2 <= |r|_2 / sigma_min(Q) <= 1.4e-10 here
    (sigma_min 0.70-0.76, sigma_max 7.2-7.3 over the momenta), against
    max |x| of about 0.25."""
    lat, ph, perm, sign = setup
    T, LX, LY, LZ = DIMS
    y0 = (3, 1, 2, 3)
    ix = ((y0[0] * LX + y0[1]) * LY + y0[2]) * LZ + y0[3]
    bs = []
    for sc in range(12):
        b = np.zeros(24 * lat.VOLUME)
        b[24 * ix + 2 * sc] = 1.0
        bs.append(b)
    xs = [np.zeros_like(b) for b in bs]
    p = cb.solver_defaults()
    p.precision = {"single": cb.PREC_SINGLE, "half": cb.PREC_HALF}[prec]
    st = lat.solve(xs, bs, p)
    assert st.converged == 12 and st.max_true_res <= 1e-10
    for sc in (0, 5, 11):
        want = ff.free_propagator(DIMS, y0, sc, ph, KAPPA, MU, perm, sign)
        got = ff.to_complex(xs[sc])
        assert np.max(np.abs(got - want)) <= 2e-9 * np.max(np.abs(want)), sc
