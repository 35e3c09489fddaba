"""Operators and reductions on the GPU against the oracle (Q_phi.c,
invert_Qtm.c:28-84).  FP64 throughout; the CUDA kernels sum in a different
order (and use FMA), so agreement is to a few units of double rounding:
tolerance 1e-14 relative to the largest component."""
import numpy as np
import pytest

from conftest import rel_err, seeded

pytestmark = pytest.mark.gpu

TOL = 1e-14
CASES = [
    ((8, 4, 4, 4), 0.15, 0.01 / 0.3, (1.0, 0.0, 0.0, 0.0)),
    ((16, 8, 8, 8), 0.15, 0.01 / 0.3, (1.0, 0.0, 0.0, 0.0)),
    ((8, 6, 4, 2), 0.137, -0.05, (1.0, 0.5, 0.0, 0.25)),
]


@pytest.fixture(scope="module", params=CASES, ids=["4^3x8", "8^3x16", "8x6x4x2-bc"])
def setup(request, cb, oracle_mod):
    dims, kappa, mu, bc = request.param
    lat = cb.Lattice(*dims, kappa=kappa, mu=mu, bc_angle=bc)
    g = cb.gauge_random(*dims, 0.3, 1234)
    lat.upload_gauge(g)
    orc = oracle_mod.Oracle(*dims, kappa, mu, bc)
    orc.set_gauge(g)
    V = lat.VOLUME
    phi = seeded(11, 24 * V)
    yield lat, orc, phi, V, kappa, mu
    lat.close()


def test_Q_phi_tbc(setup):
    lat, orc, phi, V, *_ = setup
    xi = np.zeros_like(phi)
    lat.Q_phi_tbc(xi, phi)
    assert rel_err(xi, orc.Q_phi_tbc(phi)) < TOL


def test_Hopping(setup):
    lat, orc, phi, V, *_ = setup
    xi = np.zeros_like(phi)
    lat.Hopping(xi, phi)
    assert rel_err(xi, orc.Hopping(phi)) < TOL


@pytest.mark.parametrize("sgn", [1.0, -1.0])
def test_Qf5(setup, sgn):
    lat, orc, phi, V, kappa, mu = setup
    xi = np.zeros_like(phi)
    lat.Qf5(xi, phi, sgn * mu)
    assert rel_err(xi, orc.Qf5(phi, sgn * mu)) < TOL


def test_Q_phi_explicit_mu(setup):
    lat, orc, phi, *_ = setup
    xi = np.zeros_like(phi)
    lat.Q_phi(xi, phi, 0.0731)
    assert rel_err(xi, orc.Q_phi(phi, 0.0731)) < TOL


def test_g5_and_imu(setup):
    lat, orc, phi, V, *_ = setup
    a = phi.copy()
    lat.g5_phi(a)
    assert np.array_equal(a, orc.g5_phi(phi))
    for sign, nv in [(1.0, V), (-1.0, V), (1.0, V // 2 + 3)]:
        b = phi.copy()
        lat.mul_one_pm_imu_inv(b, sign, nv)
        assert rel_err(b, orc.mul_one_pm_imu_inv(phi, sign, nv)) < TOL


def test_scalar_products(setup):
    lat, orc, phi, V, *_ = setup
    psi = seeded(12, 24 * V)
    for nv in (V, V // 3, 1):
        w = lat.spinor_scalar_product_co(phi, psi, nv)
        ref = orc.scalar_product_co(phi, psi, nv)
        assert abs(w - ref) <= 1e-13 * max(abs(ref), 1.0)
        r = lat.spinor_scalar_product_re(phi, psi, nv)
        assert abs(r - ref.real) <= 1e-13 * max(abs(ref), 1.0)
    # deterministic: identical bits on repeated calls
    w1 = lat.spinor_scalar_product_co(phi, psi, V)
    w2 = lat.spinor_scalar_product_co(phi, psi, V)
    assert w1 == w2


def test_gamma5_hermiticity(setup):
    """Q(mu)^dagger = g5 Q(-mu) g5: <a, Q(mu) b> = <g5 Q(-mu) g5 a, b>."""
    lat, orc, phi, V, kappa, mu = setup
    psi = seeded(13, 24 * V)
    qb = np.zeros_like(phi)
    lat.Q_phi(qb, psi, mu)
    lhs = lat.spinor_scalar_product_co(phi, qb, V)
    t = phi.copy()
    lat.g5_phi(t)
    u = np.zeros_like(phi)
    lat.Qf5(u, t, -mu)  # g5 Q(-mu) g5 phi
    rhs = lat.spinor_scalar_product_co(u, psi, V)
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_device_pointers(setup):
    """The same entry points accept CUDA device memory (torch tensors)."""
    torch = pytest.importorskip("torch")
    lat, orc, phi, V, *_ = setup
    d_phi = torch.from_numpy(phi).cuda()
    d_xi = torch.zeros_like(d_phi)
    lat.Q_phi_tbc(d_xi, d_phi)
    torch.cuda.synchronize()
    assert rel_err(d_xi.cpu().numpy(), orc.Q_phi_tbc(phi)) < TOL
    w = lat.spinor_scalar_product_co(d_phi, d_xi, V)
    ref = orc.scalar_product_co(phi, d_xi.cpu().numpy(), V)
    assert abs(w - ref) <= 1e-13 * abs(ref)


def test_plaquette(setup):
    lat, orc, *_ = setup
    pl, ls = lat.plaquette()
    opl, ols = orc.plaquette()
    assert abs(pl - opl) < 1e-14
    assert abs(ls - ols) < 1e-12 * abs(ols)


def test_errors(cb):
    lat = cb.Lattice(4, 4, 4, 4)
    phi = np.zeros(24 * lat.VOLUME)
    with pytest.raises(cb.CvcbError) as e:
        lat.Q_phi_tbc(phi.copy(), phi)  # no gauge field yet
    assert e.value.code == -5
    with pytest.raises(cb.CvcbError):
        cb.Lattice(3, 4, 4, 4)  # odd extent
    lat.close()
