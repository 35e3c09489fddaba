"""Momentum-space Pi_mu_nu(q) (cvcb_pi_momentum): against a numpy FFT with
the same phase convention on random fields (1e-13), and the Ward identity
in momentum space -- sum_mu 2 sin(q_mu/2) Pi_mu_nu(q) = 0 at every q --
on Pi from GPU-solved propagators (to 1e-9 of max |Pi|, the x-space WI
tolerance)."""
import numpy as np
import pytest

from conftest import rel_err, seeded

pytestmark = pytest.mark.gpu

DIMS = (8, 4, 4, 6)
V = 8 * 4 * 4 * 6
KAPPA, MU = 0.15, 0.01 / 0.3


def qgrid():
    return np.meshgrid(*[2 * np.pi * np.arange(L) / L for L in DIMS], indexing="ij")


def numpy_pi_momentum(conn, src, contact):
    z = (conn[0::2] + 1j * conn[1::2]).reshape(*DIMS, 4, 4)
    F = np.fft.fftn(z, axes=(0, 1, 2, 3))
    q = qgrid()
    t, r = divmod(src, DIMS[1] * DIMS[2] * DIMS[3])
    x, r = divmod(r, DIMS[2] * DIMS[3])
    y, zz = divmod(r, DIMS[3])
    qy = q[0] * t + q[1] * x + q[2] * y + q[3] * zz
    for mu in range(4):
        for nu in range(4):
            F[..., mu, nu] *= np.exp(1j * (qy - 0.5 * q[mu] + 0.5 * q[nu]))
    if contact is not None:
        for nu in range(4):
            F[..., nu, nu] -= contact[2 * nu] + 1j * contact[2 * nu + 1]
    out = np.zeros(32 * V)
    out[0::2] = F.real.ravel()
    out[1::2] = F.imag.ravel()
    return out


@pytest.fixture(scope="module")
def lat(cb):
    lt = cb.Lattice(*DIMS, kappa=KAPPA, mu=MU)
    lt.upload_gauge(cb.gauge_random(*DIMS, 0.3, 5))
    yield lt
    lt.close()


@pytest.mark.parametrize("src,with_contact", [(0, True), (123, True), (77, False)])
def test_against_numpy(lat, src, with_contact):
    conn = seeded(src + 1, 32 * V)
    contact = seeded(500 + src, 8) if with_contact else None
    got = lat.pi_momentum(conn, src, contact)
    assert rel_err(got, numpy_pi_momentum(conn, src, contact)) < 1e-13


def test_device_pointers(lat):
    torch = pytest.importorskip("torch")
    conn = seeded(3, 32 * V)
    out = torch.zeros(32 * V, dtype=torch.float64, device="cuda")
    lat.pi_momentum(torch.from_numpy(conn).cuda(), 5, None, out)
    assert rel_err(out.cpu().numpy(), numpy_pi_momentum(conn, 5, None)) < 1e-13


def test_ward_identity_in_momentum_space(lat, cb):
    src = 123
    p = cb.solver_defaults()
    p.tol = 1e-13
    conn, contact = lat.pi_forward(src, p)
    pm = lat.pi_momentum(conn, src, contact)
    z = (pm[0::2] + 1j * pm[1::2]).reshape(*DIMS, 4, 4)
    q = qgrid()
    qhat = [2 * np.sin(qq / 2) for qq in q]
    scale = np.max(np.abs(z))
    for nu in range(4):
        div = sum(qhat[mu] * z[..., mu, nu] for mu in range(4))
        assert np.max(np.abs(div)) < 1e-9 * scale, nu
    # without the subtraction the divergence is qhat_nu * contact_nu
    pm0 = lat.pi_momentum(conn, src, None)
    z0 = (pm0[0::2] + 1j * pm0[1::2]).reshape(*DIMS, 4, 4)
    for nu in range(4):
        div = sum(qhat[mu] * z0[..., mu, nu] for mu in range(4))
        ct = contact[2 * nu] + 1j * contact[2 * nu + 1]
        assert np.max(np.abs(div - qhat[nu] * ct)) < 1e-9 * scale
