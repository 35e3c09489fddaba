"""Algebraic known answers of the oracle's operators on random gauge fields
(no GPU): gamma5-hermiticity Q(mu)^+ = g5 Q(-mu) g5, Qf5 = g5 Q, and
Q = 1/(2 kappa) + i mu g5 + Hopping / (2 kappa), with antiperiodic time and
twisted spatial boundary phases (Q_phi.c:38-188, 399-528, 789-934,
1092-1242)."""
import numpy as np
import pytest

from conftest import rel_err, seeded

CASES = [((8, 4, 4, 4), 0.15, 0.01 / 0.3, (1.0, 0.0, 0.0, 0.0)),
         ((8, 6, 4, 2), 0.137, -0.05, (1.0, 0.5, 0.0, 0.25))]


@pytest.fixture(scope="module", params=CASES, ids=["apbc-t", "twisted"])
def orc(request, cb, oracle_mod):
    dims, kappa, mu, bc = request.param
    o = oracle_mod.Oracle(*dims, kappa, mu, bc)
    o.set_gauge(cb.gauge_random(*dims, 0.3, 1234))
    return o, kappa, mu


def cdot(a, b):
    """sum conj(a) b over the 24 V reals read as 12 V complex numbers"""
    a = a[0::2] + 1j * a[1::2]
    b = b[0::2] + 1j * b[1::2]
    return np.vdot(a, b)


def test_gamma5_hermiticity(orc):
    o, kappa, mu = orc
    V = o.V
    phi, psi = seeded(21, 24 * V), seeded(22, 24 * V)
    lhs = cdot(phi, o.Q_phi(psi, mu))
    rhs = cdot(o.Qf5(o.g5_phi(phi), -mu), psi)   # g5 Q(-mu) g5 phi
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_qf5_is_g5_q(orc):
    o, kappa, mu = orc
    phi = seeded(23, 24 * o.V)
    assert rel_err(o.Qf5(phi, mu), o.g5_phi(o.Q_phi(phi, mu))) <= 1e-15


def test_q_is_diagonal_plus_hopping(orc):
    """Q phi = (1/(2 kappa) + i mu g5) phi + Hopping(phi) / (2 kappa), since
    Hopping = -kappa * (hop sum) and Q = diag - 1/2 (hop sum)."""
    o, kappa, mu = orc
    phi = seeded(24, 24 * o.V)
    g5p = o.g5_phi(phi)
    diag = phi / (2 * kappa)
    diag[0::2] -= mu * g5p[1::2]   # i mu (re + i im) = -mu im + i mu re
    diag[1::2] += mu * g5p[0::2]
    want = diag + o.Hopping(phi) / (2 * kappa)
    assert rel_err(o.Q_phi_tbc(phi), want) <= 1e-14
