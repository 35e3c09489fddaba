"""Analytic free-field (unit links) results for the twisted-mass Wilson
operator with the boundary phase on every link, used as known-answer tests.

With U = 1 and co_phase_up[mu] = exp(i phi_mu), a plane wave
e^{i k.x} u (k_mu = 2 pi n_mu / L_mu) is an eigenfunction of Q_phi_tbc
(Q_phi.c:38-188):

    Q(k) u = [1/(2 kappa) - sum_mu cos q_mu] u + i sum_mu sin q_mu gamma_mu u
             + i mu gamma_5 u,                       q_mu = k_mu + phi_mu,

from -1/2 [(1 - gamma_mu) e^{i q_mu} + (1 + gamma_mu) e^{-i q_mu}]
= -cos q_mu + i gamma_mu sin q_mu.  The propagator of a point source at y0
with spin-colour column sc is (1/V) sum_k e^{i k.(y - y0)} Q(k)^-1 e_sc.

Gamma matrices come from the reference's permutation/sign tables
(cvc_utils.c:707-1520), applied as _fv_eq_gamma_ti_fv (cvc_linalg.h:1344)
does, so the test shares no code with the operators it checks.
"""
import numpy as np


def unit_gauge(V):
    g = np.zeros((V, 4, 9, 2))
    g[:, :, [0, 4, 8], 0] = 1.0
    return g.reshape(-1)


def gamma12(perm, sign, g):
    """gamma_g as a complex 12x12 matrix (component 3 spin + colour)."""
    m24 = np.zeros((24, 24))
    m24[np.arange(24), perm[g]] = sign[g]
    # column b of the complex matrix: the image of the real unit vector e_2b
    return m24[0::2, 0::2] + 1j * m24[1::2, 0::2]


def momentum_matrices(dims, phases, kappa, mu, perm, sign):
    """Q(k) for every lattice momentum, shape (T, LX, LY, LZ, 12, 12),
    momenta in FFT order (n_mu = 0 .. L_mu - 1)."""
    gam = [gamma12(perm, sign, g) for g in (0, 1, 2, 3, 5)]
    ph = np.angle(np.asarray(phases))
    q = np.meshgrid(*[2 * np.pi * np.arange(L) / L + ph[m] for m, L in enumerate(dims)],
                    indexing="ij")
    a = 0.5 / kappa - sum(np.cos(qm) for qm in q)
    out = a[..., None, None] * np.eye(12)
    for m in range(4):
        out = out + 1j * np.sin(q[m])[..., None, None] * gam[m]
    return out + 1j * mu * gam[4]


def coords(dims):
    """Site coordinates (t, x, y, z) in the reference's lexicographic order."""
    return np.stack(np.meshgrid(*[np.arange(L) for L in dims], indexing="ij"), -1).reshape(-1, 4)


def to_reals(c):
    """(V, 12) complex field to the reference's 24 V doubles."""
    r = np.empty(c.shape + (2,))
    r[..., 0], r[..., 1] = c.real, c.imag
    return r.reshape(-1)


def to_complex(f):
    f = np.asarray(f).reshape(-1, 12, 2)
    return f[..., 0] + 1j * f[..., 1]


def plane_wave(dims, n, u):
    """e^{i k.x} u with k_mu = 2 pi n_mu / L_mu, as (V, 12) complex."""
    k = 2 * np.pi * np.asarray(n) / np.asarray(dims)
    return np.exp(1j * coords(dims) @ k)[:, None] * np.asarray(u)[None, :]


def apply_free(dims, n, u, phases, kappa, mu, perm, sign):
    """Q_phi_tbc of the plane wave (n, u), analytically."""
    qk = momentum_matrices(dims, phases, kappa, mu, perm, sign)[tuple(np.asarray(n) % dims)]
    return plane_wave(dims, n, qk @ np.asarray(u))


def free_propagator(dims, y0, sc, phases, kappa, mu, perm, sign):
    """Solution of Q x = point source (site y0 = (t, x, y, z), column sc), (V, 12) complex."""
    qk = momentum_matrices(dims, phases, kappa, mu, perm, sign)
    e = np.zeros(12, complex)
    e[sc] = 1.0
    xk = np.linalg.solve(qk, np.broadcast_to(e[:, None], qk.shape[:-1] + (1,)))[..., 0]
    x = np.fft.ifftn(xk, axes=(0, 1, 2, 3))                          # (1/V) sum_k e^{ik.m} X_k
    x = np.roll(x, shift=tuple(y0), axis=(0, 1, 2, 3))               # m = y - y0
    return x.reshape(-1, 12)
