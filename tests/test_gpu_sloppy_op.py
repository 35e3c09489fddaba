"""The inner operator of the batched solver, M^+ M on the odd sites
(cvcb_sloppy_normal_op), in every storage the solver uses, against the
oracle's FP64 operator.

M is the odd-site Schur complement of the operator of Q_phi_tbc
(Q_phi.c:38-188): for x on odd sites, M x = A x - 1/4 H_oe A^-1 H_eo x with
A = 1/(2 kappa) + i mu g5.  The oracle builds it from its own Q_phi_tbc:
y = Q x (x odd only) has y_e = -1/2 H_eo x; z = A^-1 y_e; w = Q z (z even
only) has w_o = -1/2 H_oe z, so M x = A x - w_o; and M^+ = g5 M(-mu) g5.
Tolerances, relative to the largest component: FP64 storage 1e-13, FP32
(per-rhs and pair-tiled layouts, 12- and 18-real links) 1e-5, FP16+norm
3e-3; the two FP32 layouts agree with each other to 2e-6.  An odd number of
right-hand sides leaves the last pair of the pair-tiled layout half used."""
import numpy as np
import pytest

from conftest import rel_err, seeded

pytestmark = pytest.mark.gpu

DIMS = (16, 8, 8, 8)
KAPPA, MU = 0.155, 0.005 / 0.31
N = 5


def odd_mask(dims):
    T, LX, LY, LZ = dims
    t, x, y, z = np.meshgrid(*[np.arange(n) for n in dims], indexing="ij")
    return ((t + x + y + z) % 2 == 1).reshape(-1)


def g5(f):
    g = f.reshape(-1, 4, 6).copy()
    g[:, 2:, :] *= -1
    return g.reshape(-1)


def diag(f, a, b):
    """(a + i b g5) f on CVC-layout fields (24 doubles per site)."""
    c = f.reshape(-1, 4, 3, 2)
    z = c[..., 0] + 1j * c[..., 1]
    s = np.array([1, 1, -1, -1])[None, :, None]
    o = a * z + 1j * b * s * z
    return np.stack([o.real, o.imag], axis=-1).reshape(-1)


def schur(orc, x, mu, odd):
    """M(mu) x on odd sites with the oracle's Q_phi_tbc."""
    orc.set_params(KAPPA, mu)
    ka = 0.5 / KAPPA
    xo = x * np.repeat(odd, 24)
    y = orc.Q_phi_tbc(xo) * np.repeat(~odd, 24)
    d = ka * ka + mu * mu
    z = diag(y, ka / d, -mu / d)
    w = orc.Q_phi_tbc(z) * np.repeat(odd, 24)
    return (diag(xo, ka, mu) - w) * np.repeat(odd, 24)


@pytest.fixture(scope="module")
def env(cb, oracle_mod):
    g = cb.gauge_random(*DIMS, 0.25, 11)
    lat = cb.Lattice(*DIMS, kappa=KAPPA, mu=MU)
    lat.upload_gauge(g)
    orc = oracle_mod.Oracle(*DIMS, KAPPA, MU)
    orc.set_gauge(g)
    V = lat.VOLUME
    odd = odd_mask(DIMS)
    ins = [seeded(500 + i, 24 * V) for i in range(N)]
    want = []
    for x in ins:
        mx = schur(orc, x, MU, odd)
        want.append(g5(schur(orc, g5(mx), -MU, odd)))
    orc.set_params(KAPPA, MU)
    yield lat, ins, want
    lat.close()


@pytest.mark.parametrize("prec,recon,layout,tol", [
    (0, 18, 0, 1e-13), (1, 12, 0, 1e-5), (1, 18, 0, 1e-5), (1, 12, 1, 1e-5), (1, 18, 1, 1e-5),
    (2, 12, 0, 3e-3)], ids=["fp64", "fp32-12", "fp32-18", "pairs-12", "pairs-18", "fp16-12"])
def test_inner_operator_against_oracle(env, prec, recon, layout, tol):
    lat, ins, want = env
    outs = [np.zeros_like(x) for x in ins]
    lat.sloppy_normal_op(ins, outs, prec, recon, layout)
    for o, w in zip(outs, want):
        assert rel_err(o, w) < tol


@pytest.mark.parametrize("recon", [12, 18])
def test_pair_layout_matches_per_rhs_layout(env, recon):
    lat, ins, _ = env
    a = [np.zeros_like(x) for x in ins]
    b = [np.zeros_like(x) for x in ins]
    lat.sloppy_normal_op(ins, a, 1, recon, 0)
    lat.sloppy_normal_op(ins, b, 1, recon, 1)
    for u, v in zip(a, b):
        assert rel_err(v, u) < 2e-6


# A lattice whose half volume (432 sites) is not a whole number of 32-site
# tiles: the last tile of every pair-tiled field is partly filled, and the
# tuner's block shapes end inside it.
DIMS_PARTIAL = (4, 6, 6, 6)


@pytest.mark.parametrize("prec,recon,layout,tol", [
    (1, 12, 0, 1e-5), (1, 12, 1, 1e-5), (1, 18, 1, 1e-5)], ids=["fp32-12", "pairs-12", "pairs-18"])
def test_inner_operator_partial_tile(cb, oracle_mod, prec, recon, layout, tol):
    g = cb.gauge_random(*DIMS_PARTIAL, 0.25, 5)
    lat = cb.Lattice(*DIMS_PARTIAL, kappa=KAPPA, mu=MU)
    lat.upload_gauge(g)
    orc = oracle_mod.Oracle(*DIMS_PARTIAL, KAPPA, MU)
    orc.set_gauge(g)
    V = lat.VOLUME
    assert (V // 2) % 32 != 0
    odd = odd_mask(DIMS_PARTIAL)
    ins = [seeded(700 + i, 24 * V) for i in range(3)]
    outs = [np.zeros_like(x) for x in ins]
    lat.sloppy_normal_op(ins, outs, prec, recon, layout)
    for x, o in zip(ins, outs):
        mx = schur(orc, x, MU, odd)
        orc.set_params(KAPPA, MU)
        w = g5(schur(orc, g5(mx), -MU, odd))
        orc.set_params(KAPPA, MU)
        assert rel_err(o, w) < tol
    lat.close()


def test_batched_solve_partial_tile(cb):
    """The batched FP32 solve on pair-tiled fields (default layout and the
    tuner's shapes, the tensor-memory candidate among them) on the
    partial-tile lattice: 5 point sources reach |b - Q x| / |b| <= 1e-10."""
    lat = cb.Lattice(*DIMS_PARTIAL, kappa=KAPPA, mu=MU)
    lat.upload_gauge(cb.gauge_random(*DIMS_PARTIAL, 0.25, 5))
    V = lat.VOLUME
    bs = []
    for i in range(5):
        b = np.zeros(24 * V)
        b[24 * (53 * i + 7) + 2 * (i % 12)] = 1.0
        bs.append(b)
    xs = [np.zeros(24 * V) for _ in bs]
    p = cb.solver_defaults()
    st = lat.solve(xs, bs, p)
    assert st.converged == 5
    for x, b in zip(xs, bs):
        r = np.zeros(24 * V)
        lat.Q_phi_tbc(r, x)
        assert np.linalg.norm(r - b) / np.linalg.norm(b) <= 1e-10
    lat.close()
