"""Derivatives of Pi_mu_nu (forward/tangent/backward in the C ABI) against
central finite differences in FP64 (h = 1e-5), for
L = sum_x Re Pi_00(x) cos(2 pi x_3 / L_3).

Tolerances: the solves stop at a true residual of 1e-13, so finite
differences carry an error of about 1e-13/h = 1e-8 relative on top of the
O(h^2) truncation; derivatives are compared at 1e-6 relative."""
import numpy as np
import pytest

from conftest import seeded

pytestmark = pytest.mark.gpu

DIMS = (8, 4, 4, 4)
V = 512
KAPPA, MU = 0.150, 0.01 / 0.3
SRC = 37
H = 1e-5


def weights():
    w = np.zeros(32 * V)
    T, LX, LY, LZ = DIMS
    for lex in range(V):
        z = lex % LZ
        w[32 * lex] = np.cos(2 * np.pi * z / LZ)  # Re of (mu, nu) = (0, 0)
    return w


def L_of(conn, w):
    return float(np.dot(conn, w))


@pytest.fixture(scope="module")
def setup(cb):
    lat = cb.Lattice(*DIMS, kappa=KAPPA, mu=MU)
    g = cb.gauge_random(*DIMS, 0.3, 3)
    lat.upload_gauge(g)
    p = cb.solver_defaults()
    p.precision, p.link_recon, p.tol = cb.PREC_DOUBLE, 18, 1e-13
    yield lat, g, p
    lat.close()


def forward(lat, g, p, kappa=KAPPA, mu=MU):
    lat.set_params(kappa, mu)
    lat.upload_gauge(g)
    conn, _ = lat.pi_forward(SRC, p)
    return conn


def test_tangent_and_backward_mu_kappa(setup):
    lat, g, p = setup
    w = weights()
    conn = forward(lat, g, p)
    dpi_mu = lat.pi_tangent("mu")
    dpi_ka = lat.pi_tangent("kappa")
    dmu, dka, _ = lat.pi_backward(w, want_gauge=False)
    # central differences of the whole field
    fd_mu = (forward(lat, g, p, mu=MU + H) - forward(lat, g, p, mu=MU - H)) / (2 * H)
    fd_ka = (forward(lat, g, p, kappa=KAPPA + H) - forward(lat, g, p, kappa=KAPPA - H)) / (2 * H)
    forward(lat, g, p)
    for t, fd in ((dpi_mu, fd_mu), (dpi_ka, fd_ka)):
        assert np.linalg.norm(t - fd) <= 1e-6 * np.linalg.norm(fd)
    # reverse mode agrees with the tangent contracted with the weights
    assert abs(dmu - L_of(dpi_mu, w)) <= 1e-8 * abs(L_of(dpi_mu, w))
    assert abs(dka - L_of(dpi_ka, w)) <= 1e-8 * abs(L_of(dpi_ka, w))
    assert abs(dmu - L_of(fd_mu, w)) <= 1e-6 * abs(dmu)


def test_gauge_gradient_directional(setup):
    lat, g, p = setup
    w = weights()
    forward(lat, g, p)
    _, _, gu = lat.pi_backward(w)
    for seed in (5, 6):
        D = seeded(seed, 72 * V)
        fd = (L_of(forward(lat, g + H * D, p), w) - L_of(forward(lat, g - H * D, p), w)) / (2 * H)
        an = float(np.dot(gu, D))
        assert abs(an - fd) <= 1e-6 * max(abs(fd), 1e-12), (an, fd)
    forward(lat, g, p)


def test_gauge_gradient_source_link_only(setup):
    """A direction that touches only the source links isolates the
    source-vertex part of the gradient."""
    lat, g, p = setup
    w = weights()
    forward(lat, g, p)
    _, _, gu = lat.pi_backward(w)
    D = np.zeros(72 * V)
    D[72 * SRC:72 * SRC + 72] = seeded(8, 72)
    fd = (L_of(forward(lat, g + H * D, p), w) - L_of(forward(lat, g - H * D, p), w)) / (2 * H)
    assert abs(float(np.dot(gu, D)) - fd) <= 1e-6 * abs(fd)
    forward(lat, g, p)


def test_autograd_wrapper_and_recompute(setup, cb):
    torch = pytest.importorskip("torch")
    from autograd_pi import PiFunction
    lat, g, p = setup
    w = torch.from_numpy(weights())
    mu = torch.tensor(MU, dtype=torch.float64, requires_grad=True)
    ka = torch.tensor(KAPPA, dtype=torch.float64, requires_grad=True)
    gt = torch.from_numpy(g.copy()).requires_grad_(True)
    pi = PiFunction.apply(mu, ka, gt, lat, SRC, p)
    (pi * w).sum().backward()
    lat.set_params(KAPPA, MU)
    lat.upload_gauge(g)
    # columns recomputed (memory budget 0) give the same gradients
    lat.pi_forward(SRC, p, keep_bytes=0)
    dmu, dka, gu = lat.pi_backward(w.numpy())
    assert abs(mu.grad.item() - dmu) <= 1e-9 * abs(dmu)
    assert abs(ka.grad.item() - dka) <= 1e-9 * abs(dka)
    assert np.allclose(gt.grad.numpy(), gu, rtol=1e-8, atol=1e-12 * np.max(np.abs(gu)))


def test_tangent_mu_vs_reference_rerun(setup, oracle_mod):
    """dPi/dmu against the reference rerun at mu +- h: the 120 columns are
    solved by the reference's own invert_Qtm_her (compiled from its sources)
    at shifted mu, contracted by the oracle contraction (bit-exact with the
    reference's), and differenced."""
    import oracle_bind
    if not oracle_bind.reference_available():
        pytest.skip("reference library not built")
    lat, g, p = setup
    T, LX, LY, LZ = DIMS
    t, r = divmod(SRC, LX * LY * LZ)
    x, r = divmod(r, LY * LZ)
    y, z = divmod(r, LZ)
    c = [t, x, y, z]
    L = [T, LX, LY, LZ]
    shifted = []
    for m in range(4):
        cc = list(c)
        cc[m] = (cc[m] + 1) % L[m]
        shifted.append(((cc[0] * LX + cc[1]) * LY + cc[2]) * LZ + cc[3])
    shifted.append(SRC)
    bs = []
    for s in shifted:
        for sc in range(12):
            b = np.zeros(24 * V)
            b[24 * s + 2 * sc] = 1.0
            bs.append(b)
    ref = oracle_bind.Reference(*DIMS, KAPPA, MU)
    ref.set_gauge(g)
    orc = oracle_mod.Oracle(*DIMS, KAPPA, MU)
    orc.set_gauge(g)

    def ref_pi(mu):
        cols = []
        for sgn in (+1, -1):
            ref.set_params(KAPPA, sgn * mu)
            for b in bs:
                rc, xs = ref.invert(b, 1e-26, 5000, her=True)
                assert rc > 0
                cols.append(xs)
        conn, _ = orc.cvc_contract(cols, SRC)
        return conn

    fd = (ref_pi(MU + H) - ref_pi(MU - H)) / (2 * H)
    forward(lat, g, p)
    d = lat.pi_tangent("mu")
    assert np.linalg.norm(d - fd) / np.linalg.norm(fd) < 1e-6


def test_c4_gradients_12c24(cb):
    """The adjoint check at 12^3x24 (gauge eps 0.3 seed 3, kappa 0.150,
    2 kappa mu 0.01, source at the origin): dPi/dmu, dPi/dkappa and dL/dU
    (along a random direction) against central differences, h = 1e-5;
    the relative errors are printed with -s."""
    dims = (24, 12, 12, 12)
    vol = 24 * 12 ** 3
    lat = cb.Lattice(*dims, kappa=KAPPA, mu=MU)
    g = cb.gauge_random(*dims, 0.3, 3)
    p = cb.solver_defaults()
    p.precision, p.link_recon, p.tol = cb.PREC_DOUBLE, 18, 1e-13
    w = np.zeros(32 * vol)
    w[0::32] = np.cos(2 * np.pi * (np.arange(vol) % 12) / 12)

    def fwd(kappa=KAPPA, mu=MU, gg=g):
        lat.set_params(kappa, mu)
        lat.upload_gauge(gg)
        return lat.pi_forward(0, p)[0]

    fwd()
    dmu_t, dka_t = lat.pi_tangent("mu"), lat.pi_tangent("kappa")
    dmu, dka, gu = lat.pi_backward(w)
    fdmu = (fwd(mu=MU + H) - fwd(mu=MU - H)) / (2 * H)
    fdka = (fwd(kappa=KAPPA + H) - fwd(kappa=KAPPA - H)) / (2 * H)
    D = seeded(99, 72 * vol)
    fdu = (np.dot(fwd(gg=g + H * D), w) - np.dot(fwd(gg=g - H * D), w)) / (2 * H)
    errs = {
        "dPi/dmu": np.linalg.norm(dmu_t - fdmu) / np.linalg.norm(fdmu),
        "dPi/dkappa": np.linalg.norm(dka_t - fdka) / np.linalg.norm(fdka),
        "dL/dmu": abs(dmu - np.dot(fdmu, w)) / abs(dmu),
        "dL/dkappa": abs(dka - np.dot(fdka, w)) / abs(dka),
        "dL/dU.D": abs(np.dot(gu, D) - fdu) / abs(fdu),
    }
    print("\nC4 12^3x24 gradient relative errors: " +
          ", ".join(f"{k} {v:.2e}" for k, v in errs.items()))
    lat.close()
    assert max(errs.values()) < 1e-6
