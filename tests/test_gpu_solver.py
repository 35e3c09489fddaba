"""FP64 BiCGStab solvers (invert_Qtm.c:86-478) and the batched mixed-
precision solver against the oracle.

Tolerances: the reference stops on the squared relative residual
(solver_precision = 1e-20 for a true relative residual of 1e-10); two FP64
solutions of the same system that both meet that bound agree to about
cond(Q) * 1e-10, so solutions are compared at 1e-8 relative; the returned
true residual must meet the bound itself."""
import numpy as np
import pytest

from conftest import rel_err, seeded

pytestmark = pytest.mark.gpu

DIMS = (8, 4, 4, 4)
KAPPA, MU = 0.15, 0.01 / 0.3


@pytest.fixture(scope="module")
def env(cb, oracle_mod):
    lat = cb.Lattice(*DIMS, kappa=KAPPA, mu=MU)
    g = cb.gauge_random(*DIMS, 0.3, 1234)
    lat.upload_gauge(g)
    orc = oracle_mod.Oracle(*DIMS, KAPPA, MU)
    orc.set_gauge(g)
    yield lat, orc, g
    lat.close()


def point_source(V, sc, site=0):
    b = np.zeros(24 * V)
    b[24 * site + 2 * sc] = 1.0
    return b


def test_invert_Qtm_her_point_source(env):
    lat, orc, _ = env
    V = lat.VOLUME
    b = point_source(V, 0)
    x = np.zeros(24 * V)
    n, tr2 = lat.invert_Qtm_her(x, b, 1e-20, 1000, return_residual=True)
    rc, xo, tro = orc.invert(b, 1e-20, 1000, her=True)
    assert n > 0 and rc > 0
    assert abs(n - rc) <= max(3, rc // 10)
    assert tr2 < 1e-19
    assert rel_err(x, xo) < 1e-8


def test_invert_Qtm_breaks_down_on_point_source(env):
    """<r2, r1> = 0 at the first step for a point source (the reference's
    plain BiCGStab fails with NaN and returns -3)."""
    lat, orc, _ = env
    V = lat.VOLUME
    b = point_source(V, 3)
    x = np.zeros(24 * V)
    assert lat.invert_Qtm(x, b, 1e-20, 50) == -3
    rc, _, _ = orc.invert(b, 1e-20, 50, her=False)
    assert rc == -3
    # the GPU's reductions sum in another order, so its recursion need not
    # reach a non-finite scalar within 50 iterations: -3 or -4 from the C ABI
    from cvc_b200 import _lib
    from cvc_b200.lattice import ptr
    x[:] = 0
    rc = lat._lib.cvcb_invert_Qtm(lat._h, ptr(x), ptr(b), 1e-20, 50, None)
    assert rc in (_lib.CVCB_NO_CONVERGENCE, _lib.CVCB_BREAKDOWN)


def test_breakdown_status(env):
    """A recursion scalar that is not finite (here from a source with a NaN
    component) ends both FP64 solvers with CVCB_BREAKDOWN from the C ABI;
    the reference-facing Python mirror reports the reference's -3."""
    from cvc_b200 import _lib
    from cvc_b200.lattice import ptr
    lat, _, _ = env
    V = lat.VOLUME
    b = point_source(V, 3)
    b[24 * 5 + 1] = np.nan
    for fn in (lat._lib.cvcb_invert_Qtm, lat._lib.cvcb_invert_Qtm_her):
        x = np.zeros(24 * V)
        assert fn(lat._h, ptr(x), ptr(b), 1e-20, 50, None) == _lib.CVCB_BREAKDOWN
        assert "broke down" in lat._lib.cvcb_last_error().decode()
    x = np.zeros(24 * V)
    assert lat.invert_Qtm(x, b, 1e-20, 50) == -3
    assert lat.invert_Qtm_her(x, b, 1e-20, 50) == -3


def test_invert_Qtm_random_source_subcritical(cb, oracle_mod):
    lat = cb.Lattice(*DIMS, kappa=0.10, mu=0.02)
    g = cb.gauge_random(*DIMS, 0.3, 99)
    lat.upload_gauge(g)
    orc = oracle_mod.Oracle(*DIMS, 0.10, 0.02)
    orc.set_gauge(g)
    b = seeded(5, 24 * lat.VOLUME)
    x = np.zeros_like(b)
    n, tr2 = lat.invert_Qtm(x, b, 1e-24, 1000, return_residual=True)
    rc, xo, _ = orc.invert(b, 1e-24, 1000, her=False)
    assert n > 0 and rc > 0 and abs(n - rc) <= 3
    assert tr2 < 1e-23
    assert rel_err(x, xo) < 1e-9
    lat.close()


def test_start_guess_already_solves(env):
    """invert_Qtm.c:144-147: returns 0 and leaves xi untouched."""
    lat, orc, _ = env
    V = lat.VOLUME
    x = seeded(8, 24 * V)
    b = np.zeros(24 * V)
    lat.Q_phi_tbc(b, x)
    x0 = x.copy()
    assert lat.invert_Qtm(x, b, 1e-10, 100) == 0
    assert np.array_equal(x, x0)


def test_null_field(cb, env):
    lat, _, _ = env
    b = np.zeros(24 * lat.VOLUME)
    assert lat._lib.cvcb_invert_Qtm_her(lat._h, None, b.ctypes.data, 1e-20, 10, None) == -2


@pytest.mark.parametrize("prec,recon", [(0, 18), (1, 12), (1, 18), (2, 12)],
                         ids=["fp64", "fp32-12", "fp32-18", "fp16-12"])
def test_batched_solver(cb, env, prec, recon):
    lat, orc, _ = env
    V = lat.VOLUME
    bs = [point_source(V, sc) for sc in range(12)]
    xs = [np.zeros(24 * V) for _ in range(12)]
    p = cb.solver_defaults()
    p.precision, p.link_recon, p.tol = prec, recon, 1e-10
    st = lat.solve(xs, bs, p)
    assert st.converged == 12
    assert st.max_true_res <= 1e-10
    # true residual recomputed independently by the full FP64 operator
    for sc in (0, 5, 11):
        r = np.zeros(24 * V)
        lat.Q_phi_tbc(r, xs[sc])
        assert np.linalg.norm(r - bs[sc]) / np.linalg.norm(bs[sc]) <= 1e-10
    rc, xo, _ = orc.invert(bs[0], 1e-24, 2000, her=True)
    assert rel_err(xs[0], xo) < 1e-8


def test_batched_solver_device_pointers(cb, env):
    torch = pytest.importorskip("torch")
    lat, _, _ = env
    V = lat.VOLUME
    bs = [torch.from_numpy(seeded(20 + i, 24 * V)).cuda() for i in range(5)]
    xs = [torch.zeros(24 * V, dtype=torch.float64, device="cuda") for _ in range(5)]
    st = lat.solve(xs, bs)
    torch.cuda.synchronize()
    assert st.converged == 5 and st.max_true_res <= 1e-10
    r = np.zeros(24 * V)
    lat.Q_phi_tbc(r, xs[2].cpu().numpy())
    b2 = bs[2].cpu().numpy()
    assert np.linalg.norm(r - b2) / np.linalg.norm(b2) <= 1e-10


def test_batched_solver_zero_rhs(cb, env):
    lat, _, _ = env
    V = lat.VOLUME
    bs = [np.zeros(24 * V), point_source(V, 1)]
    xs = [np.ones(24 * V), np.zeros(24 * V)]
    st = lat.solve(xs, bs)
    assert st.converged == 2
    assert not np.any(xs[0])


@pytest.mark.parametrize("prec", [1, 2], ids=["fp32", "fp16"])
def test_batched_solver_tiny_magnitudes(cb, prec):
    """A source scaled by 1e-33: far from it the propagator and the residuals
    fall below the smallest normal float.  The FP16 store (one float scale
    per site) must write such sites as zero rather than overflow 1/scale;
    the solution is the unscaled one times 1e-33 (the solver is linear)."""
    dims = (16, 8, 8, 8)
    V = 16 * 8 ** 3
    lat = cb.Lattice(*dims, kappa=0.155, mu=0.005 / 0.31)
    lat.upload_gauge(cb.gauge_random(*dims, 0.25, 11))
    p = cb.solver_defaults()
    p.precision = prec
    b1 = [point_source(V, sc) for sc in (0, 7)]
    bt = [1e-33 * b for b in b1]
    x1 = [np.zeros(24 * V) for _ in b1]
    xt = [np.zeros(24 * V) for _ in bt]
    st1 = lat.solve(x1, b1, p)
    stt = lat.solve(xt, bt, p)
    assert st1.converged == 2 and stt.converged == 2
    assert stt.max_true_res <= 1e-10
    for a, b in zip(x1, xt):
        assert np.all(np.isfinite(b))
        assert rel_err(1e33 * b, a) < 1e-8
    lat.close()


def test_host_fields_pipeline_matches_device_fields(cb, env):
    """Host-resident fields over several batches take the copy/compute
    pipeline (sources of the next batch and solutions of the previous one
    move on copy streams; the first batch is short).  Its batches are cut
    differently from the device path's, which changes where each rhs's
    reliable updates fall, so the two agree to the solver's accuracy: both
    meet the 1e-10 residual, solutions compared at 1e-8 as elsewhere."""
    torch = pytest.importorskip("torch")
    lat, _, _ = env
    V = lat.VOLUME
    n = 19  # 3 batches of 8: two full, one ragged
    bs = [seeded(100 + i, 24 * V) for i in range(n)]
    p = cb.solver_defaults()
    p.block_rhs = 8
    xh = [np.zeros(24 * V) for _ in range(n)]
    st = lat.solve(xh, bs, p)
    assert st.converged == n and st.max_true_res <= 1e-10
    xd = [torch.zeros(24 * V, dtype=torch.float64, device="cuda") for _ in range(n)]
    bd = [torch.from_numpy(b).cuda() for b in bs]
    st2 = lat.solve(xd, bd, p)
    torch.cuda.synchronize()
    assert st2.converged == n
    for a, d in zip(xh, xd):
        assert rel_err(a, d.cpu().numpy()) < 1e-8
