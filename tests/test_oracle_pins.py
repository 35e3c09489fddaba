"""The oracle (oracle/cvc_oracle.c) pinned against the reference: against
the committed golden fixtures (outputs of the unmodified reference, made by
tests/golden/make_golden.py) and, where the compiled reference is present,
live.  The restatement follows the reference's operation order, so the
comparisons are bit-exact."""
import os

import numpy as np
import pytest

from golden import inputs

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = np.load(os.path.join(HERE, "golden", "reference_fixtures.npz"))
DIMS, V = (4, 4, 4, 4), 256
KAPPA, MU = 0.15, 0.01 / 0.3


@pytest.fixture(scope="module")
def orc(oracle_mod):
    o = oracle_mod.Oracle(*DIMS, KAPPA, MU)
    o.set_gauge(inputs.gauge(1, V))
    return o


@pytest.mark.parametrize("dims", [(8, 4, 4, 4), (6, 4, 2, 4)])
def test_geometry_tables(oracle_mod, dims):
    o = oracle_mod.Oracle(*dims, 0.15, 0.1)
    tag = "x".join(map(str, dims))
    for k, v in o.tables().items():
        assert np.array_equal(v, FIX[f"geom_{tag}_{k}"]), k


def test_gamma_and_phases(oracle_mod):
    o = oracle_mod.Oracle(8, 6, 4, 2, 0.15, 0.1, (1.0, 0.5, 0.0, 0.25))
    perm, sign = o.gamma()
    assert np.array_equal(perm, FIX["gamma_perm"])
    assert np.array_equal(sign, FIX["gamma_sign"])
    assert np.array_equal(np.array(o.L.phase[:]), FIX["phase_8x6x4x2_1.0_0.5_0.0_0.25"])


def test_operators_bit_exact(orc):
    phi = inputs.field(2, 24 * V)
    assert np.array_equal(orc.Q_phi_tbc(phi), FIX["op_Q_phi_tbc"])
    assert np.array_equal(orc.Hopping(phi), FIX["op_Hopping"])
    assert np.array_equal(orc.Qf5(phi, MU), FIX["op_Qf5_plus"])
    assert np.array_equal(orc.Qf5(phi, -MU), FIX["op_Qf5_minus"])
    assert np.array_equal(orc.Q_phi(phi, 0.0731), FIX["op_Q_phi_0.0731"])
    assert np.array_equal(orc.g5_phi(phi), FIX["op_g5_phi"])
    assert np.array_equal(orc.mul_one_pm_imu_inv(phi, 1.0, V), FIX["op_imu_plus"])
    assert np.array_equal(orc.mul_one_pm_imu_inv(phi, -1.0, V // 2), FIX["op_imu_minus_half"])


def test_reductions_and_plaquette(orc):
    phi, psi = inputs.field(2, 24 * V), inputs.field(3, 24 * V)
    assert orc.scalar_product_co(phi, psi, V) == complex(FIX["dot_co"])
    assert orc.scalar_product_co(phi, psi, 77) == complex(FIX["dot_co_part"])
    assert orc.plaquette()[0] == float(FIX["plaquette"])


def test_solvers_bit_exact(orc):
    b = np.zeros(24 * V)
    b[10] = 1.0
    n, x, tr = orc.invert(b, 1e-20, 1000, her=True)
    assert n == int(FIX["her_point_niter"])
    assert np.array_equal(x, FIX["her_point_x"])
    assert tr < 1e-18  # stopping rule is on the normal-equation residual
    n, _, _ = orc.invert(b, 1e-20, 30, her=False)
    assert n == int(FIX["bicg_point_status"]) == -3
    orc.set_params(0.10, 0.02)
    n, x, _ = orc.invert(inputs.field(2, 24 * V), 1e-24, 1000, her=False)
    orc.set_params(KAPPA, MU)
    assert n == int(FIX["bicg_rand_k0.10_niter"])
    assert np.array_equal(x, FIX["bicg_rand_k0.10_x"])


def test_contraction_bit_exact(orc):
    fields = [inputs.field(100 + i, 24 * V) for i in range(120)]
    conn, contact = orc.cvc_contract(fields, 37)
    assert np.array_equal(conn, FIX["pi_random_src37"])
    # the reference prints the contact term with 16 significant digits
    assert np.allclose(contact, FIX["pi_random_src37_contact"], rtol=1e-15, atol=0)


def test_ward_identity_fixture(orc):
    """The reference's own WI output on solved propagators: zero divergence
    except +contact at the source and -contact at source + nu."""
    wi = FIX["pi_solved_src0_wi"].reshape(V, 4, 2)
    w = wi[..., 0] + 1j * wi[..., 1]
    ct = FIX["pi_solved_src0_contact"]
    shifted = [64, 16, 4, 1]
    for nu in range(4):
        c = ct[2 * nu] + 1j * ct[2 * nu + 1]
        assert abs(w[0, nu] - c) < 1e-13
        assert abs(w[shifted[nu], nu] + c) < 1e-13
    mask = np.ones((V, 4), bool)
    mask[0, :] = False
    for nu in range(4):
        mask[shifted[nu], nu] = False
    assert np.max(np.abs(w[mask])) < 1e-13
    # the oracle's divergence of the reference's Pi is the same
    owi = orc.cvc_ward(FIX["pi_solved_src0"]).reshape(V, 4, 2)
    assert np.max(np.abs(owi - wi)) < 1e-15


def test_live_reference(oracle_mod, orc):
    """Against the compiled reference itself (skipped where it was not built)."""
    if not oracle_mod.reference_available():
        pytest.skip("oracle/_ref not built")
    ref = oracle_mod.Reference(*DIMS, KAPPA, MU)
    g = inputs.gauge(5, V)
    ref.set_gauge(g)
    orc.set_gauge(g)
    phi = inputs.field(6, 24 * V)
    assert np.array_equal(ref.Q_phi_tbc(phi), orc.Q_phi_tbc(phi))
    assert np.array_equal(ref.Qf5(phi, -MU), orc.Qf5(phi, -MU))
    b = np.zeros(24 * V)
    b[0] = 1.0
    n1, x1 = ref.invert(b, 1e-20, 1000, her=True)
    n2, x2, _ = orc.invert(b, 1e-20, 1000, her=True)
    assert n1 == n2 and np.array_equal(x1, x2)
    orc.set_gauge(inputs.gauge(1, V))
