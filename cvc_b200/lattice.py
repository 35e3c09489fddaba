"""Host-side mirror of the reference interface for the operator / solver /
contraction path, over the C ABI of libcvcb200.so.

Fields are CVC-layout float64 arrays (numpy on the host, or torch CUDA
tensors on the lattice's GPU): 24*V doubles per spinor field, 72*V per
gauge field, 32*V for Pi_mu_nu.  Methods return what the reference
functions return; failures other than the reference's own solver codes
raise CvcbError.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import ptr, ptr_array


class CvcbError(RuntimeError):
    def __init__(self, where, code):
        super().__init__(f"{where} failed with status {code}: {_lib.last_error()}")
        self.code = code


def _check(where, rc):
    if rc < 0:
        raise CvcbError(where, rc)
    return rc


def geometry_tables(T, LX, LY, LZ):
    """All tables of the reference's geometry() (cvc_geometry.c:179-341),
    single process: dict of int32 arrays keyed by the reference names."""
    V = T * LX * LY * LZ
    out = {
        "g_ipt": np.zeros((T + 2) * LX * LY * LZ, np.int32),
        "g_iup": np.zeros(4 * V, np.int32),
        "g_idn": np.zeros(4 * V, np.int32),
        "g_lexic2eo": np.zeros(V, np.int32),
        "g_eo2lexic": np.zeros(V, np.int32),
        "g_iseven": np.zeros(V, np.int32),
        "g_isevent": np.zeros(V, np.int32),
        "g_lexic2eot": np.zeros(V, np.int32),
        "g_eot2lexic": np.zeros(V, np.int32),
    }
    order = ["g_ipt", "g_iup", "g_idn", "g_lexic2eo", "g_eo2lexic", "g_iseven", "g_isevent",
             "g_lexic2eot", "g_eot2lexic"]
    _check("cvcb_geometry_tables",
           _lib.load().cvcb_geometry_tables(T, LX, LY, LZ, *[ptr(out[k]) for k in order]))
    return out


def gamma_tables():
    """(gamma_permutation[16][24], gamma_sign[16][24]) of init_gamma."""
    perm = np.zeros((16, 24), np.int32)
    sign = np.zeros((16, 24), np.int32)
    _check("cvcb_gamma_tables", _lib.load().cvcb_gamma_tables(ptr(perm), ptr(sign)))
    return perm, sign


def boundary_phases(T, LX, LY, LZ, bc_angle=(1.0, 0.0, 0.0, 0.0)):
    """co_phase_up[4] as a complex128 array."""
    bc = np.asarray(bc_angle, np.float64)
    ph = np.zeros(8)
    _check("cvcb_boundary_phases",
           _lib.load().cvcb_boundary_phases(T, LX, LY, LZ, ptr(bc), ptr(ph)))
    return ph[0::2] + 1j * ph[1::2]


def ranlxd(n, seed, level=1):
    """First n numbers of RANLUX ranlxd after rlxd_init(level, seed)."""
    r = np.zeros(n)
    _check("cvcb_ranlxd", _lib.load().cvcb_ranlxd(level, seed, ptr(r), n))
    return r


def gauge_random(T, LX, LY, LZ, eps, seed):
    """Gauge field U = exp(i eps H), H random traceless hermitian (ranlxd seed)."""
    g = np.zeros(72 * T * LX * LY * LZ)
    _check("cvcb_gauge_random", _lib.load().cvcb_gauge_random(ptr(g), T, LX, LY, LZ, eps, seed))
    return g


def solver_defaults():
    p = _lib.SolverParams()
    _lib.load().cvcb_solver_defaults(ctypes.byref(p))
    return p


class Lattice:
    """One lattice context on one GPU (the state CVC keeps in globals)."""

    def __init__(self, T, LX, LY, LZ, device=0, kappa=0.125, mu=0.0,
                 bc_angle=(1.0, 0.0, 0.0, 0.0)):
        self._lib = _lib.load()
        self.T, self.LX, self.LY, self.LZ = T, LX, LY, LZ
        self.VOLUME = T * LX * LY * LZ
        h = ctypes.c_void_p()
        _check("cvcb_lattice_create",
               self._lib.cvcb_lattice_create(ctypes.byref(h), T, LX, LY, LZ, device))
        self._h = h
        self.set_params(kappa, mu, bc_angle)

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._lib.cvcb_lattice_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- parameters and gauge field --------------------------------------
    def set_params(self, kappa, mu, bc_angle=(1.0, 0.0, 0.0, 0.0)):
        """g_kappa, g_mu (bare twisted mass) and BCangle."""
        self.g_kappa, self.g_mu = float(kappa), float(mu)
        self.BCangle = tuple(float(b) for b in bc_angle)
        bc = np.asarray(self.BCangle, np.float64)
        _check("cvcb_set_params", self._lib.cvcb_set_params(self._h, self.g_kappa, self.g_mu,
                                                             ptr(bc)))

    def upload_gauge(self, gauge):
        """Set g_gauge_field (72*V doubles, CVC layout, no boundary phase)."""
        _check("cvcb_upload_gauge", self._lib.cvcb_upload_gauge(self._h, ptr(gauge)))

    def gauge_unitarity(self):
        d = ctypes.c_double()
        _check("cvcb_gauge_unitarity", self._lib.cvcb_gauge_unitarity(self._h, ctypes.byref(d)))
        return d.value

    # -- operators (Q_phi.c) -----------------------------------------------
    def Q_phi_tbc(self, xi, phi):
        _check("Q_phi_tbc", self._lib.cvcb_Q_phi_tbc(self._h, ptr(xi), ptr(phi)))

    def Hopping(self, xi, phi):
        _check("Hopping", self._lib.cvcb_Hopping(self._h, ptr(xi), ptr(phi)))

    def Qf5(self, xi, phi, mutm):
        _check("Qf5", self._lib.cvcb_Qf5(self._h, ptr(xi), ptr(phi), float(mutm)))

    def Q_phi(self, xi, phi, mutm):
        _check("Q_phi", self._lib.cvcb_Q_phi(self._h, ptr(xi), ptr(phi), float(mutm)))

    def g5_phi(self, phi):
        _check("g5_phi", self._lib.cvcb_g5_phi(self._h, ptr(phi)))

    def mul_one_pm_imu_inv(self, phi, sign, V):
        _check("mul_one_pm_imu_inv",
               self._lib.cvcb_mul_one_pm_imu_inv(self._h, ptr(phi), float(sign), int(V)))

    # -- reductions (invert_Qtm.c:28-84) ---------------------------------
    def spinor_scalar_product_co(self, xi, phi, V):
        w = np.zeros(2)
        _check("spinor_scalar_product_co",
               self._lib.cvcb_spinor_scalar_product_co(self._h, ptr(w), ptr(xi), ptr(phi), int(V)))
        return complex(w[0], w[1])

    def spinor_scalar_product_re(self, xi, phi, V):
        r = np.zeros(1)
        _check("spinor_scalar_product_re",
               self._lib.cvcb_spinor_scalar_product_re(self._h, ptr(r), ptr(xi), ptr(phi), int(V)))
        return float(r[0])

    # -- solvers (invert_Qtm.c) ------------------------------------------
    def invert_Qtm(self, xi, phi, solver_precision, niter_max, return_residual=False):
        """BiCGStab on Q.  Returns niter, -2 or -3 as the reference does (-3
        also for a broken-down recursion, which the C ABI reports as -4)."""
        tr = np.zeros(1)
        rc = self._lib.cvcb_invert_Qtm(self._h, ptr(xi), ptr(phi), float(solver_precision),
                                       int(niter_max), ptr(tr))
        if rc == _lib.CVCB_BREAKDOWN:  # the reference returns -3 here
            rc = _lib.CVCB_NO_CONVERGENCE
        if rc < 0 and rc not in (_lib.CVCB_ERR_NULL, _lib.CVCB_NO_CONVERGENCE):
            raise CvcbError("invert_Qtm", rc)
        return (rc, float(tr[0])) if return_residual else rc

    def invert_Qtm_her(self, xi, phi, solver_precision, niter_max, return_residual=False):
        """BiCGStab on Q(-mu)^+ Q(-mu), x = g5 Q(-mu) y."""
        tr = np.zeros(1)
        rc = self._lib.cvcb_invert_Qtm_her(self._h, ptr(xi), ptr(phi), float(solver_precision),
                                           int(niter_max), ptr(tr))
        if rc == _lib.CVCB_BREAKDOWN:  # the reference returns -3 here
            rc = _lib.CVCB_NO_CONVERGENCE
        if rc < 0 and rc not in (_lib.CVCB_ERR_NULL, _lib.CVCB_NO_CONVERGENCE):
            raise CvcbError("invert_Qtm_her", rc)
        return (rc, float(tr[0])) if return_residual else rc

    def sloppy_normal_op(self, ins, outs, precision, link_recon=12, layout=0):
        """M^+ M of the batched solver's inner iterations on the odd sites of
        CVC-layout fields (even sites of the outputs zero)."""
        if len(ins) != len(outs):
            raise ValueError("ins and outs differ in length")
        _check("cvcb_sloppy_normal_op", self._lib.cvcb_sloppy_normal_op(
            self._h, int(precision), int(link_recon), int(layout), len(ins), ptr_array(ins),
            ptr_array(outs)))

    def solve(self, xs, bs, params=None):
        """Batched even/odd mixed-precision solve of Q x_i = b_i."""
        if params is None:
            params = solver_defaults()
        if len(xs) != len(bs):
            raise ValueError("xs and bs differ in length")
        st = _lib.SolverStats()
        _check("cvcb_solve", self._lib.cvcb_solve(self._h, ptr_array(xs), ptr_array(bs), len(xs),
                                                  ctypes.byref(params), ctypes.byref(st)))
        return st

    # -- contractions ----------------------------------------------------
    def cvc_contract(self, fields, source_site, conn=None, want_contact=True):
        """Pi_mu_nu(x) of cvc_exact2_xspace.c:577-861 for 120 propagator
        columns; returns (conn, contact)."""
        if len(fields) != 120:
            raise ValueError("120 propagator fields expected")
        if conn is None:
            conn = np.zeros(32 * self.VOLUME)
        contact = np.zeros(8)
        _check("cvc_contract", self._lib.cvcb_cvc_contract(
            self._h, ptr_array(fields), int(source_site), ptr(conn),
            ptr(contact) if want_contact else None))
        return conn, contact

    def cvc_ward(self, conn):
        wi = np.zeros(8 * self.VOLUME)
        _check("cvc_ward", self._lib.cvcb_cvc_ward(self._h, ptr(conn), ptr(wi)))
        return wi

    def p2gg_seq_source(self, source, prop, timeslice, momentum, gamma_id, propagator_position):
        mom = np.asarray(momentum, np.int32)
        _check("p2gg_seq_source", self._lib.cvcb_p2gg_seq_source(
            self._h, ptr(source), ptr(prop), int(timeslice), ptr(mom), int(gamma_id),
            int(propagator_position)))

    # -- derivatives of Pi (no counterpart in the reference) -------------
    def pi_forward(self, source_site, params=None, keep_bytes=float("inf"), conn=None):
        """Solve the 120 columns of source point y and contract: (conn, contact)."""
        if params is None:
            params = solver_defaults()
        if conn is None:
            conn = np.zeros(32 * self.VOLUME)
        contact = np.zeros(8)
        kb = 1e300 if keep_bytes == float("inf") else float(keep_bytes)
        _check("pi_forward", self._lib.cvcb_pi_forward(self._h, int(source_site),
                                                        ctypes.byref(params), kb, ptr(conn),
                                                        ptr(contact)))
        return conn, contact

    def pi_tangent(self, parameter):
        """dPi/dmu (parameter 'mu') or dPi/dkappa ('kappa') at the last forward state."""
        code = {"mu": 0, "kappa": 1}[parameter]
        d = np.zeros(32 * self.VOLUME)
        _check("pi_tangent", self._lib.cvcb_pi_tangent(self._h, code, ptr(d)))
        return d

    def pi_backward(self, weights, want_gauge=True):
        """For L = Re sum conj(w) Pi: (dL/dmu, dL/dkappa, dL/dU or None)."""
        w = np.ascontiguousarray(weights, np.float64)
        dmu = np.zeros(1)
        dka = np.zeros(1)
        gu = np.zeros(72 * self.VOLUME) if want_gauge else None
        _check("pi_backward", self._lib.cvcb_pi_backward(self._h, ptr(w), ptr(gu), ptr(dmu),
                                                          ptr(dka)))
        return float(dmu[0]), float(dka[0]), gu

    def pi_momentum(self, conn, source_site, contact=None, out=None):
        """Pi_mu_nu(q) with midpoint phases and the contact term subtracted
        (32*V doubles, momenta in lexicographic order)."""
        if out is None:
            out = np.zeros(32 * self.VOLUME)
        ct = None if contact is None else np.ascontiguousarray(contact, np.float64)
        _check("pi_momentum", self._lib.cvcb_pi_momentum(self._h, ptr(conn), int(source_site),
                                                          ptr(ct), ptr(out)))
        return out

    # -- hopping-parameter expansion (Q_phi.c:536-781) -------------------
    def BHn(self, xi, phi, n):
        """xi = (B H)^n phi; phi is overwritten as the reference does."""
        _check("BHn", self._lib.cvcb_BHn(self._h, ptr(xi), ptr(phi), int(n)))

    def BH(self, xi, phi):
        _check("BH", self._lib.cvcb_BH(self._h, ptr(xi), ptr(phi)))

    def BH2(self, xi, phi):
        _check("BH2", self._lib.cvcb_BH2(self._h, ptr(xi), ptr(phi)))

    def BH3(self, xi, phi):
        _check("BH3", self._lib.cvcb_BH3(self._h, ptr(xi), ptr(phi)))

    def BH5(self, xi, phi):
        _check("BH5", self._lib.cvcb_BH5(self._h, ptr(xi), ptr(phi)))

    def BH7(self, xi, phi):
        _check("BH7", self._lib.cvcb_BH7(self._h, ptr(xi), ptr(phi)))

    def gamma5_BdagH4_gamma5(self, xi, phi, work):
        _check("gamma5_BdagH4_gamma5",
               self._lib.cvcb_gamma5_BdagH4_gamma5(self._h, ptr(xi), ptr(phi), ptr(work)))

    def plaquette(self):
        pl = np.zeros(1)
        ls = np.zeros(2)
        _check("plaquette", self._lib.cvcb_plaquette(self._h, ptr(pl), ptr(ls)))
        return float(pl[0]), complex(ls[0], ls[1])
