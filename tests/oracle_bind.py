"""ctypes access to the oracle (test infrastructure only).

* `Oracle`   -- oracle/liboracle.so, the plain-C restatement of the path
               (oracle/cvc_oracle.c).  Always buildable with gcc.
* `Reference` -- oracle/_ref/libcvcref.so, the unmodified reference sources
               compiled by oracle/Makefile (present when the reference tree
               was available at build time; the built file travels with the
               repository).
* `reference_contraction` -- runs the unmodified cvc_exact2_xspace program
               (oracle/_ref/cvc_exact2_xspace) on raw-binary inputs.
"""
import ctypes
import os
import subprocess
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_LIB = os.path.join(ORACLE_DIR, "liboracle.so")
REF_DIR = os.path.join(ORACLE_DIR, "_ref")
REF_LIB = os.path.join(REF_DIR, "libcvcref.so")
REF_OMP_LIB = os.path.join(REF_DIR, "libcvcref_omp.so")
REF_CONTRACT = os.path.join(REF_DIR, "cvc_exact2_xspace")
# where the reference sources lie (only read at build time, to compile them)
REFERENCE_TREE = os.environ.get("CVC_REFERENCE_TREE", "/root/reference")

_P = ctypes.c_void_p
_D = ctypes.c_double
_I = ctypes.c_int


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def build_oracle():
    """Build liboracle.so if missing, and the reference objects when the
    reference tree is present."""
    if not os.path.exists(ORACLE_LIB):
        subprocess.run(["make", "-C", ORACLE_DIR, "liboracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    if os.path.isdir(REFERENCE_TREE) and not os.path.exists(REF_LIB):
        subprocess.run(["make", "-C", ORACLE_DIR, "ref", "-j8"], check=True,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)


def reference_available():
    return os.path.exists(REF_LIB)


def reference_ranlxd(n, seed, level=1):
    """The first n numbers of the reference's ranlxd stream (ranlxd.c) after
    rlxd_init(level, seed), without initialising a lattice."""
    lib = Reference._lib if Reference._lib is not None else ctypes.CDLL(REF_LIB)
    r = np.zeros(n)
    lib.ref_rlxd_init(level, seed)
    lib.ref_ranlxd(_p(r), n)
    return r


class OrcLattice(ctypes.Structure):
    _fields_ = [
        ("T", _I), ("LX", _I), ("LY", _I), ("LZ", _I), ("V", _I),
        ("kappa", _D), ("mu", _D),
        ("phase", _D * 8),
        ("iup", ctypes.POINTER(_I)), ("idn", ctypes.POINTER(_I)),
        ("gauge", ctypes.POINTER(_D)),
        ("gperm", _I * (16 * 24)), ("gsign", _I * (16 * 24)),
    ]


class Oracle:
    """The plain-C restatement, on one lattice."""

    def __init__(self, T, LX, LY, LZ, kappa, mu, bc=(1.0, 0.0, 0.0, 0.0)):
        build_oracle()
        self.lib = ctypes.CDLL(ORACLE_LIB)
        self.L = OrcLattice()
        self.V = T * LX * LY * LZ
        self.dims = (T, LX, LY, LZ)
        bca = np.asarray(bc, np.float64)
        rc = self.lib.orc_lattice_init(ctypes.byref(self.L), T, LX, LY, LZ, _D(kappa), _D(mu),
                                       _p(bca))
        assert rc == 0
        self._gauge = None

    def set_gauge(self, g):
        self._gauge = np.ascontiguousarray(g, np.float64)
        self.L.gauge = self._gauge.ctypes.data_as(ctypes.POINTER(_D))

    def set_params(self, kappa, mu):
        self.L.kappa = kappa
        self.L.mu = mu

    def tables(self):
        T, LX, LY, LZ = self.dims
        V = self.V
        t = {k: np.zeros(n, np.int32) for k, n in [
            ("g_ipt", (T + 2) * LX * LY * LZ), ("g_iup", 4 * V), ("g_idn", 4 * V),
            ("g_lexic2eo", V), ("g_eo2lexic", V), ("g_iseven", V), ("g_isevent", V),
            ("g_lexic2eot", V), ("g_eot2lexic", V)]}
        self.lib.orc_geometry_tables(ctypes.byref(self.L), *[_p(t[k]) for k in [
            "g_ipt", "g_iup", "g_idn", "g_lexic2eo", "g_eo2lexic", "g_iseven", "g_isevent",
            "g_lexic2eot", "g_eot2lexic"]])
        return t

    def gamma(self):
        perm = np.zeros((16, 24), np.int32)
        sign = np.zeros((16, 24), np.int32)
        self.lib.orc_gamma_tables(_p(perm), _p(sign))
        return perm, sign

    def _op(self, name, phi, *extra):
        out = np.zeros(24 * self.V)
        getattr(self.lib, name)(ctypes.byref(self.L), _p(out),
                                _p(np.ascontiguousarray(phi)), *extra)
        return out

    def Q_phi_tbc(self, phi):
        return self._op("orc_Q_phi_tbc", phi)

    def Hopping(self, phi):
        return self._op("orc_Hopping", phi)

    def Qf5(self, phi, mutm):
        return self._op("orc_Qf5", phi, _D(mutm))

    def Q_phi(self, phi, mutm):
        return self._op("orc_Q_phi", phi, _D(mutm))

    def g5_phi(self, phi):
        out = np.array(phi, dtype=np.float64, copy=True)
        self.lib.orc_g5_phi(ctypes.byref(self.L), _p(out))
        return out

    def mul_one_pm_imu_inv(self, phi, sign, V):
        out = np.array(phi, dtype=np.float64, copy=True)
        self.lib.orc_mul_one_pm_imu_inv(ctypes.byref(self.L), _p(out), _D(sign), V)
        return out

    def scalar_product_co(self, a, b, V):
        w = np.zeros(2)
        self.lib.orc_scalar_product_co(_p(w), _p(np.ascontiguousarray(a)),
                                       _p(np.ascontiguousarray(b)), V)
        return complex(w[0], w[1])

    def invert(self, phi, prec, nmax, her=True, x0=None):
        x = np.zeros(24 * self.V) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
        work = np.zeros(7 * 24 * self.V)
        tr = np.zeros(1)
        fn = self.lib.orc_invert_Qtm_her if her else self.lib.orc_invert_Qtm
        rc = fn(ctypes.byref(self.L), _p(x), _p(np.ascontiguousarray(phi)), _D(prec), nmax,
                _p(work), _p(tr))
        return rc, x, float(tr[0])

    def cvc_contract(self, fields, src):
        arr = (ctypes.c_void_p * 120)(*[f.ctypes.data for f in fields])
        conn = np.zeros(32 * self.V)
        contact = np.zeros(8)
        self.lib.orc_cvc_contract(ctypes.byref(self.L), arr, src, _p(conn), _p(contact))
        return conn, contact

    def cvc_contract_sites(self, sites, src, fetch):
        """Pi_mu_nu at the lexicographic `sites` only, and the contact term,
        for lattices whose 120 full fields would not fit the host.  Pi(x)
        reads the fields at x and x + mu-hat and the links at x (the contact
        term the fields at the source and source + nu-hat), so the oracle's
        own contraction runs unchanged on a compact lattice made of those
        sites: the same per-site arithmetic, with the neighbour table and the
        links restricted to them.  `fetch(idx)` returns the 120 columns at
        the lexicographic sites idx, each an array of shape (len(idx), 24).
        Returns (pi of shape (len(sites), 32), contact)."""
        iup = np.ctypeslib.as_array(self.L.iup, shape=(4 * self.V,)).reshape(-1, 4)
        need = sorted(set(int(x) for x in sites) | {int(src)})
        G = np.array(sorted(set(need) | set(iup[need].ravel().tolist())), np.int64)
        pos = {int(x): i for i, x in enumerate(G)}
        iup_c = np.zeros((len(G), 4), np.int32)  # sites outside `need` point at row 0
        for x in need:
            iup_c[pos[x]] = [pos[int(n)] for n in iup[x]]
        gauge_c = np.ascontiguousarray(self._gauge.reshape(-1, 72)[G])
        rows = [np.ascontiguousarray(r, np.float64) for r in fetch(G)]
        assert len(rows) == 120 and all(r.shape == (len(G), 24) for r in rows)
        Lc = OrcLattice()
        ctypes.pointer(Lc)[0] = self.L
        Lc.V = len(G)
        Lc.iup = iup_c.ctypes.data_as(ctypes.POINTER(_I))
        Lc.idn = Lc.iup
        Lc.gauge = gauge_c.ctypes.data_as(ctypes.POINTER(_D))
        arr = (ctypes.c_void_p * 120)(*[r.ctypes.data for r in rows])
        conn = np.zeros(32 * len(G))
        contact = np.zeros(8)
        self.lib.orc_cvc_contract(ctypes.byref(Lc), arr, pos[int(src)], _p(conn), _p(contact))
        return conn.reshape(-1, 32)[[pos[int(x)] for x in sites]], contact

    def cvc_ward(self, conn):
        wi = np.zeros(8 * self.V)
        self.lib.orc_cvc_ward(ctypes.byref(self.L), _p(np.ascontiguousarray(conn)), _p(wi))
        return wi

    def seq_source(self, prop, t, mom, gamma_id, pos):
        out = np.zeros(24 * self.V)
        m = np.asarray(mom, np.int32)
        self.lib.orc_p2gg_seq_source(ctypes.byref(self.L), _p(out),
                                     _p(np.ascontiguousarray(prop)), t, _p(m), gamma_id, pos)
        return out

    def plaquette(self):
        pl = np.zeros(1)
        ls = np.zeros(2)
        self.lib.orc_plaquette(ctypes.byref(self.L), _p(pl), _p(ls))
        return float(pl[0]), complex(ls[0], ls[1])


class Reference:
    """The unmodified reference functions (oracle/_ref/libcvcref.so).  The
    reference keeps global state, so only one lattice exists per process;
    `init` replaces it."""

    _lib = None

    def __init__(self, T, LX, LY, LZ, kappa, mu, bc=(1.0, 0.0, 0.0, 0.0), omp=False):
        path = REF_OMP_LIB if omp else REF_LIB
        if Reference._lib is None or Reference._lib._name != path:
            Reference._lib = ctypes.CDLL(path)
        self.lib = Reference._lib
        bca = np.asarray(bc, np.float64)
        self._quiet(lambda: self.lib.ref_init(T, LX, LY, LZ, _D(kappa), _D(mu), _p(bca)))
        self.V = self.lib.ref_volume()
        self.dims = (T, LX, LY, LZ)

    @staticmethod
    def _quiet(fn):
        # the reference prints to stdout; keep the test log readable
        import sys
        sys.stdout.flush()
        saved = os.dup(1)
        devnull = os.open(os.devnull, os.O_WRONLY)
        os.dup2(devnull, 1)
        try:
            return fn()
        finally:
            os.dup2(saved, 1)
            os.close(devnull)
            os.close(saved)

    def set_gauge(self, g):
        self.lib.ref_set_gauge(_p(np.ascontiguousarray(g, np.float64)))

    def set_params(self, kappa, mu):
        self.lib.ref_set_params(_D(kappa), _D(mu))

    def tables(self):
        T, LX, LY, LZ = self.dims
        V = self.V
        t = {k: np.zeros(n, np.int32) for k, n in [
            ("g_ipt", (T + 2) * LX * LY * LZ), ("g_iup", 4 * V), ("g_idn", 4 * V),
            ("g_lexic2eo", V), ("g_eo2lexic", V), ("g_iseven", V), ("g_isevent", V),
            ("g_lexic2eot", V), ("g_eot2lexic", V)]}
        self.lib.ref_get_tables(*[_p(t[k]) for k in [
            "g_ipt", "g_iup", "g_idn", "g_lexic2eo", "g_eo2lexic", "g_iseven", "g_isevent",
            "g_lexic2eot", "g_eot2lexic"]])
        return t

    def gamma(self):
        perm = np.zeros((16, 24), np.int32)
        sign = np.zeros((16, 24), np.int32)
        self.lib.ref_get_gamma(_p(perm), _p(sign))
        return perm, sign

    def phases(self):
        ph = np.zeros(8)
        self.lib.ref_get_phase(_p(ph))
        return ph

    def _op(self, name, phi, *extra):
        out = np.zeros(24 * self.V)
        inp = np.array(phi, dtype=np.float64, copy=True)
        getattr(self.lib, name)(_p(out), _p(inp), *extra)
        return out

    def Q_phi_tbc(self, phi):
        return self._op("ref_Q_phi_tbc", phi)

    def Hopping(self, phi):
        return self._op("ref_Hopping", phi)

    def Qf5(self, phi, mutm):
        return self._op("ref_Qf5", phi, _D(mutm))

    def Q_phi(self, phi, mutm):
        return self._op("ref_Q_phi", phi, _D(mutm))

    def g5_phi(self, phi):
        out = np.array(phi, dtype=np.float64, copy=True)
        self.lib.ref_g5_phi(_p(out))
        return out

    def mul_one_pm_imu_inv(self, phi, sign, V):
        out = np.array(phi, dtype=np.float64, copy=True)
        self.lib.ref_mul_one_pm_imu_inv(_p(out), _D(sign), V)
        return out

    def scalar_product_co(self, a, b, V):
        w = np.zeros(2)
        self.lib.ref_scalar_product_co(_p(w), _p(np.array(a, copy=True)),
                                       _p(np.array(b, copy=True)), V)
        return complex(w[0], w[1])

    def invert(self, phi, prec, nmax, her=True, x0=None):
        x = np.zeros(24 * self.V) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
        fn = self.lib.ref_invert_Qtm_her if her else self.lib.ref_invert_Qtm
        rc = fn(_p(x), _p(np.array(phi, dtype=np.float64, copy=True)), _D(prec), nmax, 1)
        return rc, x

    def hpe(self, name, phi, *extra):
        """Runs the reference's BHn / BH / BH2 / BH3 / BH5 / BH7 (extra = (n,)
        for BHn) on copies; returns (xi, phi) after the call."""
        xi = np.zeros(24 * self.V)
        ph = np.array(phi, dtype=np.float64, copy=True)
        getattr(self.lib, "ref_" + name)(_p(xi), _p(ph), *extra)
        return xi, ph

    def gamma5_BdagH4_gamma5(self, phi):
        xi = np.zeros(24 * self.V)
        work = np.zeros(24 * self.V)
        ph = np.array(phi, dtype=np.float64, copy=True)
        self.lib.ref_gamma5_BdagH4_gamma5(_p(xi), _p(ph), _p(work))
        return xi, ph, work

    def plaquette(self):
        pl = np.zeros(1)
        self._quiet(lambda: self.lib.ref_plaquette(_p(pl)))
        return float(pl[0])

    def ranlxd(self, n, seed, level=1):
        r = np.zeros(n)
        self.lib.ref_rlxd_init(level, seed)
        self.lib.ref_ranlxd(_p(r), n)
        return r

    def get_filename(self, nu, sc, sign, prefix, prefix2, nconf, fmt, src):
        buf = ctypes.create_string_buffer(512)
        self.lib.ref_get_filename(buf, nu, sc, sign, prefix.encode(), prefix2.encode(), nconf,
                                  fmt, src)
        return buf.value.decode()


def reference_contraction(gauge, fields, dims, kappa, mu, source_location, bc=(1.0, 0, 0, 0),
                          ward=False):
    """Run the unmodified cvc_exact2_xspace on raw inputs; returns conn
    (32*V doubles) and, with ward=True, the WI_X text file contents."""
    T, LX, LY, LZ = dims
    V = T * LX * LY * LZ
    with tempfile.TemporaryDirectory() as d:
        gauge.astype(np.float64).tofile(os.path.join(d, "conf.0000"))
        for mu_ in range(5):
            for sc in range(12):
                # record 0 = up (fields[12*mu+sc]), record 1 = dn (fields[60+12*mu+sc])
                rec = np.concatenate([fields[12 * mu_ + sc], fields[60 + 12 * mu_ + sc]])
                rec.astype(np.float64).tofile(
                    os.path.join(d, "prop.0000.%02d.%02d.inverted" % (mu_, sc)))
        with open(os.path.join(d, "cvc.input"), "w") as f:
            f.write(f"T = {T}\nLX = {LX}\nLY = {LY}\nLZ = {LZ}\n")
            f.write(f"kappa = {kappa!r}\nmu = {mu!r}\nNconf = 0\n")
            f.write("BCangleT = %r\nBCangleX = %r\nBCangleY = %r\nBCangleZ = %r\n" % tuple(bc))
            f.write("filename_prefix = prop\nfilename_prefix2 = prop\n")
            f.write("gaugefilename_prefix = conf\nformat = 0\n")
            f.write(f"source_location = {source_location}\n")
            f.write("outfile_prefix = NA\n")
        args = [REF_CONTRACT, "-f", "cvc.input"] + (["-w"] if ward else [])
        out = subprocess.run(args, cwd=d, capture_output=True, text=True, check=True)
        conn = np.fromfile(os.path.join(d, "cvc2_v_x.0000"), dtype=np.float64)
        assert conn.size == 32 * V
        wi = None
        if ward:
            with open(os.path.join(d, "WI_X.0000.0000")) as f:
                wi = f.read()
        return conn, wi, out.stdout
