"""Generate the golden fixtures in this directory from the UNMODIFIED
reference, compiled from its own sources by oracle/Makefile (`make -C
oracle ref`): oracle/_ref/libcvcref.so (the functions) and
oracle/_ref/cvc_exact2_xspace (the contraction program).

Run from the repository root:  python tests/golden/make_golden.py
Inputs come from tests/golden/inputs.py (splitmix64), so the fixtures hold
reference OUTPUTS plus the parameters needed to rebuild the inputs.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, HERE)

import inputs  # noqa: E402
import oracle_bind as ob  # noqa: E402


def geometry(dims):
    r = ob.Reference(*dims, 0.15, 0.1)
    t = r.tables()
    return {f"{k}": v for k, v in t.items()}


def main():
    if not ob.reference_available():
        sys.exit("oracle/_ref/libcvcref.so missing: run `make -C oracle ref` first")
    out = {}
    # --- geometry, gamma, phases (cvc_geometry.c, cvc_utils.c:707) --------
    for dims in [(8, 4, 4, 4), (6, 4, 2, 4)]:
        tag = "x".join(map(str, dims))
        for k, v in geometry(dims).items():
            out[f"geom_{tag}_{k}"] = v
    r = ob.Reference(8, 4, 4, 4, 0.15, 0.1)
    out["gamma_perm"], out["gamma_sign"] = r.gamma()
    for bc in [(1.0, 0.0, 0.0, 0.0), (1.0, 0.5, 0.0, 0.25)]:
        rr = ob.Reference(8, 6, 4, 2, 0.15, 0.1, bc)
        out["phase_8x6x4x2_" + "_".join(str(b) for b in bc)] = rr.phases()
    # --- RANLUX (ranlxd.c) ---------------------------------------------------
    for seed, level, n in [(1234, 1, 2000), (7, 2, 2000), (11, 1, 500), (3, 1, 500), (21, 1, 500),
                           (1, 1, 500)]:
        out[f"ranlxd_{seed}_{level}"] = r.ranlxd(n, seed, level)
    # --- file names (cvc_utils.c:2143), on an 8x4x4x4 lattice ------------------
    r = ob.Reference(8, 4, 4, 4, 0.15, 0.1)
    names = []
    for fmt, nu, sc, sign in [(0, 4, 7, 1), (0, 2, 11, -1), (0, 1, 0, 0), (2, 3, 5, 1), (3, 0, 9, -1),
                              (4, 4, 2, 1)]:
        names.append(r.get_filename(nu, sc, sign, "source", "dnprop", 17, fmt, 37))
    out["filenames"] = np.array(names)

    # --- operators, reductions, solvers on 4^4 (Q_phi.c, invert_Qtm.c) --------
    dims = (4, 4, 4, 4)
    V = 256
    kappa, mu = 0.15, 0.01 / 0.3
    ref = ob.Reference(*dims, kappa, mu)
    g = inputs.gauge(1, V)
    ref.set_gauge(g)
    phi = inputs.field(2, 24 * V)
    psi = inputs.field(3, 24 * V)
    out["op_Q_phi_tbc"] = ref.Q_phi_tbc(phi)
    out["op_Hopping"] = ref.Hopping(phi)
    out["op_Qf5_plus"] = ref.Qf5(phi, mu)
    out["op_Qf5_minus"] = ref.Qf5(phi, -mu)
    out["op_Q_phi_0.0731"] = ref.Q_phi(phi, 0.0731)
    out["op_g5_phi"] = ref.g5_phi(phi)
    out["op_imu_plus"] = ref.mul_one_pm_imu_inv(phi, 1.0, V)
    out["op_imu_minus_half"] = ref.mul_one_pm_imu_inv(phi, -1.0, V // 2)
    out["dot_co"] = np.array(ref.scalar_product_co(phi, psi, V))
    out["dot_co_part"] = np.array(ref.scalar_product_co(phi, psi, 77))
    out["plaquette"] = np.array(ref.plaquette())
    b = np.zeros(24 * V)
    b[2 * 5] = 1.0  # point source, spin 1 colour 2, site 0
    n, x = ref.invert(b, 1e-20, 1000, her=True)
    out["her_point_niter"] = np.array(n)
    out["her_point_x"] = x
    n, x = ref.invert(b, 1e-20, 30, her=False)
    out["bicg_point_status"] = np.array(n)
    ref.set_params(0.10, 0.02)
    n, x = ref.invert(phi, 1e-24, 1000, her=False)
    out["bicg_rand_k0.10_niter"] = np.array(n)
    out["bicg_rand_k0.10_x"] = x
    ref.set_params(kappa, mu)

    # --- contraction on random fields (cvc_exact2_xspace.c:577-861) ----------
    fields = [inputs.field(100 + i, 24 * V) for i in range(120)]
    conn, _, log = ob.reference_contraction(g, fields, dims, kappa, mu, 37)
    out["pi_random_src37"] = conn
    out["pi_random_src37_contact"] = parse_contact(log)

    # --- Ward identity with solved propagators (:928-1008) -------------------
    src = 0
    shifted = [64, 16, 4, 1, 0]
    up, dn = [], []
    for m in range(5):
        for sc in range(12):
            bb = np.zeros(24 * V)
            bb[24 * shifted[m] + 2 * sc] = 1.0
            ref.set_params(kappa, mu)
            _, xu = ref.invert(bb, 1e-26, 3000, her=True)
            ref.set_params(kappa, -mu)
            _, xd = ref.invert(bb, 1e-26, 3000, her=True)
            up.append(xu)
            dn.append(xd)
    conn, wi, log = ob.reference_contraction(g, up + dn, dims, kappa, mu, src, ward=True)
    out["pi_solved_src0"] = conn
    out["pi_solved_src0_contact"] = parse_contact(log)
    out["pi_solved_src0_wi"] = parse_wi(wi, V)
    np.savez_compressed(os.path.join(HERE, "reference_fixtures.npz"), **out)
    print("wrote", os.path.join(HERE, "reference_fixtures.npz"), len(out), "arrays")


def parse_contact(log):
    lines = log.splitlines()
    i = max(k for k, l in enumerate(lines) if l.startswith("# [cvc_exact2_xspace] contact term"))
    vals = []
    for l in lines[i + 1:i + 5]:
        f = l.split()
        vals += [float(f[1]), float(f[2])]
    return np.array(vals)


def parse_wi(text, V):
    vals = []
    for l in text.splitlines():
        if l.startswith("#"):
            continue
        f = l.split()
        vals += [float(f[1]), float(f[2])]
    a = np.array(vals)
    assert a.size == 8 * V
    return a


if __name__ == "__main__":
    main()
