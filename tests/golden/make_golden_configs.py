"""Golden fixtures at the benchmark configurations, from the UNMODIFIED
reference compiled by oracle/Makefile (`make -C oracle ref`):
oracle/_ref/libcvcref.so (invert_Qtm_her, invert_Qtm.c:276-478) and
oracle/_ref/cvc_exact2_xspace (the contraction program,
cvc_exact2_xspace.c:577-861).

    python tests/golden/make_golden_configs.py c1   # -> reference_c1.npz
    python tests/golden/make_golden_configs.py c3   # -> reference_c3.npz

Gauge fields follow the benchmark recipe (oracle/gauge_recipe.py) over the
reference's own ranlxd, so the inputs are rebuilt from the parameters stored
with the outputs.

c1: 8^3x16, kappa 0.150, 2 kappa mu 0.01, eps 0.3, seed 1234, source at the
    origin.  All 120 columns the contraction needs -- flavours +mu (up) and
    -mu (dn), point sources at y + mu-hat (mu = 0..3) and at y, 12
    spin-colour components each -- solved by the reference's invert_Qtm_her
    to solver_precision 1e-26 (relative residual 1e-13), then Pi_mu_nu(x)
    and the contact term from the reference's program on them.
c3: 24^3x48, kappa 0.155, 2 kappa mu 0.005, eps 0.25, seed 11; the first
    point source of the solver benchmark (ranlxd seed 11), spin-colour 0
    and 7 of the up flavour, solved by invert_Qtm_her to 1e-24; the
    solutions are kept at the source, its 8 neighbours and 2,048 further
    sites (their full volume is 127 MB each), with |x|^2 and the iteration
    counts.
Each solve runs in its own process (the reference keeps one lattice in
globals per process), started with the spawn method.
"""
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import gauge_recipe  # noqa: E402
import oracle_bind as ob  # noqa: E402
from inputs import sample_sites  # noqa: E402

C1 = {"dims": (16, 8, 8, 8), "kappa": 0.150, "two_kappa_mu": 0.01, "eps": 0.3, "seed": 1234,
      "source": 0, "precision": 1e-26}
C3 = {"dims": (48, 24, 24, 24), "kappa": 0.155, "two_kappa_mu": 0.005, "eps": 0.25, "seed": 11,
      "columns": (0, 7), "precision": 1e-24, "nsample": 2048}


def shifted_sites(dims, site):
    """y + mu-hat for mu = 0..3 (periodic), then y (lexicographic indices)."""
    T, LX, LY, LZ = dims
    t, r = divmod(site, LX * LY * LZ)
    x, r = divmod(r, LY * LZ)
    y, z = divmod(r, LZ)
    c, L = [t, x, y, z], [T, LX, LY, LZ]
    out = []
    for m in range(4):
        cc = list(c)
        cc[m] = (cc[m] + 1) % L[m]
        out.append(((cc[0] * LX + cc[1]) * LY + cc[2]) * LZ + cc[3])
    return out + [site]


def _gauge_file(cfg, path):
    g = gauge_recipe.gauge_random(*cfg["dims"], cfg["eps"], cfg["seed"], ob.reference_ranlxd)
    np.save(path, g)
    return g


def _solve_worker(args):
    gauge_path, dims, kappa, mu, site, sc, prec, keep = args
    ref = ob.Reference(*dims, kappa, mu)
    ref.set_gauge(np.load(gauge_path))
    b = np.zeros(24 * ref.V)
    b[24 * site + 2 * sc] = 1.0
    t = time.time()
    n, x = ref.invert(b, prec, 20000, her=True)
    return n, (x if keep is None else x.reshape(-1, 24)[keep].copy()), float(np.dot(x, x)), \
        time.time() - t


def make_c1(workers):
    cfg = C1
    dims, kappa = cfg["dims"], cfg["kappa"]
    mu = cfg["two_kappa_mu"] / (2 * kappa)
    tmp = os.path.join(HERE, "_c1_gauge.npy")
    g = _gauge_file(cfg, tmp)
    jobs = []
    for m in (mu, -mu):
        for s in shifted_sites(dims, cfg["source"]):
            for sc in range(12):
                jobs.append((tmp, dims, kappa, m, s, sc, cfg["precision"], None))
    with mp.get_context("spawn").Pool(workers) as pool:
        res = pool.map(_solve_worker, jobs, chunksize=1)
    os.unlink(tmp)
    its = np.array([r[0] for r in res])
    assert its.min() > 0, its
    fields = [r[1] for r in res]
    conn, _, log = ob.reference_contraction(g, fields, dims, kappa, mu, cfg["source"])
    out = {"pi": conn, "contact": parse_contact(log), "iterations": its,
           "plaquette": np.array(plaquette(g, dims, kappa, mu))}
    out.update({f"cfg_{k}": np.array(v) for k, v in cfg.items()})
    np.savez_compressed(os.path.join(HERE, "reference_c1.npz"), **out)
    print("c1: iterations", its.min(), its.max(), "|Pi|", np.max(np.abs(conn)),
          "solve s", sum(r[3] for r in res))


def make_c3(workers):
    cfg = C3
    dims, kappa = cfg["dims"], cfg["kappa"]
    mu = cfg["two_kappa_mu"] / (2 * kappa)
    T, LX, LY, LZ = dims
    r = ob.reference_ranlxd(4, cfg["seed"])
    c = [int(r[i] * n) for i, n in enumerate(dims)]
    site = ((c[0] * LX + c[1]) * LY + c[2]) * LZ + c[3]
    keep = sample_sites(dims, site, cfg["nsample"])
    tmp = os.path.join(HERE, "_c3_gauge.npy")
    g = _gauge_file(cfg, tmp)
    jobs = [(tmp, dims, kappa, mu, site, sc, cfg["precision"], keep) for sc in cfg["columns"]]
    with mp.get_context("spawn").Pool(min(workers, len(jobs))) as pool:
        res = pool.map(_solve_worker, jobs, chunksize=1)
    os.unlink(tmp)
    out = {"source_site": np.array(site), "sites": keep,
           "iterations": np.array([x[0] for x in res]),
           "x_sites": np.stack([x[1] for x in res]),
           "x_norm2": np.array([x[2] for x in res]),
           "plaquette": np.array(plaquette(g, dims, kappa, mu))}
    assert out["iterations"].min() > 0, out["iterations"]
    out.update({f"cfg_{k}": np.array(v) for k, v in cfg.items()})
    np.savez_compressed(os.path.join(HERE, "reference_c3.npz"), **out)
    print("c3: source", c, "iterations", out["iterations"], "solve s", [x[3] for x in res])


def plaquette(g, dims, kappa, mu):
    ref = ob.Reference(*dims, kappa, mu)
    ref.set_gauge(g)
    return ref.plaquette()


def parse_contact(log):
    lines = log.splitlines()
    i = max(k for k, l in enumerate(lines) if l.startswith("# [cvc_exact2_xspace] contact term"))
    vals = []
    for l in lines[i + 1:i + 5]:
        f = l.split()
        vals += [float(f[1]), float(f[2])]
    return np.array(vals)


if __name__ == "__main__":
    if not ob.reference_available():
        sys.exit("oracle/_ref/libcvcref.so missing: run `make -C oracle ref` first")
    nw = max(1, (os.cpu_count() or 2) - 1)
    for what in sys.argv[1:] or ["c1", "c3"]:
        {"c1": make_c1, "c3": make_c3}[what](nw)
