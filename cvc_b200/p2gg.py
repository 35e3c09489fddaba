"""P -> gamma gamma three-point function of p2gg_xspace.c, end to end on the GPU.

For one source position y the reference (p2gg_xspace.c:434-585) reads the
forward propagators of both flavours for the point sources at y + mu (mu =
0..3) and at y itself -- 5 x 12 columns each, the conserved current at the
source needs the shifted ones -- builds from every up column the sequential
source on timeslice (t_y + dt) % T (p2gg_xspace.c:525-539), inverts it with
the flavour of g_propagator_position, and contracts the conserved current
(p2gg_xspace.c:615-899, the contraction of cvc_exact2_xspace.c:577-861) with
the up fields replaced by the sequential propagators.  The reference takes
its forward propagators from files and its solves from tmLQCD; here all 180
columns are solved by the batched solver and every field stays in device
memory (torch CUDA tensors).

    python -m cvc_b200.p2gg --dims 64 32 32 32 --kappa 0.156 --mu2k 0.004 \\
        --eps 0.3 --seed 21 --dt 16 --sources 1

prints the solves, their time and Pi's norm.
"""
import argparse
import time

import numpy as np

from .lattice import Lattice, gauge_random, solver_defaults


def shifted_sites(dims, site):
    """Lexicographic indices of y + mu-hat (mu = 0..3, periodic) and of y."""
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


def p2gg(lat, source_site, dt, momentum, gamma_id, propagator_position=0, params=None,
         device="cuda", keep=None):
    """Pi_mu_nu(x) of the P -> gamma gamma three-point function for the source
    at lexicographic site `source_site`; returns (conn, contact, stats) with
    conn the 32*V doubles of the reference layout (a torch CUDA tensor) and
    stats a dict of solve counts and times.  With a dict `keep`, the first
    forward up column ("up0"), its sequential source ("seq_source0") and the
    120 contracted columns ("fields": sequential propagators, then dn) are
    left in it for checks."""
    import torch
    if params is None:
        params = solver_defaults()
    V = lat.VOLUME
    dims = (lat.T, lat.LX, lat.LY, lat.LZ)
    kappa, mu, bc = lat.g_kappa, lat.g_mu, lat.BCangle
    sites = shifted_sites(dims, source_site)
    z = lambda: torch.zeros(24 * V, dtype=torch.float64, device=device)  # noqa: E731
    src = []
    for s in sites:
        for sc in range(12):
            b = z()
            b[24 * s + 2 * sc] = 1.0
            src.append(b)
    up = [z() for _ in range(60)]
    dn = [z() for _ in range(60)]
    stats = {"solves": 0, "solve_s": 0.0, "iterations": 0, "max_true_res": 0.0}

    def solve(xs, bs, m):
        lat.set_params(kappa, m, bc)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st = lat.solve(xs, bs, params)
        torch.cuda.synchronize()
        stats["solve_s"] += time.perf_counter() - t0
        stats["solves"] += len(xs)
        stats["iterations"] += st.iterations
        stats["max_true_res"] = max(stats["max_true_res"], st.max_true_res)
        if st.converged != len(xs):
            raise RuntimeError(f"{len(xs) - st.converged} columns did not converge")

    solve(up, src, mu)
    solve(dn, src, -mu)
    # sequential sources from the up columns (the point sources are not needed
    # any more: their storage takes the sequential sources)
    t_seq = (source_site // (lat.LX * lat.LY * lat.LZ) + dt) % lat.T
    if keep is not None:
        keep["up0"] = up[0].clone()
    for i in range(60):
        lat.p2gg_seq_source(src[i], up[i], t_seq, momentum, gamma_id, propagator_position)
    if keep is not None:
        keep["seq_source0"] = src[0].clone()
        keep["t_seq"] = t_seq
    # the sequential propagators replace the up columns
    solve(up, src, mu if propagator_position == 0 else -mu)
    lat.set_params(kappa, mu, bc)
    del src, b
    torch.cuda.empty_cache()  # the library allocates with cudaMalloc, outside torch's cache
    conn = torch.zeros(32 * V, dtype=torch.float64, device=device)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    conn, contact = lat.cvc_contract(up + dn, source_site, conn=conn)
    torch.cuda.synchronize()
    stats["contract_s"] = time.perf_counter() - t0
    if keep is not None:
        keep["fields"] = up + dn
    return conn, contact, stats


def main(argv=None):
    ap = argparse.ArgumentParser(description="P -> gamma gamma pipeline on one GPU")
    ap.add_argument("--dims", type=int, nargs=4, default=(64, 32, 32, 32),
                    metavar=("T", "LX", "LY", "LZ"))
    ap.add_argument("--kappa", type=float, default=0.156)
    ap.add_argument("--mu2k", type=float, default=0.004, help="2 kappa mu")
    ap.add_argument("--eps", type=float, default=0.3)
    ap.add_argument("--seed", type=int, default=21)
    ap.add_argument("--dt", type=int, default=16)
    ap.add_argument("--sources", type=int, default=1)
    ap.add_argument("--precision", default="single", choices=("double", "single", "half"))
    ap.add_argument("--block-rhs", type=int, default=12)
    a = ap.parse_args(argv)
    import torch
    from . import lattice as _l
    dims = tuple(a.dims)
    V = int(np.prod(dims))
    lat = Lattice(*dims, kappa=a.kappa, mu=a.mu2k / (2 * a.kappa),
                  bc_angle=(1.0, 0.0, 0.0, 0.0))
    lat.upload_gauge(gauge_random(*dims, a.eps, a.seed))
    p = solver_defaults()
    p.precision = {"double": 0, "single": 1, "half": 2}[a.precision]
    p.link_recon = 18 if p.precision == 0 else 12
    p.block_rhs = a.block_rhs
    # source positions: ranlxd stream of the seed, as the solver benchmark does
    r = _l.ranlxd(4 * a.sources, a.seed)
    tot = {"solves": 0, "solve_s": 0.0, "contract_s": 0.0}
    for k in range(a.sources):
        c = [int(r[4 * k + i] * n) % n for i, n in enumerate(dims)]
        site = ((c[0] * dims[1] + c[1]) * dims[2] + c[2]) * dims[3] + c[3]
        conn, contact, st = p2gg(lat, site, a.dt, (0, 0, 0), 5, 0, p)
        for key in tot:
            tot[key] += st[key]
        print(f"source {c}: {st['solves']} solves in {st['solve_s']:.2f} s "
              f"(max true residual {st['max_true_res']:.2e}), contraction {st['contract_s']:.3f} s, "
              f"|Pi| = {float(torch.linalg.norm(conn)):.6e}")
    print(f"total: {tot['solves']} solves, {tot['solves'] / tot['solve_s']:.1f} solves/s, "
          f"contraction {tot['contract_s'] / a.sources:.3f} s per source, V = {V}")
    lat.close()


if __name__ == "__main__":
    main()
