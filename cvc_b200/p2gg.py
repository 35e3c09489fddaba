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

from . import _lib
from .lattice import CvcbError, Lattice, gauge_random, solver_defaults


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
    conn = torch.zeros(32 * V, dtype=torch.float64, device=device)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    try:
        conn, contact = lat.cvc_contract(up + dn, source_site, conn=conn)
    except CvcbError as e:
        # the contraction's buffers are allocated by the library (cudaMalloc,
        # outside torch's cache): give it the memory of the sources that
        # torch still caches, and try once more
        if e.code != _lib.CVCB_ERR_NOMEM:
            raise
        torch.cuda.empty_cache()
        conn, contact = lat.cvc_contract(up + dn, source_site, conn=conn)
    torch.cuda.synchronize()
    stats["contract_s"] = time.perf_counter() - t0
    if keep is not None:
        keep["fields"] = up + dn
    return conn, contact, stats


def source_positions(dims, n, seed):
    """n source positions (lexicographic) from the ranlxd stream of `seed`,
    4 numbers per position scaled to (T, LX, LY, LZ), as the benchmarks do."""
    from . import lattice as _l
    r = _l.ranlxd(4 * n, seed)
    out = []
    for k in range(n):
        c = [int(r[4 * k + i] * m) % m for i, m in enumerate(dims)]
        out.append(((c[0] * dims[1] + c[1]) * dims[2] + c[2]) * dims[3] + c[3])
    return out


def run_sources(sources, make_gauge, compute, n_gauge, device=None, group=None):
    """The multi-source P -> gamma gamma run on one or several ranks (one
    process per GPU): rank 0 makes the gauge field and broadcasts it (one
    collective, before any solve), every rank takes its round-robin share of
    the source positions, and Pi of all sources is gathered on every rank.
    compute(gauge, source) -> (conn, contact) tensors on `device`; returns
    (conn [n_sources, 32 V], contact [n_sources, 8])."""
    from . import sharding
    world, rank = sharding.world_rank(group)
    gauge = sharding.broadcast_field(make_gauge() if rank == 0 else None, n_gauge, device, group)
    return sharding.pi_sharded(sources, lambda s: compute(gauge, s), group)


def main(argv=None):
    ap = argparse.ArgumentParser(description="P -> gamma gamma pipeline, one process per GPU "
                                             "(under torchrun for several GPUs)")
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
    import os
    import torch
    import torch.distributed as dist
    from . import sharding
    dims = tuple(a.dims)
    V = int(np.prod(dims))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=device)
    lat = Lattice(*dims, device=local, kappa=a.kappa, mu=a.mu2k / (2 * a.kappa),
                  bc_angle=(1.0, 0.0, 0.0, 0.0))
    p = solver_defaults()
    p.precision = {"double": 0, "single": 1, "half": 2}[a.precision]
    p.link_recon = 18 if p.precision == 0 else 12
    p.block_rhs = a.block_rhs
    sources = source_positions(dims, a.sources, a.seed)
    tot = {"solves": 0, "solve_s": 0.0, "contract_s": 0.0}
    uploaded = []

    def compute(gauge, site):
        if not uploaded:
            lat.upload_gauge(gauge)
            uploaded.append(True)
        conn, contact, st = p2gg(lat, site, a.dt, (0, 0, 0), 5, 0, p, device=device)
        for key in tot:
            tot[key] += st[key]
        print(f"[rank {sharding.world_rank()[1]}] source {site}: {st['solves']} solves in "
              f"{st['solve_s']:.2f} s (max true residual {st['max_true_res']:.2e}), contraction "
              f"{st['contract_s']:.3f} s", flush=True)
        return conn, torch.as_tensor(contact, device=device)

    conn, contact = run_sources(sources, lambda: gauge_random(*dims, a.eps, a.seed), compute,
                                72 * V, device)
    solve_s = sharding.max_over_ranks(tot["solve_s"], device)
    if sharding.world_rank()[1] == 0:
        for k, s in enumerate(sources):
            print(f"source {s}: |Pi| = {float(torch.linalg.norm(conn[k])):.6e}")
        n = 180 * len(sources)
        print(f"total: {n} solves on {world} GPU(s), {n / solve_s:.1f} solves/s (slowest rank), "
              f"V = {V}")
    lat.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
