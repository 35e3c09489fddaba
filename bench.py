"""Benchmark: propagator solves/s of the batched mixed-precision solver on
the 24^3x48 twisted-mass workload, against the plain FP64 solver and the
reference's CPU implementation.

Workload (one step): 8 point-source positions x 12 spin-colour columns = 96
right-hand sides on a 24^3x48 lattice, kappa = 0.155, 2 kappa mu = 0.005,
gauge U = exp(i 0.25 H) from ranlxd seed 11, periodic in space and
antiperiodic in time (BCangleT = 1).  Each solve is brought to a true FP64
residual |b - Q x| / |b| <= 1e-10, checked with the full FP64 operator.
Source positions: ranlxd (level 1) seed 11 + 1000*rank, 4 numbers per
position scaled to (T, LX, LY, LZ).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--precision single|half|double]

With --gpus N > 1 it must run under torchrun (one rank per GPU); each rank
solves its own 96 columns (weak scaling) and the step time is the maximum
over ranks.  Prints one JSON line on rank 0.
"""
import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "propagator solves/s & Dslash HBM GB/s, mixed+batched vs FP64, at 1e-10 resid"
DIMS = (48, 24, 24, 24)
KAPPA = 0.155
MU = 0.005 / (2 * KAPPA)
EPS, SEED = 0.25, 11
NSRC, TOL = 8, 1e-10
# the P -> gamma gamma configuration: 32^3x64, kappa 0.156, 2 kappa mu 0.004,
# eps 0.3 gauge field (seed 21), sequential source at separation 16
C5_DIMS, C5_KAPPA, C5_MU2K, C5_EPS, C5_SEED, C5_DT = (64, 32, 32, 32), 0.156, 0.004, 0.3, 21, 16
WORKLOAD = ("24^3x48 twisted-mass Wilson, kappa 0.155, 2*kappa*mu 0.005, eps 0.25 gauge "
            "(ranlxd seed 11), 8 point sources x 12 spin-colour = 96 rhs per GPU, "
            "true FP64 residual <= 1e-10")
FALLBACK_HBM_GBS = 6650.0


def measured_hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def source_sites(rank, ranlxd):
    """Lexicographic indices of the rank's point sources; `ranlxd(n, seed)`
    is the library's generator or the reference's own (the same stream)."""
    T, LX, LY, LZ = DIMS
    r = ranlxd(4 * NSRC, SEED + 1000 * rank)
    sites = []
    for k in range(NSRC):
        t, x, y, z = (int(r[4 * k] * T), int(r[4 * k + 1] * LX), int(r[4 * k + 2] * LY),
                      int(r[4 * k + 3] * LZ))
        sites.append(((t * LX + x) * LY + y) * LZ + z)
    return sites


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        try:
            self.file.flush()
            rows = [l.split(",") for l in open(self.file.name).read().splitlines() if l.strip()]
        except Exception:
            rows = []
        os.unlink(self.file.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4)
                          if len(r) > 5 + i and r[5 + i].strip().lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def stencil_traffic_ratio(key):
    """DRAM bytes over algorithmic bytes of the stencil from the committed ncu
    summary of the same kernel and batch (profiles/*.md lines
    'traffic_ratio <key> <ratio>'), or None."""
    pdir = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pdir):
        return None
    for fn in sorted(os.listdir(pdir)):
        if not fn.endswith(".md"):
            continue
        for line in open(os.path.join(pdir, fn)):
            f = line.strip().strip("`").split()
            if len(f) == 3 and f[0] == "traffic_ratio" and f[1] == key:
                return float(f[2])
    return None


# ---------------------------------------------------------------------------
# The reference's own CPU solver (oracle/_ref), for the reference arm and the
# cpu_baseline leg.  Its inputs are built without the CUDA library: the gauge
# field by the numpy restatement of the recipe (oracle/gauge_recipe.py) over
# the reference's own ranlxd, the source positions from the same stream as
# the GPU arm's.
# ---------------------------------------------------------------------------
def _ref_worker(gauge_path, cmd_q, res_q, wid):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_bind as ob
    ref = ob.Reference(*DIMS, KAPPA, MU)
    ref.set_gauge(np.load(gauge_path))
    V = ref.V
    res_q.put((wid, "ready", 0.0))
    while True:
        cmd = cmd_q.get()
        if cmd is None:
            return
        site, sc, nmax = cmd
        b = np.zeros(24 * V)
        b[24 * site + 2 * sc] = 1.0
        t = time.perf_counter()
        rc, _ = ref.invert(b, TOL * TOL, nmax, her=True)
        res_q.put((wid, rc, time.perf_counter() - t))


class ReferencePool:
    """`workers` processes, each holding one unmodified reference instance
    (its globals: one lattice per process) on the benchmark's gauge field.
    Started with the spawn method, before any GPU work of this process."""

    def __init__(self, workers):
        import multiprocessing as mp
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle_bind as ob
        import gauge_recipe
        self.workers = workers
        self.sites = source_sites(0, ob.reference_ranlxd)
        gauge = gauge_recipe.gauge_random(*DIMS, EPS, SEED, ob.reference_ranlxd)
        self.tmp = tempfile.NamedTemporaryFile(suffix=".npy", delete=False)
        np.save(self.tmp, gauge)
        self.tmp.close()
        del gauge
        ctx = mp.get_context("spawn")
        self.res = ctx.Queue()
        self.cmds = [ctx.Queue() for _ in range(workers)]
        self.procs = [ctx.Process(target=_ref_worker, args=(self.tmp.name, self.cmds[w], self.res, w))
                      for w in range(workers)]
        for p in self.procs:
            p.start()
        for _ in range(workers):
            self.res.get()
        os.unlink(self.tmp.name)

    def column(self, w):
        """Worker w's column: source position w // 12 (mod the 8), spin-colour w % 12."""
        return self.sites[(w // 12) % NSRC], w % 12

    def run(self, nmax):
        """Every worker runs invert_Qtm_her on its own column with niter_max =
        nmax; returns (wall seconds of the whole round, [(rc, seconds)])."""
        t = time.perf_counter()
        for w in range(self.workers):
            self.cmds[w].put((*self.column(w), nmax))
        out = [None] * self.workers
        for _ in range(self.workers):
            w, rc, dt = self.res.get()
            out[w] = (rc, dt)
        return time.perf_counter() - t, out

    def close(self):
        for q in self.cmds:
            q.put(None)
        for p in self.procs:
            p.join()


def reference_rate(pool, warmup, steps, n_conv=None):
    """Reference solves/s on the pool.  The iteration count to convergence
    is measured (every worker solves its column to the benchmark's residual)
    unless given.  A run with niter_max = n costs (n + 1 + c) iterations,
    c the fixed part (the initial residual and the final Qf5); c comes from
    runs of 1 and 3 iterations, after which each step is one bounded round
    of 1 iteration per worker."""
    full = None
    if n_conv is None:
        wall, res = pool.run(20000)
        its = [rc for rc, _ in res]
        if min(its) < 0:
            raise RuntimeError(f"reference solve did not converge: {its}")
        n_conv = float(np.mean(its))
        full = {"iterations": its, "wall_s": wall,
                "solves_per_s": pool.workers / max(dt for _, dt in res)}
    _, r1 = pool.run(0)
    _, r3 = pool.run(2)
    t1 = max(dt for _, dt in r1)
    t3 = max(dt for _, dt in r3)
    t_it = (t3 - t1) / 2
    c = max(t1 / t_it - 1.0, 0.0)
    times, walls = [], []
    for i in range(warmup + steps):
        wall, r = pool.run(0)
        if i >= warmup:
            times.append(max(dt for _, dt in r) / (1.0 + c))
            walls.append(wall)
    sec_it = float(np.mean(times))
    return {"value": pool.workers / (sec_it * n_conv), "sec_per_iteration": sec_it,
            "n_conv": n_conv, "fixed_iterations": c, "step_wall_s": walls, "full": full}


def workload_config(world):
    """The workload, identical in both arms (implementation details go
    elsewhere in the line)."""
    return {"workload": WORKLOAD, "lattice": list(DIMS), "kappa": KAPPA, "two_kappa_mu": 0.005,
            "gauge": {"eps": EPS, "seed": SEED}, "rhs_per_gpu": NSRC * 12,
            "true_residual": TOL, "parallelism": f"rhs-sharded x{world}",
            "l2": "inputs larger than L2 (96 x 127 MB fields)"}


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def ref_workers():
    cores = host_cores()
    try:
        avail = int([l for l in open("/proc/meminfo") if l.startswith("MemAvailable")][0].split()[1])
        by_mem = max(1, int(avail * 1024 / 2.5e9))  # ~1.6 GB per 24^3x48 reference process
    except Exception:
        by_mem = 8
    return max(1, min(cores, by_mem, 64))


# ---------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="single", choices=["single", "half", "double"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fp64", action="store_true",
                    help="skip the plain FP64 GPU solver comparison")
    ap.add_argument("--no-c5", action="store_true",
                    help="skip the P->gamma gamma pipeline at 32^3x64")
    ap.add_argument("--ref-niter", type=int, default=0,
                    help="reference arm: iterations per solve given instead of measured "
                         "(0: measured by solving every worker's column first)")
    ap.add_argument("--block-rhs", type=int, default=0,
                    help="rhs per batch (0: autotuned); pins the batch for profiling runs, "
                         "whose timings would mislead the tuner")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        run_reference_arm(args)
        return 0

    import cvc_b200 as cb

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    T, LX, LY, LZ = DIMS
    from cvc_b200 import sharding
    lat = cb.Lattice(*DIMS, device=local, kappa=KAPPA, mu=MU, bc_angle=(1.0, 0.0, 0.0, 0.0))
    # the gauge field is made on rank 0 and broadcast (one collective, untimed)
    gauge = sharding.broadcast_field(cb.gauge_random(*DIMS, EPS, SEED) if rank == 0 else None,
                                     72 * T * LX * LY * LZ, torch.device("cuda", local))
    lat.upload_gauge(gauge)
    V = lat.VOLUME
    sites = source_sites(rank, cb.ranlxd)
    nrhs = NSRC * 12
    prec = {"single": cb.PREC_SINGLE, "half": cb.PREC_HALF, "double": cb.PREC_DOUBLE}[args.precision]
    params = cb.solver_defaults()
    params.precision, params.tol = prec, TOL
    params.link_recon = 18 if prec == cb.PREC_DOUBLE else 12
    params.block_rhs = args.block_rhs

    # device-resident inputs (point sources) and outputs
    dev = torch.device("cuda", local)
    bs = []
    for s in sites:
        for sc in range(12):
            b = torch.zeros(24 * V, dtype=torch.float64, device=dev)
            b[24 * s + 2 * sc] = 1.0
            bs.append(b)
    xs = [torch.zeros(24 * V, dtype=torch.float64, device=dev) for _ in range(nrhs)]
    torch.cuda.synchronize()

    def step():
        st = lat.solve(xs, bs, params)
        if st.converged != nrhs:
            raise RuntimeError(f"only {st.converged}/{nrhs} converged (max res {st.max_true_res})")
        return st

    for _ in range(args.warmup):
        step()
    # timed region
    stream = torch.cuda.current_stream()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    lat._lib.cvcb_profile(lat._h, 1)
    n0 = ctypes.c_longlong()
    lat._lib.cvcb_counters(lat._h, ctypes.byref(n0), None, None, None)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    worst_res, iters, nb = 0.0, 0, 12
    with Clocks(local) as clk:
        e0.record(stream)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            st = step()
            worst_res = max(worst_res, st.max_true_res)
            iters += st.iterations
            nb = st.batch_rhs
        e1.record(stream)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    if world > 1:
        dist.barrier()
    ms_total = e0.elapsed_time(e1)
    # the library works on its own stream and synchronises before returning,
    # so the events on torch's stream bracket the whole solve; take the larger
    ms_total = max(ms_total, wall * 1e3)
    n1, pl = ctypes.c_longlong(), ctypes.c_longlong()
    pms, pbytes = ctypes.c_double(), ctypes.c_double()
    lat._lib.cvcb_counters(lat._h, ctypes.byref(n1), ctypes.byref(pl), ctypes.byref(pms),
                           ctypes.byref(pbytes))
    lat._lib.cvcb_profile(lat._h, 0)
    ms_step = ms_total / args.steps
    if world > 1:
        t = torch.tensor([ms_step], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_step = float(t.item())
    value = world * nrhs / (ms_step / 1e3)

    # dominant kernel: the batched stencil, timed live inside the region above
    peak, peak_kind = measured_hbm_peak()
    stencil_avg_ms = pms.value / max(pl.value, 1)
    stencil_bytes = pbytes.value / max(pl.value, 1)
    achieved = stencil_bytes / (stencil_avg_ms * 1e-3) / 1e9 if pl.value else None
    shape = [ctypes.c_int() for _ in range(4)]
    lat._lib.cvcb_tuned_shape(lat._h, prec, params.link_recon, nb, *[ctypes.byref(v) for v in shape])
    traffic_key = f"{args.precision}-{params.link_recon}-n{nb}-{T}x{LX}x{LY}x{LZ}"
    ratio = stencil_traffic_ratio(traffic_key)
    traffic = ratio * stencil_bytes if ratio and pl.value else None

    result = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": {"single": "f32", "half": "f16-storage/f32", "double": "f64"}[args.precision],
        "data": "synthetic",
        "config": workload_config(world),
        "run": {
            "solver": "even/odd CG on M^+M, "
            f"{args.precision} inner iterations, FP64 reliable updates, batched",
            "link_recon": params.link_recon, "rhs_per_batch": nb,
            "stencil_shape": {"sites_per_block": shape[0].value, "rows_per_block": shape[1].value,
                              "rhs_per_thread": shape[2].value,
                              "variant": ["per-thread links", "shared-memory links",
                                          "packed FP32x2 rhs pairs", "pair-tiled fields",
                                          "pair-tiled fields, TMEM accumulator",
                                          "pair-tiled fields, TMEM accumulator, pipelined",
                                          "pair-tiled fields, bulk-staged t/x neighbours"]
                                         [shape[3].value]},
            "inner_iterations_per_step": iters // max(args.steps, 1),
            "max_true_residual": worst_res,
        },
        "roofline": {
            "kernel": ["k_eo_hop", "k_eo_hop_staged", "k_eo_hop_x2", "k_eo_hop_pt",
                       "k_eo_hop_ptm", "k_eo_hop_ptm", "k_eo_hop_ptb"][shape[3].value] +
                      " (batched even/odd stencil sweep, "
                      f"{args.precision}, {params.link_recon}-real links)",
            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": (achieved / peak) if achieved else None, "traffic": traffic,
            "traffic_source": "DRAM bytes / algorithmic bytes of the same kernel from its ncu "
                              "capture (profiles/), times this run's algorithmic bytes per launch"
                              if traffic else None,
            "peak_source": peak_kind, "launches_timed": pl.value,
            "avg_launch_ms": stencil_avg_ms, "algorithmic_bytes_per_launch": stencil_bytes,
        },
        "gpu_launches": int(n1.value - n0.value),
    }
    result["clocks"] = clk.summary()

    # plain FP64 GPU solver (the reference's algorithm, invert_Qtm_her) on 12 columns
    if rank == 0 and not args.no_fp64:
        xh = np.zeros(24 * V)
        t = time.perf_counter()
        its = []
        for sc in range(12):
            b = np.zeros(24 * V)
            b[24 * sites[0] + 2 * sc] = 1.0
            xh[:] = 0
            n, tr = lat.invert_Qtm_her(xh, b, TOL * TOL, 20000, return_residual=True)
            its.append(n)
        dt = time.perf_counter() - t
        result["fp64_plain_gpu"] = {"value": 12 / dt, "unit": "solves/s",
                                    "algorithm": "BiCGStab on Q^+Q (invert_Qtm_her), FP64",
                                    "iterations": its}
        result["speedup_vs_fp64_plain_gpu"] = value / world / (12 / dt)

    # end to end through the public API with host buffers
    if not args.no_e2e:
        pin_b = [torch.zeros(24 * V, dtype=torch.float64).pin_memory() for _ in range(nrhs)]
        for k, s in enumerate(sites):
            for sc in range(12):
                pin_b[12 * k + sc][24 * s + 2 * sc] = 1.0
        pin_x = [torch.zeros(24 * V, dtype=torch.float64).pin_memory() for _ in range(nrhs)]
        # one untimed call sets up the pipeline's staging buffers and stream
        st = lat.solve(pin_x, pin_b, params)
        assert st.converged == nrhs
        ke = max(1, args.steps)
        if world > 1:
            dist.barrier()
        t = time.perf_counter()
        for _ in range(ke):
            st = lat.solve(pin_x, pin_b, params)
            assert st.converged == nrhs
        dt = (time.perf_counter() - t) / ke
        if world > 1:
            tt = torch.tensor([dt], device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            dt = float(tt.item())
        result["e2e"] = {"value": world * nrhs / dt, "unit": "solves/s",
                         "h2d_bytes_per_step": nrhs * 24 * V * 8,
                         "d2h_bytes_per_step": nrhs * 24 * V * 8,
                         "steps": ke,
                         "note": "host pinned buffers through cvcb_solve (copies overlap the "
                                 "solve on a second stream); copies and the CVC<->device layout "
                                 "transforms inside the timed region"}
        del pin_b, pin_x

    # CPU baseline: the reference's own solver on one host core, bounded sample
    if rank == 0 and world == 1 and not args.no_cpu:
        result["cpu_baseline"] = cpu_baseline_leg(result)

    del xs, bs
    lat.close()
    if rank == 0 and world == 1 and not args.no_c5:
        torch.cuda.empty_cache()
        try:
            result["p2gg_c5"] = p2gg_c5_leg(local)
        except Exception as e:  # an extra figure: its failure must not cost the headline line
            result["p2gg_c5"] = {"unavailable": f"{type(e).__name__}: {e}"[:300]}
            torch.cuda.empty_cache()

    if rank == 0:
        print(json.dumps(result), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def p2gg_c5_leg(local):
    """The P -> gamma gamma pipeline of the 32^3x64 configuration for the
    first of its four source positions (cvc_b200.p2gg, p2gg_xspace.c:434-899):
    180 batched mixed-precision solves (both flavours at the source and its
    four forward neighbours, then the 60 sequential propagators), the
    sequential sources and the conserved-current contraction, all fields in
    device memory.  A first pass tunes the solver for this volume; the second
    is timed (CUDA-synchronised wall time of the whole pipeline)."""
    import torch
    import cvc_b200 as cb
    from cvc_b200 import p2gg as pg
    lat = cb.Lattice(*C5_DIMS, device=local, kappa=C5_KAPPA, mu=C5_MU2K / (2 * C5_KAPPA),
                     bc_angle=(1.0, 0.0, 0.0, 0.0))
    lat.upload_gauge(cb.gauge_random(*C5_DIMS, C5_EPS, C5_SEED))
    p = cb.solver_defaults()
    p.precision, p.link_recon, p.tol = cb.PREC_SINGLE, 12, TOL
    site = pg.source_positions(C5_DIMS, 4, C5_SEED)[0]
    dev = torch.device("cuda", local)
    out = {}
    for rep in range(2):
        torch.cuda.synchronize()
        t = time.perf_counter()
        conn, contact, st = pg.p2gg(lat, site, C5_DT, (0, 0, 0), 5, 0, p, device=dev)
        torch.cuda.synchronize()
        total = time.perf_counter() - t
        out = {"value": st["solves"] / st["solve_s"], "unit": "solves/s",
               "seconds_per_source": total, "solves_per_source": st["solves"],
               "solve_s": st["solve_s"], "contract_s": st["contract_s"],
               "inner_iterations": st["iterations"], "max_true_residual": st["max_true_res"],
               "pi_norm": float(torch.linalg.norm(conn)),
               "workload": "32^3x64 P->gamma gamma, kappa 0.156, 2*kappa*mu 0.004, eps 0.3 "
                           f"(ranlxd seed 21), source site {site}, sequential source at dt "
                           f"{C5_DT}, FP32 inner iterations, true FP64 residual <= 1e-10",
               "passes": rep + 1}
        del conn
    lat.close()
    torch.cuda.empty_cache()
    return out


def cpu_baseline_leg(result):
    """The unmodified reference invert_Qtm_her on one host core, a bounded
    sample (runs of 1, 3 and 1 iterations on one column), extrapolated to
    the iteration count that the same algorithm needed on the GPU."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_bind as ob
    if not ob.reference_available():
        return {"value": None, "unit": "solves/s", "cores": 0, "kind": "reference",
                "sample": "unavailable: oracle/_ref/libcvcref.so not built"}
    its = result.get("fp64_plain_gpu", {}).get("iterations")
    pool = ReferencePool(1)
    try:
        r = reference_rate(pool, 0, 1, n_conv=float(np.mean(its)) if its else None)
    finally:
        pool.close()
    return {"value": r["value"], "unit": "solves/s", "cores": 1, "kind": "reference",
            "sample": f"unmodified invert_Qtm_her (oracle/_ref, serial) on one 24^3x48 "
                      f"point-source column: bounded runs of 1, 3 and 1 iterations, "
                      f"{r['sec_per_iteration']:.2f} s per iteration, extrapolated to "
                      f"{r['n_conv']:.1f} iterations per solve "
                      + ("(the count the same algorithm needed on the GPU)" if its else
                         "(measured to convergence)")}


def run_reference_arm(args):
    """The reference's CPU solver on all usable host cores: one unmodified
    invert_Qtm_her per worker process, each on its own column of the
    workload.  Before the steps every worker solves its column to the
    benchmark's residual, which measures the iteration count; each step is
    then one bounded round (1 iteration per worker), and the rate is
    workers / (seconds per iteration x iterations to convergence)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_bind as ob
    if not ob.reference_available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/libcvcref.so not built (needs the reference tree at "
                          "build time)"}))
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    workers = ref_workers()
    cores = host_cores()
    t_start = time.perf_counter()
    pool = ReferencePool(workers)
    try:
        r = reference_rate(pool, args.warmup, args.steps,
                           n_conv=float(args.ref_niter) if args.ref_niter else None)
    finally:
        pool.close()
    value = r["value"]
    ms_step = 1e3 * float(np.mean(r["step_wall_s"]))
    how = ("measured: every worker solved its column to the benchmark's residual first"
           if r["full"] else "given by --ref-niter")
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(world),
        "run": {"solver": "reference invert_Qtm_her (BiCGStab on Q^+Q), serial per process",
                "processes": workers, "iterations_to_convergence": r["n_conv"],
                "iteration_count": how, "fixed_iterations_per_call": r["fixed_iterations"],
                "sec_per_iteration": r["sec_per_iteration"], "full_solves": r["full"],
                "total_s": time.perf_counter() - t_start},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": workers, "kind": "reference",
                         "sample": f"{workers} processes, each step one round of 1 "
                                   f"invert_Qtm_her iteration per process "
                                   f"({r['sec_per_iteration']:.2f} s per iteration), "
                                   f"{r['n_conv']:.1f} iterations per solve ({how}); "
                                   f"host has {cores} cores"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    sys.exit(main())
