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


def source_sites(rank, cb):
    T, LX, LY, LZ = DIMS
    r = cb.ranlxd(4 * NSRC, SEED + 1000 * rank)
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


def stencil_traffic_from_profile(key):
    """DRAM bytes per launch of the stencil from the committed ncu summary
    (profiles/*.md lines 'traffic <key> <bytes>'), or None."""
    pdir = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pdir):
        return None
    for fn in sorted(os.listdir(pdir)):
        if not fn.endswith(".md"):
            continue
        for line in open(os.path.join(pdir, fn)):
            f = line.strip().strip("`").split()
            if len(f) == 3 and f[0] == "traffic" and f[1] == key:
                return float(f[2])
    return None


# ---------------------------------------------------------------------------
# reference arm: the reference's own CPU solver (oracle/_ref)
# ---------------------------------------------------------------------------
def _ref_worker(args):
    col, niters, q = args
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_bind as ob
    import cvc_b200 as cb
    ref = ob.Reference(*DIMS, KAPPA, MU)
    ref.set_gauge(cb.gauge_random(*DIMS, EPS, SEED))
    V = ref.V
    b = np.zeros(24 * V)
    b[2 * (col % 12)] = 1.0
    out = []
    for n in niters:
        t = time.perf_counter()
        ref.invert(b, 1e-20, n - 1, her=True)  # runs n BiCGStab iterations (no convergence)
        out.append(time.perf_counter() - t)
    q.put(out)


def reference_iteration_seconds(workers, n_lo=1, n_hi=3):
    """Seconds per invert_Qtm_her iteration per worker process, from two
    bounded runs (n_lo and n_hi iterations) so that set-up cost cancels."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_ref_worker, args=((w, [n_lo, n_hi], q),)) for w in range(workers)]
    for p in procs:
        p.start()
    res = [q.get() for _ in procs]
    for p in procs:
        p.join()
    per = [(r[1] - r[0]) / (n_hi - n_lo) for r in res]
    return max(per), per


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
    ap.add_argument("--block-rhs", type=int, default=0,
                    help="rhs per batch (0: autotuned); pins the batch for profiling runs, "
                         "whose timings would mislead the tuner")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    import cvc_b200 as cb

    if args.impl == "reference":
        if rank != 0:
            return 0
        run_reference_arm(args, cb)
        return 0

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    T, LX, LY, LZ = DIMS
    lat = cb.Lattice(*DIMS, device=local, kappa=KAPPA, mu=MU, bc_angle=(1.0, 0.0, 0.0, 0.0))
    gauge = cb.gauge_random(*DIMS, EPS, SEED)
    lat.upload_gauge(gauge)
    V = lat.VOLUME
    sites = source_sites(rank, cb)
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
    traffic = stencil_traffic_from_profile(traffic_key)

    result = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": {"single": "f32", "half": "f16-storage/f32", "double": "f64"}[args.precision],
        "data": "synthetic",
        "config": {
            "workload": WORKLOAD,
            "lattice": list(DIMS), "rhs_per_gpu": nrhs, "solver": "even/odd CG on M^+M, "
            f"{args.precision} inner iterations, FP64 reliable updates, batched",
            "link_recon": params.link_recon, "parallelism": f"rhs-sharded x{world}",
            "l2": "inputs larger than L2 (96 x 127 MB fields)",
            "rhs_per_batch": nb,
            "stencil_shape": {"sites_per_block": shape[0].value, "rows_per_block": shape[1].value,
                              "rhs_per_thread": shape[2].value,
                              "variant": ["per-thread links", "shared-memory links",
                                          "packed FP32x2 rhs pairs"][shape[3].value]},
            "inner_iterations_per_step": iters // max(args.steps, 1),
            "max_true_residual": worst_res,
        },
        "roofline": {
            "kernel": ["k_eo_hop", "k_eo_hop_staged", "k_eo_hop_x2"][shape[3].value] +
                      " (batched even/odd stencil sweep, "
                      f"{args.precision}, {params.link_recon}-real links)",
            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": (achieved / peak) if achieved else None, "traffic": traffic,
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

    # CPU baseline: the reference's own solver, serial, bounded sample
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            ref_its = result.get("fp64_plain_gpu", {}).get("iterations", [90])
            n_conv = float(np.mean(ref_its))
            sec_it, _ = reference_iteration_seconds(1)
            result["cpu_baseline"] = {
                "value": 1.0 / (sec_it * n_conv), "unit": "solves/s", "cores": 1,
                "kind": "reference",
                "sample": f"2 invert_Qtm_her iterations of the unmodified reference (serial, "
                          f"oracle/_ref) on one 24^3x48 point-source column: {sec_it:.2f} s per "
                          f"iteration, extrapolated to {n_conv:.0f} iterations per solve "
                          "(the count the same algorithm needs on the GPU)"}
        except Exception as e:  # the reference build is absent
            result["cpu_baseline"] = {"value": None, "unit": "solves/s", "cores": 0,
                                      "kind": "reference", "sample": f"unavailable: {e}"}

    if rank == 0:
        print(json.dumps(result), flush=True)
    lat.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def run_reference_arm(args, cb):
    """The reference's CPU solver on all usable host cores: one unmodified
    invert_Qtm_her per worker process on its own column; each step is a
    bounded sample (runs of one and two iterations per worker, whose
    difference is the time of one iteration without the set-up)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_bind as ob
    if not ob.reference_available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/libcvcref.so not built (needs the reference tree at "
                          "build time)"}))
        return
    workers = ref_workers()
    n_conv = 89.0  # iterations of invert_Qtm_her for these columns (FP64 mirror on the GPU)
    times = []
    for i in range(args.warmup + args.steps):
        sec_it, _ = reference_iteration_seconds(workers, 1, 2)
        if i >= args.warmup:
            times.append(sec_it)
    sec_it = float(np.mean(times))
    value = workers / (sec_it * n_conv)
    cores = host_cores()
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s",
        "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": sec_it * 2e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "lattice": list(DIMS),
                   "solver": "reference invert_Qtm_her (BiCGStab on Q^+Q), serial per process",
                   "processes": workers},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": workers, "kind": "reference",
                         "sample": f"{workers} processes x 1 + 2 invert_Qtm_her iterations per step "
                                   f"({sec_it:.2f} s/iteration), extrapolated to {n_conv:.0f} "
                                   f"iterations per solve; host has {cores} cores"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    sys.exit(main())
