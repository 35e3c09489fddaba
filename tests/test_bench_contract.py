"""The reference arm of bench.py on the host cores: one JSON line with the
metric, unit and workload config of the GPU arm, a cpu_baseline describing
the sample, and an e2e entry without host-device traffic (the reference's
CPU solver, compiled from its own sources, times a bounded sample).  The
iteration count to convergence is given here (--ref-niter), because solving
a 24^3x48 column to convergence on the reference takes minutes; the
benchmark run measures it."""
import json
import os
import subprocess
import sys

from conftest import ROOT


def test_reference_arm_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "0", "--ref-niter", "89"],
                         capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    if "unavailable" in d:  # the compiled reference needs the reference tree at build time
        return
    sys.path.insert(0, ROOT)
    import bench
    assert d["metric"] == bench.METRIC and d["unit"] == "solves/s"
    assert d["higher_is_better"] is True and d["steps"] == 1 and d["warmup"] == 0
    # the same workload description as the GPU arm's line
    assert d["config"] == json.loads(json.dumps(bench.workload_config(1)))
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["run"]["iterations_to_convergence"] == 89.0
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == d["value"] and cb["cores"] >= 1
    assert cb["unit"] == d["unit"] and cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_loads_no_cuda_library():
    """The reference arm builds its inputs with the reference's ranlxd and
    the numpy gauge recipe; the CUDA library is never mapped."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_bind as ob
    if not ob.reference_available():
        import pytest
        pytest.skip("the compiled reference needs the reference tree at build time")
    code = ("import sys, os; sys.argv=['bench.py']; sys.path.insert(0, %r); import bench; "
            "sys.path.insert(0, os.path.join(%r, 'tests')); "
            "sys.path.insert(0, os.path.join(%r, 'oracle')); import oracle_bind as ob, "
            "gauge_recipe as gr; "
            "s = bench.source_sites(0, ob.reference_ranlxd); "
            "g = gr.gauge_random(4, 4, 4, 4, 0.25, 11, ob.reference_ranlxd); "
            "maps = open('/proc/self/maps').read(); "
            "print('LOADED' if 'libcvcb200' in maps else 'CLEAN', len(s))") % (ROOT, ROOT, ROOT)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    assert out.stdout.split() == ["CLEAN", "8"]
