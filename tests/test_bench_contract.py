"""The reference arm of bench.py on the host cores: one JSON line with the
metric, unit and workload of the GPU arm, a cpu_baseline describing the
sample, and an e2e entry without host-device traffic (the reference's CPU
solver, compiled from its own sources, times a bounded sample)."""
import json
import os
import subprocess
import sys

from conftest import ROOT


def test_reference_arm_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "0"], capture_output=True, text=True,
                         timeout=900, cwd=ROOT)
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
    assert d["config"]["workload"] == bench.WORKLOAD
    assert d["config"]["lattice"] == list(bench.DIMS)
    assert d["value"] > 0
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == d["value"] and cb["cores"] >= 1
    assert cb["unit"] == d["unit"] and cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
