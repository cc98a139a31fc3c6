"""The reference arm of bench.py: the reference's own CPU solver (or its CPU
restatement when that build is absent) timed on a bounded sample of the
workload.  It needs no GPU, so it runs here on a 64^3 band sample and must
print one JSON line with the keys the benchmark contract names, the GPU arm's
metric and unit, and no host-device traffic."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "3",
           "--cpu-sample-n", "64"]
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [line for line in out.stdout.splitlines() if line.startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference"
    assert rec["metric"].startswith("MGPCG time & MDOF/s") and rec["unit"] == "MDOF/s"
    assert rec["higher_is_better"] is True and rec["steps"] == 1 and rec["warmup"] == 3
    assert rec["value"] > 0 and rec["ms_per_step"] > 0
    assert rec["config"]["workload"] == "spheres_band64" and rec["config"]["sample_of"] == "spheres_band1024"
    cb = rec["cpu_baseline"]
    assert cb["value"] == rec["value"] and cb["kind"] in ("reference", "port") and cb["cores"] >= 1
    assert "spheres_band64" in cb["sample"]
    e2e = rec["e2e"]
    assert e2e["value"] == rec["value"] and e2e["unit"] == rec["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
