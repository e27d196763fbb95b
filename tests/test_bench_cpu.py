"""The bench's reference arm (``bench.py --impl reference``) on the CPU.

The arm times the oracle (the OpenMP transcription of the reference kernel
logic) on a band of rows of the bench scene and prints one JSON line. This
runs it on a tiny scene and checks the line's contract: the metric, a positive
value, the reference label, a CPU baseline describing the run, and an e2e
entry with no host-device copies.
"""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def test_reference_arm_prints_one_json_line():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", OMP_NUM_THREADS="2")
    cmd = [sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--width", "96", "--height", "72",
           "--views", "3", "--steps", "2", "--warmup", "1"]
    res = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, res.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    assert line["metric"].startswith("depth maps/s")
    assert line["unit"] == "depth maps/s" and line["higher_is_better"] is True
    assert line["value"] > 0 and line["steps"] == 2 and line["warmup"] == 1
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"]
    assert "rows" in cb["sample"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
