"""The bench's CPU legs (the reference arm and the CPU baselines) run on the
host without a GPU: a small window of each workload through the oracle."""

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_split_cpu_leg_small_window():
    sys.path.insert(0, ROOT)
    import bench
    out = bench.split_cpu_leg(8, window=6, steps=1)
    assert out["value"] > 0 and out["kind"] == "port" and out["unit"] == "cell-steps/s"


def test_reference_arm_prints_one_json_line():
    env = dict(os.environ, RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0", "--cpu-window", "6", "--nz", "8"], capture_output=True, text=True,
                       cwd=ROOT, env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] == "port"
