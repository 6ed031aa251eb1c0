"""bench.py's reference arm on CPU: the oracle port of the path timed on the
host's cores through a persistent spawned worker pool, one JSON line with
the reference-arm keys."""
from __future__ import annotations

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
                        "--warmup", "3", "--frames", "4"], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["steps"] == 2 and line["warmup"] == 3
    assert line["value"] > 0 and line["unit"] == "GB/s" and line["higher_is_better"] is True
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_cpu_pool_steps_repeat():
    sys.path.insert(0, ROOT)
    import bench

    pool = bench.CpuPool(2, 12345, 2)
    try:
        a, b = pool.step(), pool.step()
    finally:
        pool.close()
    assert a["cores"] == b["cores"] == 2
    assert a["value"] > 0 and b["value"] > 0
