"""bench.py's reference arm on CPU: one JSON line with the keys the
benchmark contract names (metric, value, unit, impl, config.workload,
cpu_baseline and an e2e block with no host-device traffic).  It times the
oracle's C Dijkstra on the host; no GPU."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.mark.timeout(300)
def test_reference_arm_json_line():
    cmd = [sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--nx", "20", "--ny", "16", "--nz", "4",
           "--sources", "2", "--steps", "2", "--warmup", "3"]
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=280)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    r = json.loads(lines[0])
    assert r["impl"] == "reference"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config"):
        assert k in r, k
    assert r["unit"] == "GTEPS" and r["higher_is_better"] is True and r["value"] > 0
    assert r["steps"] == 2 and r["warmup"] == 3 and r["n_gpus"] == 1
    assert r["config"]["workload"] == "sssp_20x16x4_2src_full"
    cb = r["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] == r["value"]
    assert cb["unit"] == r["unit"] and cb["sample"]
    assert r["e2e"] == {"value": r["value"], "unit": r["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
