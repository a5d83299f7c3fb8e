"""bench.py's reference arm on the host (no GPU): one JSON line carrying the
metric, unit and config of the GPU arm, with the CPU timing described in
cpu_baseline and an e2e block that moves no bytes.  The timed steps are
real: steps x ms_per_step fits inside the process's wall time, and the
value is the pair fraction those steps cover over that time."""
import json
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    t0 = time.perf_counter()
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
                          "--warmup", "0"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    wall = time.perf_counter() - t0
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "3D transform pairs/s at lmax=511 nr=256" and d["unit"] == "pairs/s"
    assert d["value"] > 0 and d["higher_is_better"] is True
    assert d["config"]["lmax"] == 511 and d["config"]["nz"] == 256 and d["config"]["fields"] == 4
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["steps"] == 2 and d["steps"] * d["ms_per_step"] * 1e-3 < wall
    sys.path.insert(0, ROOT)
    import bench
    assert abs(d["value"] - (2 / bench.PAIR_SLICES) / (2 * d["ms_per_step"] * 1e-3)) < 1e-9 * d["value"]
