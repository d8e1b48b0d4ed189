"""bench.py's reference arm on the CPU: one JSON line with the contract's keys.

`bench.py --impl reference` times the reference's CPU implementation of the path
(the oracle's restatement of its AVX2 scoring, on all host threads) on the same
workload, metric and unit as the GPU arm; here on a small scale so the CPU suite
stays quick.
"""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "2", "--warmup", "1",
                        "--scale", "0.005"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "higher_is_better", "scaling", "vs_baseline",
              "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["unit"] == "GCUPS" and d["higher_is_better"] is True and d["value"] > 0
    assert d["steps"] == 2 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["kind"] in ("port", "reference")
    assert d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert "workload" in d["config"]
    # the arm runs no product code: only the oracle and the input generator are mapped
    assert d["libraries_mapped"], d
    assert all(not x.endswith("libsabertooth_b200.so") for x in d["libraries_mapped"]), d["libraries_mapped"]
    assert "oracle/liboracle.so" in d["libraries_mapped"]
