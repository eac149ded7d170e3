"""The bench's reference arm on CPU: one JSON line with the contract's keys,
timing the reference's own compiled engine (or the oracle port where it is
not built) on a bounded sample of the workload."""
import json
import os
import subprocess
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    cmd = [sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference",
           "--workload", "fodo", "--steps", "2", "--warmup", "1",
           "--ref-step-seconds", "0.3", "--no-reference-gpu"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=REPO,
                         env=dict(os.environ, OMP_NUM_THREADS="2"))
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["steps"] == 2
    assert d["unit"] == "particle-turns/s" and d["higher_is_better"] is True
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    assert "FODO" in d["config"]["workload"]
