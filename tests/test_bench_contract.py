"""The reference arm of bench.py (the CPU restatement on the host cores) prints the bench's JSON
line: run here on a tiny sample and checked key by key.  The GPU arm needs a B200."""
import json
import subprocess
import sys
from pathlib import Path

import oracle_ref as O

ROOT = Path(__file__).resolve().parent.parent


def test_reference_arm_json_line():
    O.build_oracle()
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "0",
                        "--scale", "0.002"], capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "query Mbp/s" and d["unit"] == "Mbp/s"
    assert d["higher_is_better"] is True and d["value"] > 0 and d["steps"] == 1
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] == "port" and cb["cores"] >= 1
    assert cb["cpu_model"] and "queries" in cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
    assert d["config"]["workload"] == "plain"
