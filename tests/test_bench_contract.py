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
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "2", "--warmup", "0",
                        "--scale", "0.002"], capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "query Mbp/s" and d["unit"] == "Mbp/s"
    assert d["higher_is_better"] is True and d["value"] > 0 and d["steps"] == 2
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] == "port" and cb["cores"] >= 1
    assert cb["cpu_model"] and "queries" in cb["sample"]
    assert cb["spread"]["min"] <= d["value"] <= cb["spread"]["max"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
    # the default workload is the learned-schedule configuration, keys as in the GPU arm's line
    cfg = d["config"]
    assert cfg["workload"] == "batched" and cfg["schedule"] == "learned" and cfg["pipeline"] == "batched"
    assert cfg["chunks"] == 40 and cfg["chunks_per_step"] == 40 and cfg["word_size"] == 11


def test_bench_parity_witness_and_steps():
    """The bench's own host logic: step batches cycle through the workload, and the parity witness
    picks the sampled queries' lines out of the GPU text by qseqid."""
    import bench
    a = bench.parse(["--steps", "20", "--warmup", "5"])
    assert a.workload == "batched" and a.schedule == "learned" and a.pipeline == "batched"
    nb = 20
    timed = [(a.warmup + k) % nb for k in range(a.steps)]
    assert sorted(timed) == list(range(nb))  # 20 timed steps are the whole query set once
    gpu = "10\t1.0\tchunk1\t1\t2\tcons0\t1\t2\n20\t2.0\tchunk2\t1\t2\tcons0\t1\t2\n"
    w = bench.parity_witness(gpu, "10\t1.0\tchunk1\t1\t2\tcons0\t1\t2\n", ["chunk1"])
    assert w["identical"] and w["lines"] == 1
    assert not bench.parity_witness(gpu, "", ["chunk1"])["identical"]
