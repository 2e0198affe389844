"""The preliminary-DP thread body of k_prelim_stream, built for the host, against the oracle.

rmb_prelim_stream.cuh holds the per-thread loop the GPU kernel runs (band ring, row ends, record
queue, origin moves); tests/stream_host.cu compiles it as host code with nvcc and compares every
record it completes with the oracle's score-only extension (search/gapped.rs:124-337), cells
included.  Records the thread lists for the warp kernel (window or cell budget) are skipped.
"""
import re
import shutil
import subprocess
from pathlib import Path

import pytest

import oracle_ref as O

ROOT = Path(__file__).resolve().parent.parent
pytestmark = pytest.mark.skipif(shutil.which("nvcc") is None and not Path("/usr/local/cuda/bin/nvcc").exists(),
                                reason="nvcc not found")


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    O.build_oracle()
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    out = tmp_path_factory.mktemp("stream_host") / "stream_host"
    lib = ROOT / "oracle" / "build"
    subprocess.run([nvcc, "-std=c++17", "-O2", "-diag-suppress", "20014", "-o", str(out),
                    str(ROOT / "tests" / "stream_host.cu"), "-L", str(lib), "-lrmb_oracle",
                    "-Xlinker", "-rpath", "-Xlinker", str(lib)], check=True)
    return out


def _run(exe, records, seed, max_len, max_div, cutoff, max_cells):
    r = subprocess.run([str(exe), str(records), str(seed), str(max_len), str(max_div), str(cutoff), str(max_cells),
                        str(O.GOLDEN / "comparison.matrix")], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    v = dict((k, int(x)) for k, x in re.findall(r"(\w+) (\d+)", r.stdout))
    assert v["bad"] == 0 and v["cells"] == v["oracle_cells"], r.stdout
    assert v["checked"] > v["records"] // 2
    return v


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_stream_thread_matches_oracle(harness, seed):
    _run(harness, 20000, seed, 600, 40, 0, 65536)


def test_stream_thread_cutoff_and_cell_budget(harness):
    v = _run(harness, 20000, 4, 600, 40, 50, 8192)
    assert v["overflow"] > 0


def test_stream_thread_origin_moves(harness):
    # long near-identical records: extension scores pass 4096, where the origin moves
    v = _run(harness, 2000, 5, 5000, 3, 0, 1_000_000)
    assert v["big"] > 100
