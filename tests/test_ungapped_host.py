"""The ungapped walk of k_ungapped, built for the host, against the oracle's extension.

rmb_ungapped.cuh holds the resumable walk each lane of k_ungapped runs (left walk, then right
walk, one base a step); tests/ungapped_host.cu compiles it as host code with nvcc and compares
score and box with the oracle's extend_ungapped (search/ungapped.rs:38-121) on random hits:
shared mutated segments, N codes, sequence ends.
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
    out = tmp_path_factory.mktemp("ungapped_host") / "ungapped_host"
    lib = ROOT / "oracle" / "build"
    subprocess.run([nvcc, "-std=c++17", "-O2", "-o", str(out), str(ROOT / "tests" / "ungapped_host.cu"),
                    "-L", str(lib), "-lrmb_oracle", "-Xlinker", "-rpath", "-Xlinker", str(lib)], check=True)
    return out


@pytest.mark.parametrize("seed,xdrop", [(1, 400), (2, 20), (3, 100)])
def test_walk_matches_oracle(harness, seed, xdrop):
    r = subprocess.run([str(harness), "20000", str(seed), str(xdrop), str(O.GOLDEN / "comparison.matrix")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    v = dict((k, int(x)) for k, x in re.findall(r"(\w+) (\d+)", r.stdout))
    assert v["bad"] == 0 and v["hits"] == 20000 and v["steps"] > 20000
