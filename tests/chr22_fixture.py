"""The chr22 fixtures of the reference's regression goldens (tests/golden/make_fixtures.py):
the chromosome, the NCBI chunking of rmblast-lib/tests/ungapped_regression.rs:29-50, and the
golden digests.  Test infrastructure."""
from __future__ import annotations

import hashlib
import json
import lzma
from functools import lru_cache
from pathlib import Path

from twobit_util import read_twobit_ascii

GOLDEN = Path(__file__).resolve().parent / "golden"
STAGE_PARAMS = dict(gap_open=20, gap_extend=5, word_size=14, xdrop_ungap=400, xdrop_gap=100, xdrop_gap_final=200,
                    min_raw_gapped_score=200, complexity_adjust=1, dust=0, mask_level=80)


@lru_cache(maxsize=1)
def chr22() -> tuple[str, bytes]:
    return read_twobit_ascii(lzma.decompress((GOLDEN / "chr22.2bit.xz").read_bytes()))[0]


def stage_digests() -> dict:
    return json.loads((GOLDEN / "chr22_stage_goldens.json").read_text())


def chunked_golden() -> str:
    return lzma.decompress((GOLDEN / "expected_chr22_30M-33M_ws7.ncbi-2.17.1.tsv.xz").read_bytes()).decode()


def chunks(qlen: int) -> list[tuple[int, int]]:
    """ungapped_regression.rs:29-50 compute_chunks (NCBI BlastSplitQuery: 1,000,000-base chunks
    with a 100-base overlap)."""
    nch = qlen // (1_000_000 - 100)
    if nch <= 1:
        cs, eff = qlen, 1
    else:
        cs = (qlen + (nch - 1) * 100) // nch
        if nch < max(cs - 100, 0):
            cs += 1
        eff = nch
    step = max(cs - 100, 0)
    out = []
    for k in range(eff):
        st = k * step
        if st >= qlen:
            break
        out.append((st, min(st + cs, qlen)))
    return out


def digest(text: str) -> tuple[int, str]:
    b = text.encode()
    return b.count(b"\n"), hashlib.sha256(b).hexdigest()


def write_fasta(path: Path, name: str, seq: bytes) -> Path:
    path.write_bytes(b">" + name.encode() + b"\n" + b"\n".join(seq[i:i + 60] for i in range(0, len(seq), 60)) + b"\n")
    return path
