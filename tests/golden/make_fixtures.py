"""Copies the reference's NCBI-2.17.1 golden fixtures used by the parity tests into this folder.

The fixtures are the reference's own test vectors (rmblastn/tests/data/): a three-record query,
a 17-record TE library, the RMBlast matrices, NCBI rmblastn 2.17.1 outfmt-6 and pairwise outputs
for the command lines listed in rmblastn/tests/cli.rs:11-35 and 197-212, and a small .2bit
database.

The chr22 fixtures let the chr22 goldens run where the reference tree is absent (the GPU tests):
  chr22.2bit.xz            the reference's tests/data/chr22.fa as an xz-compressed UCSC .2bit
                           (its only letters are ACGTN, upper case, so the .2bit holds it exactly)
  chr22_stage_goldens.json line count and SHA-256 of rmblast-lib/tests/data/chr22_dedup_seeds.txt
                           and chr22_ungapped_hits.txt (247,629 lines each, 21 MB of text)
  expected_chr22_30M-33M_ws7.ncbi-2.17.1.tsv.xz  the chunked-query golden (cli.rs:246-274)

Run once in a checkout that has the reference tree next to it:
    python tests/golden/make_fixtures.py /path/to/RMBlast     (or set RMB_REFERENCE_ROOT)
"""
import hashlib
import json
import lzma
import os
import shutil
import struct
import sys
from pathlib import Path

import numpy as np

FILES = [
    "query.fa", "query_dash.fa", "db.fa", "db_dash.fa",
    "comparison.matrix", "asym_freqs.matrix", "identity.matrix",
    "expected_nomask_nodust.ncbi-2.17.1.tsv", "expected_rm_defaults.ncbi-2.17.1.tsv",
    "expected_query_dash.ncbi-2.17.1.tsv", "expected_db_dash.ncbi-2.17.1.tsv",
    "expected_asym_freqs.ncbi-2.17.1.tsv", "expected_defaults.ncbi-2.17.1.tsv",
    "expected_pairwise_defaults.ncbi-2.17.1.txt", "expected_pairwise_rm.ncbi-2.17.1.txt",
]
# the .2bit database of the chr22 stage goldens (rmblast-lib/tests/*_regression.rs), from the
# reference's top-level tests/data
TOP_FILES = ["alu.2bit"]
STAGE_GOLDENS = {"seeds": "chr22_dedup_seeds.txt", "ungapped": "chr22_ungapped_hits.txt"}
CHUNKED_GOLDEN = "expected_chr22_30M-33M_ws7.ncbi-2.17.1.tsv"


def twobit_bytes(name: str, seq: bytes) -> bytes:
    """One-record little-endian UCSC .2bit (T=0 C=1 A=2 G=3, N runs as N blocks, no mask blocks:
    the sequence must be upper-case ACGTN)."""
    s = np.frombuffer(seq, dtype=np.uint8)
    code = np.zeros(256, np.uint8)
    for ch, v in zip(b"TCAGN", (0, 1, 2, 3, 0)):
        code[ch] = v
    bad = ~np.isin(s, np.frombuffer(b"ACGTN", np.uint8))
    if bad.any():
        raise ValueError("the .2bit fixture holds upper-case ACGTN only")
    isn = np.concatenate([[0], (s == ord("N")).astype(np.int8), [0]])
    d = np.diff(isn)
    starts = np.nonzero(d == 1)[0]
    lens = np.nonzero(d == -1)[0] - starts
    c = code[s]
    c = np.concatenate([c, np.zeros((-len(c)) % 4, np.uint8)]).reshape(-1, 4)
    packed = ((c[:, 0] << 6) | (c[:, 1] << 4) | (c[:, 2] << 2) | c[:, 3]).astype(np.uint8).tobytes()
    rec = struct.pack("<II", len(s), len(starts)) + starts.astype("<u4").tobytes() + lens.astype("<u4").tobytes()
    rec += struct.pack("<II", 0, 0) + packed
    head = struct.pack("<IIII", 0x1A412743, 0, 1, 0)
    off = len(head) + 1 + len(name) + 4
    return head + bytes([len(name)]) + name.encode() + struct.pack("<I", off) + rec


def main(ref_root: str) -> None:
    ref = Path(ref_root)
    src = ref / "rmblastn" / "tests" / "data"
    dst = Path(__file__).resolve().parent
    for name in FILES:
        shutil.copyfile(src / name, dst / name)
        print("copied", name)
    for name in TOP_FILES:
        shutil.copyfile(ref / "tests" / "data" / name, dst / name)
        print("copied", name)
    lines = (ref / "tests" / "data" / "chr22.fa").read_bytes().split(b"\n")
    name = lines[0][1:].split()[0].decode()
    seq = b"".join(ln.strip() for ln in lines[1:] if not ln.startswith(b">"))
    (dst / "chr22.2bit.xz").write_bytes(lzma.compress(twobit_bytes(name, seq), preset=9))
    print("wrote chr22.2bit.xz", len(seq), "bases")
    digests = {}
    for key, fname in STAGE_GOLDENS.items():
        text = (ref / "rmblast-lib" / "tests" / "data" / fname).read_bytes()
        digests[key] = {"file": f"rmblast-lib/tests/data/{fname}", "lines": text.count(b"\n"),
                        "sha256": hashlib.sha256(text).hexdigest()}
    (dst / "chr22_stage_goldens.json").write_text(json.dumps(digests, indent=1) + "\n")
    print("wrote chr22_stage_goldens.json")
    (dst / (CHUNKED_GOLDEN + ".xz")).write_bytes(lzma.compress((src / CHUNKED_GOLDEN).read_bytes(), preset=9))
    print("wrote", CHUNKED_GOLDEN + ".xz")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("RMB_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_fixtures.py <reference checkout>   (or set RMB_REFERENCE_ROOT)")
    main(root)
