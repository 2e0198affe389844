"""Copies the reference's NCBI-2.17.1 golden fixtures used by the parity tests into this folder.

The fixtures are the reference's own test vectors (rmblastn/tests/data/): a three-record query,
a 17-record TE library, the RMBlast matrices, NCBI rmblastn 2.17.1 outfmt-6 and pairwise outputs
for the command lines listed in rmblastn/tests/cli.rs:11-35 and 197-212, and a small .2bit
database.  Run once in a checkout that has the
reference tree next to it:  python tests/golden/make_fixtures.py /path/to/RMBlast
"""
import shutil
import sys
from pathlib import Path

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


def main(ref_root: str) -> None:
    src = Path(ref_root) / "rmblastn" / "tests" / "data"
    dst = Path(__file__).resolve().parent
    for name in FILES:
        shutil.copyfile(src / name, dst / name)
        print("copied", name)
    for name in TOP_FILES:
        shutil.copyfile(Path(ref_root) / "tests" / "data" / name, dst / name)
        print("copied", name)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
