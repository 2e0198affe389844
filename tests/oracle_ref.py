"""ctypes access to the CPU oracle (oracle/build/librmb_oracle.so) for the parity tests.

Test infrastructure only: the oracle is the checker the CUDA path is compared against.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
ORACLE_DIR = ROOT / "oracle"
ORACLE_LIB = ORACLE_DIR / "build" / "librmb_oracle.so"
ORACLE_CLI = ORACLE_DIR / "build" / "rmblastn_oracle"
GOLDEN = Path(__file__).resolve().parent / "golden"

RM_FIELDS = ("6 score perc_sub perc_query_gap perc_db_gap qseqid qstart qend qlen sstrand sseqid sstart send "
             "slen kdiv cpg_kdiv transi transv cpg_sites qseq sseq")
RM_PARAMS = dict(gap_open=20, gap_extend=5, word_size=14, xdrop_ungap=400, xdrop_gap_final=200, xdrop_gap=100,
                 min_raw_gapped_score=200)


class OParams(C.Structure):
    _fields_ = [(n, C.c_int32) for n in (
        "gap_open", "gap_extend", "word_size", "xdrop_ungap", "xdrop_gap", "xdrop_gap_final",
        "min_raw_gapped_score", "complexity_adjust", "dust", "mask_level")] + [
        ("evalue", C.c_double), ("cli_stats", C.c_double * 4)]


def build_oracle() -> None:
    subprocess.run(["make", "-s", "-C", str(ORACLE_DIR)], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        build_oracle()
        _lib = C.CDLL(str(ORACLE_LIB))
        _lib.rmbo_search_text.argtypes = [C.c_char_p] * 4 + [C.POINTER(OParams), C.c_char_p, C.c_int,
                                                              C.POINTER(C.c_void_p), C.POINTER(C.c_uint64),
                                                              C.POINTER(C.c_double), C.c_char_p, C.c_size_t]
        _lib.rmbo_stage_text.argtypes = [C.c_char_p] * 4 + [C.POINTER(OParams), C.c_int,
                                                             C.POINTER(C.POINTER(C.c_uint32)),
                                                             C.POINTER(C.c_uint64), C.c_char_p, C.c_size_t]
        _lib.rmbo_free.argtypes = [C.c_void_p]
    return _lib


def oparams(p: dict) -> OParams:
    cli = p.get("cli_stats", (0.0, 0.0, 0.0, 0.0))
    return OParams(p["gap_open"], p["gap_extend"], p["word_size"], p["xdrop_ungap"], p["xdrop_gap"],
                   p["xdrop_gap_final"], p["min_raw_gapped_score"], int(p.get("complexity_adjust", 0)),
                   int(p.get("dust", 0)), int(p.get("mask_level", -1)), float(p.get("evalue", 0.0)),
                   (C.c_double * 4)(*cli))


def search_text(query_fasta: str, db_fasta: str, matrix_text: str, matrix_name: str, p: dict, outfmt: str,
                threads: int = 8):
    out = C.c_void_p()
    ctr = (C.c_uint64 * 9)()
    sec = C.c_double()
    err = C.create_string_buffer(512)
    rc = lib().rmbo_search_text(query_fasta.encode(), db_fasta.encode(), matrix_text.encode(), matrix_name.encode(),
                                C.byref(oparams(p)), outfmt.encode(), threads, C.byref(out), ctr, C.byref(sec), err,
                                512)
    if rc:
        raise RuntimeError(err.value.decode())
    try:
        text = C.string_at(out.value).decode()
    finally:
        lib().rmbo_free(out)
    names = "word_hits seeds ungapped prelim_dp prelims tb_dp finals so_cells tb_cells".split()
    return text, dict(zip(names, list(ctr))), sec.value


def stage_text(query_fasta: str, db_fasta: str, matrix_text: str, matrix_name: str, p: dict, stage: int) -> np.ndarray:
    rec = C.POINTER(C.c_uint32)()
    n = C.c_uint64()
    err = C.create_string_buffer(512)
    rc = lib().rmbo_stage_text(query_fasta.encode(), db_fasta.encode(), matrix_text.encode(), matrix_name.encode(),
                               C.byref(oparams(p)), stage, C.byref(rec), C.byref(n), err, 512)
    if rc:
        raise RuntimeError(err.value.decode())
    width = {0: 3, 1: 6, 2: 8, 4: 9}[stage]
    try:
        a = np.ctypeslib.as_array(rec, shape=(int(n.value) * width,)).copy() if n.value else np.zeros(0, np.uint32)
    finally:
        lib().rmbo_free(C.cast(rec, C.c_void_p))
    return a.reshape(-1, width)


def run_cli(args: list[str]) -> str:
    build_oracle()
    r = subprocess.run([str(ORACLE_CLI), *args], check=True, capture_output=True, text=True)
    return r.stdout
