"""Pins the CPU oracle to the reference's NCBI-2.17.1 golden outputs.

The CLI goldens are the reference's rmblastn/tests/data fixtures (copied into tests/golden by
tests/golden/make_fixtures.py) with the command lines of rmblastn/tests/cli.rs:11-35, 144-290.
The chr22 stage goldens (rmblast-lib/tests/*_regression.rs, 247,629 records each) and the chunked
chr22 golden (rmblastn/tests/cli.rs:246-274) are checked against the fixtures of
tests/golden/make_fixtures.py: chr22 itself as a compressed .2bit, the stage goldens as line count
and SHA-256 of their text, the chunked golden's text.
"""
import pytest

import chr22_fixture as F
import oracle_ref as O

G = O.GOLDEN
RM = ["--gapopen", "20", "--gapextend", "5", "--word-size", "14", "--xdrop-ungap", "400",
      "--xdrop-gap-final", "200", "--xdrop-gap", "100", "--min-raw-gapped-score", "200", "--outfmt", O.RM_FIELDS]


def _run(db, q, m, extra):
    return O.run_cli(["--db", str(G / db), "--query", str(G / q), "--matrix", str(G / m), *extra])


CASES = [
    ("nomask_nodust", "db.fa", "query.fa", "comparison.matrix", RM + ["--mask-level", "101", "--dust", "no", "--num-threads", "4"]),
    ("rm_defaults", "db.fa", "query.fa", "comparison.matrix", RM + ["--mask-level", "80", "--complexity-adjust", "--dust", "yes"]),
    ("query_dash", "db.fa", "query_dash.fa", "comparison.matrix", RM + ["--mask-level", "80", "--complexity-adjust", "--dust", "yes"]),
    ("db_dash", "db_dash.fa", "query.fa", "comparison.matrix", RM + ["--mask-level", "80", "--complexity-adjust", "--dust", "yes"]),
    ("asym_freqs", "db.fa", "query.fa", "asym_freqs.matrix", RM + ["--mask-level", "101", "--complexity-adjust", "--dust", "yes"]),
    ("defaults", "db.fa", "query.fa", "comparison.matrix", ["--gapopen", "20", "--gapextend", "5", "--outfmt", O.RM_FIELDS]),
]


@pytest.mark.parametrize("name,db,q,m,extra", CASES, ids=[c[0] for c in CASES])
def test_oracle_matches_ncbi_golden(name, db, q, m, extra):
    got = _run(db, q, m, extra)
    want = (G / f"expected_{name}.ncbi-2.17.1.tsv").read_text()
    assert got == want


def test_identity_matrix_has_no_score_zero_hits():
    # rmblastn/tests/cli.rs:210-226
    out = _run("db.fa", "query.fa", "identity.matrix",
               ["--gapopen", "20", "--gapextend", "5", "--word-size", "14", "--dust", "no", "--outfmt", "6 score qstart qend"])
    lines = out.splitlines()
    assert len(lines) > 300
    for ln in lines:
        s, a, b = map(int, ln.split("\t"))
        assert s >= 1 and b >= a


@pytest.fixture(scope="module")
def chr22_fasta(tmp_path_factory):
    name, seq = F.chr22()
    return F.write_fasta(tmp_path_factory.mktemp("chr22") / "chr22.fa", name, seq)


@pytest.mark.parametrize("stage,key", [(0, "seeds"), (1, "ungapped")])
def test_oracle_matches_chr22_stage_goldens(chr22_fasta, stage, key):
    """chr22 (51 chunks of ~1 Mb) against alu.2bit at word 14: the deduplicated seeds (sorted
    text) and the ungapped hits (chunk, then subject, then the reference's hit order), content
    and order, against the reference's 247,629-line goldens."""
    import ctypes as C
    lib = O.lib()
    lib.rmbo_stage_file.argtypes = [C.c_char_p] * 3 + [C.POINTER(O.OParams), C.c_int, C.POINTER(C.c_void_p),
                                                       C.c_char_p, C.c_size_t]
    p = O.oparams(dict(O.RM_PARAMS, complexity_adjust=1, dust=0, mask_level=80))
    out = C.c_void_p()
    err = C.create_string_buffer(512)
    rc = lib.rmbo_stage_file(str(chr22_fasta).encode(), str(G / "alu.2bit").encode(),
                             str(G / "comparison.matrix").encode(), C.byref(p), stage, C.byref(out), err, 512)
    assert rc == 0, err.value
    got = C.string_at(out.value).decode()
    lib.rmbo_free(out)
    want = F.stage_digests()[key]
    assert F.digest(got) == (want["lines"], want["sha256"])


def test_oracle_chunked_path_matches_chr22_golden(tmp_path):
    """The multi-chunk path (a 3 Mb query: three chunks, DUST on the whole query, cross-chunk
    merge, full-query traceback) against NCBI 2.17.1: rmblastn/tests/cli.rs:246-274."""
    _, seq = F.chr22()
    q = F.write_fasta(tmp_path / "chr22_30M_33M.fa", "chr22_30M_33M", seq[30_000_000:33_000_000])
    got = O.run_cli(["--db", str(G / "db.fa"), "--query", str(q), "--matrix", str(G / "comparison.matrix"),
                     "--gapopen", "20", "--gapextend", "5", "--word-size", "7", "--min-raw-gapped-score", "200",
                     "--mask-level", "80", "--num-threads", "8",
                     "--outfmt", "6 score qseqid qstart qend sstrand sseqid sstart send"])
    assert got.count("\n") == 4236
    assert got == F.chunked_golden()


@pytest.mark.parametrize("name,extra", [
    ("defaults", []),
    ("rm", ["--word-size", "14", "--mask-level", "80", "--complexity-adjust", "--min-raw-gapped-score", "200",
            "--xdrop-ungap", "400", "--xdrop-gap-final", "200", "--xdrop-gap", "100"]),
])
def test_oracle_pairwise_matches_ncbi(name, extra):
    """Pairwise output (outfmt 0, the default) against NCBI 2.17.1: rmblastn/tests/cli.rs:197-212,
    run from the fixtures' folder so the database prints under its own name; the "Posted date"
    line (the file's time) is left out, as the reference's test does."""
    import subprocess
    O.build_oracle()
    r = subprocess.run([str(O.ORACLE_CLI), "--db", "db.fa", "--query", "query.fa", "--matrix", "comparison.matrix",
                        "--gapopen", "20", "--gapextend", "5", "--num-threads", "2", *extra],
                       cwd=G, check=True, capture_output=True, text=True)
    want = "".join(ln for ln in (G / f"expected_pairwise_{name}.ncbi-2.17.1.txt").read_text().splitlines(True)
                   if not ln.startswith("    Posted date:"))
    assert r.stdout == want
