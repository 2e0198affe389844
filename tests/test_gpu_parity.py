"""Parity of the CUDA search core with the oracle and the reference's NCBI goldens.

Every comparison is exact (byte-identical outfmt-6 text, identical stage records): the path is
integer arithmetic plus the reference's own f64/f32 formulas on the host, so there is no
tolerance.  Inputs are the reference's fixtures and seeded synthetic genome/library workloads.
"""
import numpy as np
import pytest

import oracle_ref as O
from rmblast_b200 import api, build, synth

pytestmark = pytest.mark.gpu
G = O.GOLDEN


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def searcher(p: dict, matrix_text: str, matrix_name: str, db_fasta: str, kernels: int = 0, pipeline: int = 0,
             schedule: int = 0):
    m = api.ScoreMatrix.from_text(matrix_text, matrix_name)
    sp = api.SearchParams(gap_open=p["gap_open"], gap_extend=p["gap_extend"], word_size=p["word_size"],
                          xdrop_ungap=p["xdrop_ungap"], xdrop_gap=p["xdrop_gap"], xdrop_gap_final=p["xdrop_gap_final"],
                          min_raw_gapped_score=p["min_raw_gapped_score"],
                          complexity_adjust=bool(p.get("complexity_adjust", 0)), dust=bool(p.get("dust", 0)),
                          mask_level=p.get("mask_level", -1), kernels=kernels, evalue=p.get("evalue", 0.0),
                          pipeline=pipeline, schedule=schedule,
                          **dict(zip(("matrix_lambda", "matrix_k", "matrix_alpha", "matrix_beta"),
                                     p.get("cli_stats", (0.0, 0.0, 0.0, 0.0)))))
    s = api.Searcher(sp, m, api.SubjectDb.from_fasta(db_fasta))
    if schedule >= 1:
        from rmblast_b200 import train_sched
        s.set_schedule_model(train_sched.load_model())
    return s


def gpu_text(p, matrix_text, matrix_name, db_fasta, query_fasta, outfmt):
    s = searcher(p, matrix_text, matrix_name, db_fasta)
    recs = api.read_fasta(query_fasta)
    res = s.search([api.encode(seq) for _, seq in recs], [n for n, _ in recs])
    return res.tabular(outfmt), res


def test_golden_nomask_nodust_through_c_abi():
    p = dict(O.RM_PARAMS, mask_level=101)
    txt, _ = gpu_text(p, (G / "comparison.matrix").read_text(), "comparison.matrix", (G / "db.fa").read_text(),
                      (G / "query.fa").read_text(), O.RM_FIELDS)
    assert txt == (G / "expected_nomask_nodust.ncbi-2.17.1.tsv").read_text()


DUST_GOLDENS = [
    # name, db, query, matrix, parameters: the reference's CLI tests (rmblastn/tests/cli.rs)
    ("rm_defaults", "db.fa", "query.fa", "comparison.matrix",
     dict(O.RM_PARAMS, mask_level=80, complexity_adjust=1, dust=1)),
    ("query_dash", "db.fa", "query_dash.fa", "comparison.matrix",
     dict(O.RM_PARAMS, mask_level=80, complexity_adjust=1, dust=1)),
    ("db_dash", "db_dash.fa", "query.fa", "comparison.matrix",
     dict(O.RM_PARAMS, mask_level=80, complexity_adjust=1, dust=1)),
    ("asym_freqs", "db.fa", "query.fa", "asym_freqs.matrix",
     dict(O.RM_PARAMS, mask_level=101, complexity_adjust=1, dust=1)),
    ("defaults", "db.fa", "query.fa", "comparison.matrix",
     dict(gap_open=20, gap_extend=5, word_size=11, xdrop_ungap=20, xdrop_gap=30, xdrop_gap_final=100,
          min_raw_gapped_score=0, mask_level=101, dust=1)),
]


@pytest.mark.parametrize("name,db,q,m,p", DUST_GOLDENS, ids=[c[0] for c in DUST_GOLDENS])
def test_golden_with_dust_through_c_abi(name, db, q, m, p):
    """The NCBI-2.17.1 goldens whose command lines mask the query with DUST (dust on is the
    reference's default): the device masker, then the whole path, byte for byte."""
    txt, _ = gpu_text(p, (G / m).read_text(), m, (G / db).read_text(), (G / q).read_text(), O.RM_FIELDS)
    assert txt == (G / f"expected_{name}.ncbi-2.17.1.tsv").read_text()


def with_low_complexity(seqs, seed):
    """Plants microsatellites, poly-A tails, near-repeats and N runs: DUST's cases."""
    rng = np.random.default_rng(seed)
    units = [b"CA", b"A", b"AAAAT", b"GGC", b"TTAGGG", b"ACGTTGCA", b"AT"]
    out = []
    for s in seqs:
        s = bytearray(s.tobytes())
        for _ in range(max(1, len(s) // 3000)):
            u = units[rng.integers(len(units))]
            rep = bytearray(u * int(rng.integers(8, 120)))
            for k in range(len(rep)):  # a few point mutations: low but not zero complexity
                if rng.random() < 0.04:
                    rep[k] = b"ACGTN"[rng.integers(5)]
            at = int(rng.integers(0, max(1, len(s) - len(rep))))
            s[at:at + len(rep)] = rep
        out.append(np.frombuffer(bytes(s), dtype=np.uint8))
    return out


@pytest.mark.parametrize("ws", [7, 11, 14])
def test_dust_on_synthetic_matches_oracle(ws):
    qs, db, prm = synth.workload("small", scale=0.3)
    p = dict(prm, **synth.RM_FLAGS)
    p.update(dust=1, word_size=ws)
    seqs = with_low_complexity([s for _, s in qs], 11 + ws)
    qf = synth.to_fasta([n for n, _ in qs], seqs)
    dbf = synth.to_fasta([n for n, _ in db], [s for _, s in db])
    s = searcher(p, synth.MATRIX_TEXT, synth.MATRIX_NAME, dbf)
    recs = api.read_fasta(qf)
    enc = [api.encode(x) for _, x in recs]
    for stage in (0, 1):
        got = s.stage(enc, stage)
        want = O.stage_text(qf, dbf, synth.MATRIX_TEXT, synth.MATRIX_NAME, p, stage)
        assert got.shape == want.shape, (stage, got.shape, want.shape)
        assert np.array_equal(got, want), stage
    res = s.search(enc, [n for n, _ in recs])
    want_txt, _, _ = O.search_text(qf, dbf, synth.MATRIX_TEXT, synth.MATRIX_NAME, p, FIELDS)
    assert res.tabular(FIELDS) == want_txt
    # the planted runs are masked: without DUST the reference finds other seeds
    unmasked = O.stage_text(qf, dbf, synth.MATRIX_TEXT, synth.MATRIX_NAME, dict(p, dust=0), 0)
    assert unmasked.shape != want.shape or not np.array_equal(unmasked, want)


def test_scan_long_lookup_cells_match_oracle():
    """Low-complexity runs in queries and library with DUST off: the runs' words fill lookup cells
    far past 32 entries, so the scan's write loop takes its path for long cells; seeds and
    ungapped hits against the oracle."""
    qs, db, prm = synth.workload("small", scale=0.3)
    p = dict(prm, **synth.RM_FLAGS)
    p.update(dust=0, word_size=11)
    qseqs = with_low_complexity([s for _, s in qs], 5)
    dseqs = with_low_complexity([s for _, s in db], 6)
    qf = synth.to_fasta([n for n, _ in qs], qseqs)
    dbf = synth.to_fasta([n for n, _ in db], dseqs)
    s = searcher(p, synth.MATRIX_TEXT, synth.MATRIX_NAME, dbf)
    enc = [api.encode(x) for _, x in api.read_fasta(qf)]
    for stage in (0, 1):
        got = s.stage(enc, stage)
        want = O.stage_text(qf, dbf, synth.MATRIX_TEXT, synth.MATRIX_NAME, p, stage)
        assert got.shape == want.shape, (stage, got.shape, want.shape)
        assert np.array_equal(got, want), stage
    # some query has a word more than 32 times (a cell past the write loop's 32-entry mask)
    from collections import Counter
    assert max(max(Counter(bytes(q[i:i + 8]) for i in range(len(q) - 8)).values()) for q in qseqs) > 32


def test_golden_db_dash_subjects_nomask():
    # '-' in subjects is N: CRandom-resolved for the scan, restored for the traceback
    p = dict(O.RM_PARAMS, mask_level=101)
    mt = (G / "comparison.matrix").read_text()
    db = (G / "db_dash.fa").read_text()
    q = (G / "query.fa").read_text()
    txt, _ = gpu_text(p, mt, "comparison.matrix", db, q, O.RM_FIELDS)
    want, _, _ = O.search_text(q, db, mt, "comparison.matrix", p, O.RM_FIELDS)
    assert txt == want


def test_identity_matrix_default_cutoff_matches_oracle():
    p = dict(gap_open=20, gap_extend=5, word_size=14, xdrop_ungap=20, xdrop_gap=30, xdrop_gap_final=100,
             min_raw_gapped_score=0)
    mt = (G / "identity.matrix").read_text()
    db, q = (G / "db.fa").read_text(), (G / "query.fa").read_text()
    txt, _ = gpu_text(p, mt, "identity.matrix", db, q, "6 score qstart qend sstart send sseqid perc_sub")
    want, _, _ = O.search_text(q, db, mt, "identity.matrix", p, "6 score qstart qend sstart send sseqid perc_sub")
    assert txt.count("\n") > 300
    assert txt == want


def synthetic(name, scale, flags):
    qs, db, prm = synth.workload(name, scale=scale)
    p = dict(prm)
    p.update(flags)
    qf = synth.to_fasta([n for n, _ in qs], [s for _, s in qs])
    dbf = synth.to_fasta([n for n, _ in db], [s for _, s in db])
    return qf, dbf, p


FIELDS = "6 score perc_sub perc_query_gap perc_db_gap qseqid qstart qend sseqid sstart send kdiv cpg_kdiv qseq sseq"


@pytest.mark.parametrize("flags", ["rm", "default"])
def test_synthetic_small_matches_oracle(flags):
    qf, dbf, p = synthetic("small", 0.25, synth.RM_FLAGS if flags == "rm" else synth.DEFAULT_FLAGS)
    txt, res = gpu_text(p, synth.MATRIX_TEXT, synth.MATRIX_NAME, dbf, qf, FIELDS)
    want, ctr, _ = O.search_text(qf, dbf, synth.MATRIX_TEXT, synth.MATRIX_NAME, p, FIELDS)
    assert txt.count("\n") > 10
    assert txt == want
    assert res.counters["ungapped"] == ctr["ungapped"]
    # the GPU runs the prelim DP of every ungapped record, contained ones too
    assert res.counters["so_cells"] >= ctr["so_cells"]


def test_synthetic_plain_matches_oracle():
    qf, dbf, p = synthetic("plain", 0.003, synth.RM_FLAGS)
    txt, res = gpu_text(p, synth.MATRIX_TEXT, synth.MATRIX_NAME, dbf, qf, FIELDS)
    want, ctr, _ = O.search_text(qf, dbf, synth.MATRIX_TEXT, synth.MATRIX_NAME, p, FIELDS)
    assert txt.count("\n") > 20
    assert txt == want
    assert res.counters["ungapped"] == ctr["ungapped"]
    assert res.counters["prelim_dp"] >= ctr["prelim_dp"]
    assert res.counters["so_cells"] >= ctr["so_cells"]


@pytest.mark.parametrize("ws", [4, 5, 6, 7, 8, 9, 10, 11, 12, 14, 16, 24])
def test_word_sizes_stage_taps_and_output(ws):
    qf, dbf, p = synthetic("small", 0.04, synth.RM_FLAGS)
    p["word_size"] = ws
    s = searcher(p, synth.MATRIX_TEXT, synth.MATRIX_NAME, dbf)
    recs = api.read_fasta(qf)
    qs = [api.encode(seq) for _, seq in recs]
    for stage in (0, 1):
        got = s.stage(qs, stage)
        want = O.stage_text(qf, dbf, synth.MATRIX_TEXT, synth.MATRIX_NAME, p, stage)
        assert got.shape == want.shape, (stage, got.shape, want.shape)
        assert np.array_equal(got, want), stage
    got = s.stage(qs, 2)
    want = O.stage_text(qf, dbf, synth.MATRIX_TEXT, synth.MATRIX_NAME, p, 2)
    assert sorted(map(tuple, got.tolist())) == sorted(map(tuple, want.tolist()))
    res = s.search(qs, [n for n, _ in recs])
    want_txt, _, _ = O.search_text(qf, dbf, synth.MATRIX_TEXT, synth.MATRIX_NAME, p, FIELDS)
    assert res.tabular(FIELDS) == want_txt


@pytest.mark.parametrize("kernels", [0, 1])
@pytest.mark.parametrize("gaps", [(20, 5, 100, 0.2), (3, 1, 120, 0.03)])
def test_prelim_kernels_match_oracle(kernels, gaps):
    """Both preliminary-DP paths: the thread-per-extension kernel with its fallback for bands wider
    than its ring (cheap gaps with a large X-drop widen the band), and the warp kernel alone."""
    qf, dbf, p = synthetic("small", gaps[3], synth.RM_FLAGS)
    p.update(gap_open=gaps[0], gap_extend=gaps[1], xdrop_gap=gaps[2])
    s = searcher(p, synth.MATRIX_TEXT, synth.MATRIX_NAME, dbf, kernels=kernels)
    recs = api.read_fasta(qf)
    qs = [api.encode(seq) for _, seq in recs]
    got = s.stage(qs, 2)
    want = O.stage_text(qf, dbf, synth.MATRIX_TEXT, synth.MATRIX_NAME, p, 2)
    assert len(want) > 10
    assert sorted(map(tuple, got.tolist())) == sorted(map(tuple, want.tolist()))
    res = s.search(qs, [n for n, _ in recs])
    want_txt, ctr, _ = O.search_text(qf, dbf, synth.MATRIX_TEXT, synth.MATRIX_NAME, p, FIELDS)
    assert res.tabular(FIELDS) == want_txt
    assert res.counters["so_cells"] >= ctr["so_cells"]


def test_golden_stage_taps_match_oracle():
    p = dict(O.RM_PARAMS, mask_level=101)
    mt, db, q = (G / "comparison.matrix").read_text(), (G / "db.fa").read_text(), (G / "query.fa").read_text()
    s = searcher(p, mt, "comparison.matrix", db)
    qs = [api.encode(seq) for _, seq in api.read_fasta(q)]
    for stage in (0, 1):
        assert np.array_equal(s.stage(qs, stage), O.stage_text(q, db, mt, "comparison.matrix", p, stage))


def test_edge_cases():
    p = dict(O.RM_PARAMS, mask_level=101)
    mt, db = (G / "comparison.matrix").read_text(), (G / "db.fa").read_text()
    s = searcher(p, mt, "comparison.matrix", db)
    # shorter than the word size, exactly the word size, all N, empty batch
    qs = [api.encode(b"ACGT"), api.encode(b"A" * 14), api.encode(b"N" * 5000)]
    res = s.search(qs)
    assert res.n_hsps == 0
    assert s.search([]).n_hsps == 0


def test_lookup_tables_match_reference_rules():
    """Stage 3: the device-built tables hold, per cell, exactly the positions of the reference's
    table in its retrieval order (ascending for lw <= 8, descending for the megablast table)."""
    p = dict(O.RM_PARAMS, mask_level=101)
    mt, db, q = (G / "comparison.matrix").read_text(), (G / "db.fa").read_text(), (G / "query.fa").read_text()
    s = searcher(p, mt, "comparison.matrix", db)
    qs = [api.encode(seq) for _, seq in api.read_fasta(q)]
    got = s.stage(qs, 3)
    comp = np.array([3, 2, 1, 0, 5, 4, 7, 6, 8, 9, 13, 12, 11, 10, 14, 15], np.uint8)
    for qi, e in enumerate(qs):
        n = len(e) - 2
        comb = np.concatenate([e[1:n + 1], [14], comp[e[1:n + 1][::-1]]]).astype(np.int64)
        lw = 8 if 2 * n < 8500 else 11 if 2 * n < 300000 else 12  # choose_lut_width, word 14
        ent = []
        for s0 in range(2 * n + 1):
            end = n - 1 if s0 < n else 2 * n
            if s0 == n or s0 + lw - 1 > end:
                continue
            w = comb[s0:s0 + lw]
            if (w > 3).any():
                continue
            c = 0
            for b in w:
                c = (c << 2) | int(b)
            ent.append((c, s0))
        ent.sort(key=lambda t: (t[0], t[1] if lw <= 8 else -t[1]))
        want = np.array([(qi, c, x) for c, x in ent], dtype=np.uint32).reshape(-1, 3)
        assert np.array_equal(got[got[:, 0] == qi], want), qi


@pytest.mark.parametrize("case", ["golden", "small_default"])
def test_traceback_stage_matches_oracle(case):
    """Stage 4: improve_seed + traceback DP + gap pruning of every prelim, unfiltered."""
    if case == "golden":
        p = dict(O.RM_PARAMS, mask_level=101)
        mt, mn, db, q = (G / "comparison.matrix").read_text(), "comparison.matrix", (G / "db.fa").read_text(), \
            (G / "query.fa").read_text()
    else:
        q, db, p = synthetic("small", 0.05, synth.DEFAULT_FLAGS)
        mt, mn = synth.MATRIX_TEXT, synth.MATRIX_NAME
    s = searcher(p, mt, mn, db)
    qs = [api.encode(seq) for _, seq in api.read_fasta(q)]
    got = s.stage(qs, 4)
    want = O.stage_text(q, db, mt, mn, p, 4)
    assert len(want) > 0
    assert np.array_equal(got, want)


@pytest.mark.parametrize("scale,dust", [(21.0, 1), (26.0, 0)])
def test_chunked_long_query_matches_oracle(scale, dust):
    """Queries of 1,999,800 bp or more take the multi-chunk path (two and three chunks here),
    in one call with short queries: every line against the oracle's chunked pipeline, which the
    chr22 NCBI golden pins."""
    qs, db, prm = synth.workload("small", scale=scale)
    short, _, _ = synth.workload("small", scale=0.2)
    p = dict(prm, **synth.RM_FLAGS)
    p["dust"] = dust
    names = [n for n, _ in short] + [n for n, _ in qs] + ["short_b"]
    seqs = [s for _, s in short] + [s for _, s in qs] + [short[0][1][5000:15000]]
    assert len(qs[0][1]) >= 1_999_800
    qf = synth.to_fasta(names, seqs)
    dbf = synth.to_fasta([n for n, _ in db], [s for _, s in db])
    txt, res = gpu_text(p, synth.MATRIX_TEXT, synth.MATRIX_NAME, dbf, qf, FIELDS)
    want, _, _ = O.search_text(qf, dbf, synth.MATRIX_TEXT, synth.MATRIX_NAME, p, FIELDS)
    assert txt.count("\n") > 1000
    assert txt == want


@pytest.mark.parametrize("name,scale", [("batched", 0.002), ("allvsall", 0.04)])
def test_config_workloads_match_oracle(name, scale):
    """The other configurations' shapes: many chunks of mixed lengths (1-200 kb, three lookup
    widths in one call) against the 2,000-consensus library, and the library searched against
    itself (word 7, masklevel off, derived and high-divergence consensi)."""
    qs, db, prm = synth.workload(name, scale=scale)
    p = dict(prm, **synth.RM_FLAGS)
    qf = synth.to_fasta([n for n, _ in qs], [s for _, s in qs])
    dbf = synth.to_fasta([n for n, _ in db], [s for _, s in db])
    txt, res = gpu_text(p, synth.MATRIX_TEXT, synth.MATRIX_NAME, dbf, qf, FIELDS)
    want, ctr, _ = O.search_text(qf, dbf, synth.MATRIX_TEXT, synth.MATRIX_NAME, p, FIELDS)
    assert txt.count("\n") > 150
    assert txt == want
    assert res.counters["ungapped"] == ctr["ungapped"]


def test_pair_ranges_match_oracle():
    """A batch with more word hits than one pass holds (500 consensi against themselves at word 7:
    ~760 M hits, two pair ranges): output and counters as in one pass, against the oracle."""
    qs, db, prm = synth.workload("allvsall", scale=0.1)
    p = dict(prm, **synth.RM_FLAGS)
    qf = synth.to_fasta([n for n, _ in qs], [s for _, s in qs])
    dbf = synth.to_fasta([n for n, _ in db], [s for _, s in db])
    txt, res = gpu_text(p, synth.MATRIX_TEXT, synth.MATRIX_NAME, dbf, qf, FIELDS)
    assert res.counters["word_hits"] > (1 << 29)
    want, ctr, _ = O.search_text(qf, dbf, synth.MATRIX_TEXT, synth.MATRIX_NAME, p, FIELDS)
    assert txt == want
    assert res.counters["ungapped"] == ctr["ungapped"]


STATS_FIELDS = "6 score evalue bitscore qseqid qstart qend sseqid sstart send"


@pytest.mark.parametrize("case", ["table", "command_line", "matrix_comment"])
def test_evalues_and_reap_match_oracle(case):
    """E-value and bit-score columns and the --evalue reap (before masklevel): statistics from the
    built-in table (comparison.matrix at 20/5), from the command line, and from a "# KARLIN"
    matrix comment."""
    if case == "table":
        p = dict(O.RM_PARAMS, mask_level=80, complexity_adjust=1, dust=1, evalue=1e-30)
        mt, name = (G / "comparison.matrix").read_text(), "comparison.matrix"
        qf, dbf = (G / "query.fa").read_text(), (G / "db.fa").read_text()
    else:
        qf, dbf, p = synthetic("small", 0.3, synth.RM_FLAGS)
        mt, name = synth.MATRIX_TEXT, synth.MATRIX_NAME
        if case == "command_line":
            p.update(cli_stats=(0.11, 0.09, 0.9, -20.0), evalue=1e-12)
        else:
            mt = "# KARLIN lambda 0.105 k 0.08 h 0.12\n" + mt
    txt, res = gpu_text(p, mt, name, dbf, qf, STATS_FIELDS)
    want, _, _ = O.search_text(qf, dbf, mt, name, p, STATS_FIELDS)
    assert txt == want
    lines = txt.splitlines()
    assert len(lines) > 10
    assert all(ln.split("\t")[1] != "1.0" for ln in lines)  # statistics were applied
    if p.get("evalue"):
        unreaped, _, _ = O.search_text(qf, dbf, mt, name, dict(p, evalue=0.0), STATS_FIELDS)
        assert unreaped.count("\n") > txt.count("\n")  # the cut dropped some HSPs


PAIRWISE_RM = dict(O.RM_PARAMS, mask_level=80, complexity_adjust=1, dust=1)
PAIRWISE_DEFAULTS = dict(gap_open=20, gap_extend=5, word_size=11, xdrop_ungap=20, xdrop_gap=30,
                         xdrop_gap_final=100, min_raw_gapped_score=0, mask_level=101, dust=1)


@pytest.mark.parametrize("name,p", [("defaults", PAIRWISE_DEFAULTS), ("rm", PAIRWISE_RM)])
def test_pairwise_goldens_through_c_abi(name, p):
    """Pairwise output (outfmt 0) of the device search against NCBI 2.17.1 (cli.rs:197-212): the
    statistics blocks, alignment rows, DUST-masked query bases in lower case, headers and footer;
    the "Posted date" line (the database file's time) is left out as in the reference's test."""
    s = searcher(p, (G / "comparison.matrix").read_text(), "comparison.matrix", (G / "db.fa").read_text())
    recs = api.read_fasta_records((G / "query.fa").read_text())
    enc = [api.encode(x) for _, _, x in recs]
    res = s.search(enc, [i for i, _, _ in recs])
    txt = res.pairwise(enc, [d for _, d, _ in recs], "db.fa")
    want = "".join(ln for ln in (G / f"expected_pairwise_{name}.ncbi-2.17.1.txt").read_text().splitlines(True)
                   if not ln.startswith("    Posted date:"))
    assert txt == want


def test_twobit_databases_match_oracle(tmp_path):
    """Searches against .2bit databases (seq/twobit.rs): the reference's alu.2bit, and a synthetic
    library with N blocks, each against the oracle's own .2bit reader."""
    from twobit_util import write_twobit
    import re
    qf = (G / "query.fa").read_text()
    _, db, _ = synth.workload("small", scale=0.3)
    rng = np.random.default_rng(9)
    recs = []
    for n, sq in db:
        b = bytearray(sq.tobytes())
        for _ in range(2):
            a = int(rng.integers(0, len(b)))
            b[a:a + 30] = b"N" * len(b[a:a + 30])
        recs.append((n, bytes(b)))
    syn = tmp_path / "lib.2bit"
    write_twobit(syn, recs)
    sq, _, prm = synth.workload("small", scale=0.3)
    sqf = synth.to_fasta([n for n, _ in sq], [x for _, x in sq])
    cases = [(G / "alu.2bit", qf, (G / "comparison.matrix").read_text(), "comparison.matrix",
              dict(O.RM_PARAMS, mask_level=80, complexity_adjust=1, dust=1)),
             (syn, sqf, synth.MATRIX_TEXT, synth.MATRIX_NAME, dict(prm, **synth.RM_FLAGS))]
    for path, q, mt, mname, p in cases:
        m = api.ScoreMatrix.from_text(mt, mname)
        sp = api.SearchParams(gap_open=p["gap_open"], gap_extend=p["gap_extend"], word_size=p["word_size"],
                              xdrop_ungap=p["xdrop_ungap"], xdrop_gap=p["xdrop_gap"],
                              xdrop_gap_final=p["xdrop_gap_final"], min_raw_gapped_score=p["min_raw_gapped_score"],
                              complexity_adjust=bool(p.get("complexity_adjust")), dust=bool(p.get("dust")),
                              mask_level=p.get("mask_level", -1))
        s = api.Searcher(sp, m, api.SubjectDb.from_twobit(path))
        qr = api.read_fasta(q)
        got = s.search([api.encode(x) for _, x in qr], [n for n, _ in qr]).tabular(FIELDS)
        mfile = tmp_path / mname
        mfile.write_text(mt)
        qfile = tmp_path / "q.fa"
        qfile.write_text(q)
        args = ["--db", str(path), "--query", str(qfile), "--matrix", str(mfile), "--gapopen", str(p["gap_open"]),
                "--gapextend", str(p["gap_extend"]), "--word-size", str(p["word_size"]),
                "--xdrop-ungap", str(p["xdrop_ungap"]), "--xdrop-gap", str(p["xdrop_gap"]),
                "--xdrop-gap-final", str(p["xdrop_gap_final"]),
                "--min-raw-gapped-score", str(p["min_raw_gapped_score"]), "--dust", "yes" if p.get("dust") else "no",
                "--mask-level", str(p.get("mask_level", 101)), "--outfmt", FIELDS, "--num-threads", "8"]
        if p.get("complexity_adjust"):
            args.append("--complexity-adjust")
        want = O.run_cli(args)
        assert got.count("\n") > 2
        assert got == want


def test_gilist_matches_oracle(tmp_path):
    qf, dbf, p = synthetic("small", 0.3, synth.RM_FLAGS)
    sdb = api.SubjectDb.from_fasta(dbf)
    pick = sdb.ids[::3]
    s = api.Searcher(api.SearchParams(gap_open=p["gap_open"], gap_extend=p["gap_extend"], word_size=p["word_size"],
                                      xdrop_ungap=p["xdrop_ungap"], xdrop_gap=p["xdrop_gap"],
                                      xdrop_gap_final=p["xdrop_gap_final"],
                                      min_raw_gapped_score=p["min_raw_gapped_score"],
                                      complexity_adjust=bool(p.get("complexity_adjust")), mask_level=p["mask_level"]),
                     api.ScoreMatrix.from_text(synth.MATRIX_TEXT, synth.MATRIX_NAME), sdb.select(pick))
    qr = api.read_fasta(qf)
    got = s.search([api.encode(x) for _, x in qr], [n for n, _ in qr]).tabular(FIELDS)
    for name, text in (("db.fa", dbf), ("q.fa", qf), (synth.MATRIX_NAME, synth.MATRIX_TEXT),
                       ("gi.txt", "\n".join(pick) + "\n")):
        (tmp_path / name).write_text(text)
    want = O.run_cli(["--db", str(tmp_path / "db.fa"), "--query", str(tmp_path / "q.fa"),
                      "--matrix", str(tmp_path / synth.MATRIX_NAME), "--gilist", str(tmp_path / "gi.txt"),
                      "--gapopen", str(p["gap_open"]), "--gapextend", str(p["gap_extend"]),
                      "--word-size", str(p["word_size"]), "--xdrop-ungap", str(p["xdrop_ungap"]),
                      "--xdrop-gap", str(p["xdrop_gap"]), "--xdrop-gap-final", str(p["xdrop_gap_final"]),
                      "--min-raw-gapped-score", str(p["min_raw_gapped_score"]), "--dust", "no",
                      "--mask-level", str(p["mask_level"]), "--complexity-adjust", "--outfmt", FIELDS])
    assert got.count("\n") > 2
    assert got == want


# ---- the reference's chr22 goldens through the device path --------------------------------

def _stage_lines(got: np.ndarray, stage: int) -> str:
    if stage == 0:
        lines = sorted(f"SEED strand={'+-'[r[0]]} q={r[1]} s={r[2]}" for r in got.tolist())
    else:
        lines = [f"UNGAP strand={'+-'[r[0]]} qs={r[1]} qe={r[2]} ss={r[3]} se={r[4]} score={np.int32(r[5])}"
                 for r in got.tolist()]
    return "".join(ln + "\n" for ln in lines)


@pytest.mark.parametrize("stage,key", [(0, "seeds"), (1, "ungapped")])
def test_chr22_stage_goldens_through_gpu(stage, key):
    """The reference's chr22 regression goldens (rmblast-lib/tests/dedup_seeds_regression.rs and
    ungapped_regression.rs): chr22 in its 50 NCBI chunks of ~1 Mb against alu.2bit at word 14,
    through the device lookup tables, scan, exact word extension, ungapped extension and
    diagonal-hash dedup (stage taps 0 and 1), 247,629 records each, content and order, compared
    with the goldens' SHA-256."""
    import chr22_fixture as F
    _, seq = F.chr22()
    p = F.STAGE_PARAMS
    m = api.ScoreMatrix.from_text((G / "comparison.matrix").read_text(), "comparison.matrix")
    sp = api.SearchParams(gap_open=p["gap_open"], gap_extend=p["gap_extend"], word_size=p["word_size"],
                          xdrop_ungap=p["xdrop_ungap"], xdrop_gap=p["xdrop_gap"], xdrop_gap_final=p["xdrop_gap_final"],
                          min_raw_gapped_score=p["min_raw_gapped_score"], complexity_adjust=True, dust=False,
                          mask_level=p["mask_level"])
    s = api.Searcher(sp, m, api.SubjectDb.from_twobit(G / "alu.2bit"))
    q = api.encode(seq)
    chunks = [np.concatenate([q[:1], q[1 + a:1 + b], q[-1:]]) for a, b in F.chunks(len(seq))]
    assert len(chunks) == 50
    text = _stage_lines(s.stage(chunks, stage), stage)
    s.close()
    want = F.stage_digests()[key]
    assert F.digest(text) == (want["lines"], want["sha256"])


def test_chr22_chunked_golden_through_c_abi():
    """rmblastn/tests/cli.rs:246-274: chr22 30-33 Mb (3 Mb, three chunks) against db.fa at word 7,
    DUST on, masklevel 80, through rmb_search_batch's multi-chunk path, against NCBI 2.17.1's
    4,236 lines byte for byte."""
    import chr22_fixture as F
    _, seq = F.chr22()
    p = dict(gap_open=20, gap_extend=5, word_size=7, xdrop_ungap=20, xdrop_gap=30, xdrop_gap_final=100,
             min_raw_gapped_score=200, mask_level=80, dust=1)
    s = searcher(p, (G / "comparison.matrix").read_text(), "comparison.matrix", (G / "db.fa").read_text())
    res = s.search([api.encode(seq[30_000_000:33_000_000])], ["chr22_30M_33M"])
    txt = res.tabular("6 score qseqid qstart qend sstrand sseqid sstart send")
    s.close()
    assert txt.count("\n") == 4236
    assert txt == F.chunked_golden()


# ---- the configurations at full or near-full size, and the pipelines ----------------------

def _config_case(name: str, scale: float, **kw):
    qf, dbf, p = synthetic(name, scale, synth.RM_FLAGS)
    s = searcher(p, synth.MATRIX_TEXT, synth.MATRIX_NAME, dbf, **kw)
    recs = api.read_fasta(qf)
    res = s.search([api.encode(x) for _, x in recs], [n for n, _ in recs])
    txt = res.tabular(FIELDS)
    s.close()
    want, ctr, _ = O.search_text(qf, dbf, synth.MATRIX_TEXT, synth.MATRIX_NAME, p, FIELDS, threads=16)
    return txt, want, res, ctr


def test_small_workload_full_size_matches_oracle():
    """The small workload at its full size: the 100 kb genome with 300 planted copies against 50 consensi,
    word 7, every line against the oracle."""
    txt, want, res, ctr = _config_case("small", 1.0)
    assert txt == want
    assert txt.count("\n") > 50
    assert res.counters["ungapped"] == ctr["ungapped"]


def test_plain_workload_full_size_matches_oracle():
    """The plain workload at its full size: all 1,000 chunks of 60 kb (60 Mb) against the 2,000-consensus
    library, word 11, through the batched pipeline (tuned defaults, the device chain as a graph); every one of the
    ~25,000 lines against the oracle (about a minute on 16 host cores)."""
    txt, want, res, ctr = _config_case("plain", 1.0)
    assert txt.count("\n") > 20000
    assert txt == want
    assert res.counters["ungapped"] == ctr["ungapped"] and res.counters["prelims"] >= ctr["prelims"]


def test_plain_workload_fifty_chunks_matches_oracle():
    """The plain workload's shape at 50 of its 1,000 chunks of 60 kb (3 Mb) against the 2,000-consensus
    library, word 11."""
    txt, want, res, ctr = _config_case("plain", 0.05)
    assert txt.count("\n") > 500
    assert txt == want
    assert res.counters["ungapped"] == ctr["ungapped"]


@pytest.mark.parametrize("schedule", [1, 2])
def test_batched_workload_learned_order_matches_oracle(schedule):
    """The batched workload: chunks of 1-200 kb through the batched pipeline with the learned record order
    (the committed network; front-loaded and full cost order), every line against the oracle."""
    txt, want, res, ctr = _config_case("batched", 0.005, schedule=schedule)
    assert txt.count("\n") > 500
    assert txt == want
    assert res.counters["ungapped"] == ctr["ungapped"]


@pytest.mark.parametrize("name,scale", [("plain", 0.02), ("batched", 0.002)])
def test_plain_pipeline_matches_oracle(name, scale):
    """The plain pipeline (one launch per stage, one work item per thread, arrival order): the
    same text as the oracle, and the same DP cells as the batched pipeline (only the
    assignment of work to threads differs)."""
    txt, want, res, ctr = _config_case(name, scale, pipeline=1)
    assert txt == want
    txt_b, _, res_b, _ = _config_case(name, scale, pipeline=0)
    assert txt_b == txt
    for k in ("word_hits", "ungapped", "prelim_dp", "prelims", "so_cells", "tb_cells"):
        assert res.counters[k] == res_b.counters[k], k


@pytest.mark.parametrize("name,scale", [("plain", 0.01), ("allvsall", 0.03)])
def test_tune_knobs_leave_output_unchanged(name, scale):
    """The launch knobs (rmb_tune) shape only how the work is laid out: extreme settings of each,
    both dedup paths (the fused bucket-parallel dedup-extension and the extend-then-dedup pair),
    one and two pipeline lanes, the device chain as a graph or stage by stage, and the
    autotuner's pick give the oracle's text byte for byte."""
    qf, dbf, p = synthetic(name, scale, synth.RM_FLAGS)
    s = searcher(p, synth.MATRIX_TEXT, synth.MATRIX_NAME, dbf)
    recs = api.read_fasta(qf)
    enc = [api.encode(x) for _, x in recs]
    ids = [n for n, _ in recs]
    want, _, _ = O.search_text(qf, dbf, synth.MATRIX_TEXT, synth.MATRIX_NAME, p, FIELDS, threads=16)
    assert want.count("\n") > 20
    default = s.tune()
    assert s.search(enc, ids).tabular(FIELDS) == want
    for knobs in (dict(prelim_group=4), dict(prelim_group=16), dict(prelim_window=16, prelim_budget_div=16),
                  dict(prelim_blocks_per_sm=1, ungapped_blocks_per_sm=1), dict(prelim_budget_div=4096), dict(lanes=2),
                  dict(graph=0), dict(graph=2), dict(graph=0, lanes=2), dict(dedup_extend_hits_per_pair=0),
                  dict(dedup_extend_hits_per_pair=-1)):
        s.set_tune(dict(default, **knobs))
        assert s.search(enc, ids).tabular(FIELDS) == want, knobs
    s.set_tune(default)
    with pytest.raises(api.RmbError):
        s.set_tune(dict(default, prelim_group=5))
    r = s.autotune(enc[:max(1, len(enc) // 2)])
    assert r["best_ms"] <= r["default_ms"] and r["tune"] == s.tune()
    assert s.search(enc, ids).tabular(FIELDS) == want
    s.close()
