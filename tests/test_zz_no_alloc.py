"""rmb_traceback_noalloc: the traceback for callers that may not allocate device memory.

Some callers cannot call cudaMalloc: code embedded in a process whose device memory belongs to
another allocator (a caching allocator that must account for every byte, a stream-ordered pool)
or code running where an allocation could fail or stall.  For them the library keeps the
traceback's scratch in a fixed 32 MiB array and takes every input and output as device memory
the caller owns.  This test (collected last, so a failure here comes after every other test)
checks that two calls in a row give exactly the records of the allocating path's traceback stage
(rmb_debug_stage stage 4) for the same prelim HSPs, and those records against the oracle's for the
same pair; the path is integer arithmetic, so the comparison is exact.  The test allocates its own inputs and outputs with torch; the entry point
allocates nothing.
"""
import ctypes as C

import numpy as np
import pytest

import oracle_ref as O
from rmblast_b200 import api, build

pytestmark = pytest.mark.gpu
G = O.GOLDEN
COMP = np.array([3, 2, 1, 0, 5, 4, 7, 6, 8, 9, 13, 12, 11, 10, 14, 15], np.uint8)


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def _lib():
    lib = api.lib()
    p8, p32 = C.c_void_p, C.c_void_p
    lib.rmb_traceback_noalloc.argtypes = [C.c_int32, p8, p8, C.c_uint32, p8, p8, C.c_uint32, p32, C.c_uint32,
                                          C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_int32), p32, p32, C.c_uint32,
                                          C.c_void_p, C.c_char_p, C.c_size_t]
    return lib


def _dev(a: np.ndarray):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_traceback_noalloc_matches_stage_four_twice():
    import torch
    lib = _lib()
    mt = (G / "comparison.matrix").read_text()
    m = api.ScoreMatrix.from_text(mt, "comparison.matrix")
    sp = api.SearchParams(gap_open=20, gap_extend=5, word_size=14, xdrop_ungap=400, xdrop_gap=100,
                          xdrop_gap_final=200, min_raw_gapped_score=200, mask_level=101)
    queries = api.read_fasta((G / "query.fa").read_text())
    subjects = api.read_fasta((G / "db_dash.fa").read_text())
    scores = (C.c_int32 * 256)(*m.scores.ravel().tolist())
    checked = 0
    for sname, sseq in subjects[:8]:
        s = api.Searcher(sp, m, api.SubjectDb.from_records([(sname, sseq)]))
        align = api.encode(sseq)  # the subject with its ambiguity codes, as the traceback reads it
        align_rc = COMP[align[::-1]]
        for qname, qseq in queries[:2]:
            q = api.encode(qseq)
            pre = s.stage([q], 2)
            want = s.stage([q], 4)
            if len(pre) == 0:
                continue
            assert len(want) == len(pre)
            # the allocating path's stage 4 is itself the oracle's, for this very pair
            oracle = O.stage_text(f">{qname}\n{qseq.decode()}\n", f">{sname}\n{sseq.decode()}\n", mt,
                                  "comparison.matrix", dict(O.RM_PARAMS, mask_level=101), 4)
            assert np.array_equal(want, oracle), (sname, qname)
            d = [_dev(x) for x in (q, COMP[q[::-1]], align, align_rc, pre.astype(np.uint32))]
            ops_cap = 4096
            for call in range(2):
                out = torch.full((len(pre), 9), 7, dtype=torch.int32, device="cuda")
                ops = torch.zeros((len(pre), ops_cap), dtype=torch.int32, device="cuda")
                err = C.create_string_buffer(512)
                rc = lib.rmb_traceback_noalloc(0, d[0].data_ptr(), d[1].data_ptr(), len(q) - 2, d[2].data_ptr(),
                                               d[3].data_ptr(), len(align) - 2, d[4].data_ptr(), len(pre), 20, 5, 200,
                                               scores, out.data_ptr(), ops.data_ptr(), ops_cap, None, err, 512)
                assert rc == 0, err.value
                got = out.cpu().numpy().view(np.uint32)
                assert np.array_equal(got, want), (sname, qname, call)
            checked += len(pre)
        s.close()
    assert checked > 5


def test_traceback_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    lib = _lib()
    buf = torch.zeros(64, dtype=torch.uint8, device="cuda")
    err = C.create_string_buffer(512)
    scores = (C.c_int32 * 256)()
    p = buf.data_ptr()
    # 8 x (5,000,000 + 2) bytes of row table alone exceed the scratch: refused before any launch
    rc = lib.rmb_traceback_noalloc(0, p, p, 5_000_000, p, p, 10, p, 1, 20, 5, 200, scores, p, p, 16, None, err, 512)
    assert rc == 5 and b"32 MiB" in err.value


def test_traceback_noalloc_skips_records_outside_the_sequences():
    """Records from the caller are checked before any sequence byte is read: a box or seed past
    either sequence, or a strand other than 0/1, comes back with status 4, and the valid records
    of the same call still align as the allocating path does."""
    import torch
    lib = _lib()
    mt = (G / "comparison.matrix").read_text()
    m = api.ScoreMatrix.from_text(mt, "comparison.matrix")
    sp = api.SearchParams(gap_open=20, gap_extend=5, word_size=14, xdrop_ungap=400, xdrop_gap=100,
                          xdrop_gap_final=200, min_raw_gapped_score=200, mask_level=101)
    qname, qseq = api.read_fasta((G / "query.fa").read_text())[0]
    scores = (C.c_int32 * 256)(*m.scores.ravel().tolist())
    for sname, sseq in api.read_fasta((G / "db.fa").read_text()):
        s = api.Searcher(sp, m, api.SubjectDb.from_records([(sname, sseq)]))
        q = api.encode(qseq)
        pre = s.stage([q], 2)
        want = s.stage([q], 4)
        s.close()
        if len(pre):
            break
    assert len(pre)
    align = api.encode(sseq)
    qlen, slen = len(q) - 2, len(align) - 2
    bad = []
    for k, (col, val) in enumerate([(0, 2), (2, qlen + 1), (4, slen + 7), (6, qlen), (7, slen), (1, qlen + 5)]):
        r = pre[k % len(pre)].astype(np.uint32).copy()
        r[col] = val
        bad.append(r)
    recs = np.concatenate([pre.astype(np.uint32), np.array(bad, np.uint32)])
    d = [_dev(x) for x in (q, COMP[q[::-1]], align, COMP[align[::-1]], recs)]
    out = torch.full((len(recs), 9), 7, dtype=torch.int32, device="cuda")
    ops = torch.zeros((len(recs), 4096), dtype=torch.int32, device="cuda")
    err = C.create_string_buffer(512)
    torch.cuda.set_device(0)
    rc = lib.rmb_traceback_noalloc(0, d[0].data_ptr(), d[1].data_ptr(), qlen, d[2].data_ptr(), d[3].data_ptr(), slen,
                                   d[4].data_ptr(), len(recs), 20, 5, 200, scores, out.data_ptr(), ops.data_ptr(),
                                   4096, None, err, 512)
    assert rc == 0, err.value
    assert torch.cuda.current_device() == 0
    got = out.cpu().numpy().view(np.uint32)
    assert np.array_equal(got[:len(pre)], want)
    assert (got[len(pre):, 1] == 4).all()
    assert (got[len(pre):, 2:] == 0).all()
