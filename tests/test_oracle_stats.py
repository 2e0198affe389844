"""Pins the oracle's E-value statistics to the reference's known answers
(rmblast-stats/rmstats/tests/stats_tests.rs, rmblast-lib/src/matrix.rs tests): the built-in
table, the table / command line / matrix comment / none order, the length adjustment's fixed
point, and the E-value and bit-score formulas with their no-statistics values."""
import ctypes as C
import math

import oracle_ref as O

G = O.GOLDEN
CMP = (G / "comparison.matrix").read_text()


def stats(name, go, ge, cli=None, text=CMP):
    lib = O.lib()
    lib.rmbo_stats.argtypes = [C.c_char_p, C.c_char_p, C.c_int32, C.c_int32, C.POINTER(C.c_double),
                               C.POINTER(C.c_double), C.c_char_p, C.c_size_t]
    out = (C.c_double * 6)()
    err = C.create_string_buffer(256)
    c = (C.c_double * 4)(*cli) if cli else None
    assert lib.rmbo_stats(name.encode(), text.encode(), go, ge, c, out, err, 256) == 0, err.value
    return list(out)


def evalue(ka, score, qlen, dblen, dbnum):
    lib = O.lib()
    lib.rmbo_evalue.argtypes = [C.POINTER(C.c_double), C.c_int32, C.c_int32, C.c_int64, C.c_int32,
                                C.POINTER(C.c_double)]
    out = (C.c_double * 3)()
    lib.rmbo_evalue((C.c_double * 5)(*ka[:5]), score, qlen, dblen, dbnum, out)
    return list(out)


def length_adjustment(k, alpha_d_lambda, beta, m, n, nseq):
    lib = O.lib()
    lib.rmbo_length_adjustment.restype = C.c_int32
    lib.rmbo_length_adjustment.argtypes = [C.c_double] * 4 + [C.c_int32, C.c_int64, C.c_int32,
                                                              C.POINTER(C.c_int32)]
    conv = C.c_int32()
    ell = lib.rmbo_length_adjustment(k, math.log(k), alpha_d_lambda, beta, m, n, nseq, C.byref(conv))
    return ell, bool(conv.value)


def test_table_rows():
    s = stats("14p35g.matrix", 29, 6)
    assert s[:3] == [0.1241860392, 0.2565118357, 0.3349210581] and s[5] == 1
    assert stats("14P35G.MATRIX", 29, 6)[5] == 1                    # case-insensitive base name
    assert stats("/some/dir/14p35g.matrix", 29, 6)[5] == 1           # base name of a path
    c = stats("comparison.matrix", 20, 5)
    assert abs(c[0] - 0.0983622300) < 1e-10 and abs(c[1] - 0.0789918084) < 1e-10
    assert stats("nosuch.matrix", 29, 6)[0] == -1.0                  # no statistics
    assert stats("comparison.matrix", 20, 6)[0] == -1.0              # gap costs not fitted


def test_source_order():
    assert stats("25p41g.matrix", 22, 5)[5] == 1
    s = stats("custom.matrix", 20, 5, cli=(0.1227, 0.0919, 1.5, -4.0))
    assert s[:5] == [0.1227, 0.0919, 0.1227 / 1.5, 1.5, -4.0] and s[5] == 2
    # the table wins over the command line; its alpha/beta then come from the command line
    t = stats("25p41g.matrix", 22, 5, cli=(0.1227, 0.0919, 1.5, -4.0))
    assert t[5] == 1 and t[3:5] == [1.5, -4.0]
    karlin = "# KARLIN lambda 0.1276 K 0.0179 H 0.3562 beta -26.84\n" + CMP
    k = stats("custom.matrix", 20, 5, text=karlin)
    assert k[5] == 3 and k[0] == 0.1276 and k[1] == 0.0179 and abs(k[3] - 0.1276 / 0.3562) < 1e-15
    assert k[4] == -26.84
    assert stats("custom.matrix", 20, 5)[5] == 0


def test_length_adjustment_fixed_point():
    s = stats("25p41g.matrix", 22, 5)
    lam, k, h = s[0], s[1], s[2]
    alpha = lam / h
    m, n, nseq = 64_444_167, 1_838_298, 1_580
    ell, conv = length_adjustment(k, alpha / lam, 0.0, m, n, nseq)
    assert conv and ell > 0

    def f(x):
        return (alpha / lam) * (math.log(k) + math.log((m - x) * (n - nseq * x)))
    assert f(ell) >= ell
    assert f(ell + 1) < ell + 1 + 1.0
    assert length_adjustment(1e-9, 2.0, 0.0, 10, 10, 1) == (0, False)


def test_evalue_bitscore_and_search_space():
    s = stats("20p41g.matrix", 25, 5)
    e, b, sp = evalue(s, 250, 1_000_000, 1_838_298, 1_580)
    ell, _ = length_adjustment(s[1], s[3] / s[0], s[4], 1_000_000, 1_838_298, 1_580)
    assert ell > 0
    assert sp == (1_838_298 - 1_580 * ell) * (1_000_000 - ell)
    assert e == sp * math.exp(-s[0] * 250 + math.log(s[1]))
    assert abs(b - (250 * s[0] - math.log(s[1])) / math.log(2)) < 1e-12
    none = stats("comparison.matrix", 20, 6)
    assert evalue(none, 250, 1_000_000, 1_838_298, 1_580) == [1.0, 0.0, 0.0]
