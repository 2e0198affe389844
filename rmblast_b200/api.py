"""Python host over the C ABI of include/rmb_gpu.h (librmb_b200.so).

Mirrors the reference's library surface for the search path:
  ScoreMatrix.from_text/from_file   rmblast-lib/src/matrix.rs:76-224
  SearchParams                       rmblast-lib/src/options.rs:12-104
  SubjectDb.from_fasta / from_records  rmblast-lib/src/seq/mod.rs:155-291 (CRandom decode)
  Searcher.search                    rmblastn/src/main.rs:1133-1236 search_db_parallel, per query
  Searcher.stage                     search/engine.rs:796-832 stage taps (seeds, ungapped, prelims)
  Results.tabular                    rmblast-lib/src/output.rs:294-367 write_tabular

There is no CPU path: every call goes to the CUDA library, and importing this module
fails if librmb_b200.so was not built.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "lib" / "librmb_b200.so"


class RmbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"rmb error {code}: {msg}")
        self.code = code


class _Params(C.Structure):
    _fields_ = [(n, C.c_int32) for n in (
        "gap_open", "gap_extend", "word_size", "xdrop_ungap", "xdrop_gap", "xdrop_gap_final",
        "min_raw_gapped_score", "complexity_adjust", "dust", "mask_level", "ungapped_cutoff",
        "device", "schedule", "kernels", "pipeline")] + [(n, C.c_double) for n in (
        "ka_lambda", "ka_k", "ka_h", "ka_alpha", "ka_beta", "evalue")]


class _Tune(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("prelim_group", "prelim_blocks_per_sm", "prelim_window", "prelim_budget_div",
                                         "ungapped_blocks_per_sm", "dedup_extend_hits_per_pair", "lanes", "graph")]


class _Hsp(C.Structure):
    _fields_ = [("score", C.c_int32)] + [(n, C.c_uint32) for n in (
        "q_start", "q_end", "q_len", "s_start", "s_end", "s_len", "subject_oid", "strand", "matches",
        "mismatches", "query_gaps", "subject_gaps", "transitions", "transversions", "cpg_sites")] + [
        ("perc_sub", C.c_float), ("perc_query_gap", C.c_float), ("perc_db_gap", C.c_float),
        ("kdiv", C.c_double), ("cpg_kdiv", C.c_double), ("ops_off", C.c_uint64), ("ops_len", C.c_uint32),
        ("aln_len", C.c_uint32), ("seq_off", C.c_uint64), ("evalue", C.c_double), ("bitscore", C.c_double)]


class _Counters(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in (
        "word_hits", "seeds", "ungapped", "prelim_dp", "prelims", "tb_dp", "finals", "so_cells", "tb_cells")] + [
        (n, C.c_double) for n in ("ms_lookup", "ms_scan", "ms_ungapped", "ms_dedup", "ms_prelim_dp", "ms_host_2a",
                                  "ms_traceback", "ms_host_2b", "gpu_ms_scan", "gpu_ms_ungapped", "gpu_ms_dedup",
                                  "gpu_ms_prelim", "gpu_ms_traceback", "gpu_ms_lookup")] + [("launches", C.c_uint64)] + [
        ("gpu_ms_prelim_main", C.c_double), ("so_cells_main", C.c_uint64), ("gpu_ms_dust", C.c_double),
        ("gpu_ms_sched", C.c_double)]


class _Results(C.Structure):
    _fields_ = [("n_queries", C.c_uint32), ("query_off", C.POINTER(C.c_uint64)), ("n_hsps", C.c_uint64),
                ("hsps", C.POINTER(_Hsp)), ("ops", C.POINTER(C.c_uint32)), ("q_seq", C.POINTER(C.c_uint8)),
                ("s_seq", C.POINTER(C.c_uint8)), ("counters", _Counters)]


def load_library(path: Path = LIB_PATH) -> C.CDLL:
    if not path.exists():
        raise ImportError(f"{path} is missing: build it with `python -m rmblast_b200.build`")
    lib = C.CDLL(str(path))
    u8p, u8pp = C.POINTER(C.c_uint8), C.POINTER(C.POINTER(C.c_uint8))
    lib.rmb_ctx_create.argtypes = [C.POINTER(_Params), C.POINTER(C.c_int32), C.POINTER(C.c_double), C.c_double,
                                   C.c_char_p, C.POINTER(C.c_void_p), C.c_char_p, C.c_size_t]
    lib.rmb_db_load.argtypes = [C.c_void_p, C.c_uint32, u8pp, C.POINTER(C.c_uint32), u8pp,
                                C.POINTER(C.c_char_p), C.c_char_p, C.c_size_t]
    lib.rmb_search_batch.argtypes = [C.c_void_p, C.c_uint32, u8pp, C.POINTER(C.c_uint32),
                                     C.POINTER(C.POINTER(_Results)), C.c_char_p, C.c_size_t]
    lib.rmb_format_tabular.argtypes = [C.c_void_p, C.POINTER(_Results), C.POINTER(C.c_char_p), C.c_char_p,
                                       C.POINTER(C.c_void_p), C.POINTER(C.c_size_t), C.c_char_p, C.c_size_t]
    lib.rmb_debug_stage.argtypes = [C.c_void_p, C.c_uint32, u8pp, C.POINTER(C.c_uint32), C.c_int32,
                                    C.POINTER(C.POINTER(C.c_uint32)), C.POINTER(C.c_uint64), C.c_char_p, C.c_size_t]
    lib.rmb_matrix_parse.argtypes = [C.c_char_p, C.POINTER(C.c_int32), C.POINTER(C.c_double),
                                     C.POINTER(C.c_double), C.c_char_p, C.c_size_t]
    lib.rmb_encode_iupac.argtypes = [C.c_char_p, C.c_size_t, u8p]
    lib.rmb_encode_iupac.restype = None
    lib.rmb_resolve_subject.argtypes = [u8p, C.c_uint32, u8p, u8p, C.POINTER(C.c_int32)]
    lib.rmb_resolve_subject.restype = None
    lib.rmb_results_free.argtypes = [C.POINTER(_Results)]
    lib.rmb_results_free.restype = None
    lib.rmb_text_free.argtypes = [C.c_void_p]
    lib.rmb_text_free.restype = None
    lib.rmb_ctx_destroy.argtypes = [C.c_void_p]
    lib.rmb_tune_get.argtypes = [C.c_void_p, C.POINTER(_Tune)]
    lib.rmb_tune_set.argtypes = [C.c_void_p, C.POINTER(_Tune), C.c_char_p, C.c_size_t]
    lib.rmb_autotune.argtypes = [C.c_void_p, C.c_uint32, u8pp, C.POINTER(C.c_uint32), C.POINTER(_Tune),
                                 C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_char_p, C.c_size_t]
    lib.rmb_ctx_destroy.restype = None
    lib.rmb_version.restype = C.c_char_p
    lib.rmb_queries_upload.argtypes = [C.c_void_p, C.c_uint32, u8pp, C.POINTER(C.c_uint32), C.POINTER(C.c_void_p),
                                       C.c_char_p, C.c_size_t]
    lib.rmb_search_resident.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.POINTER(_Results)), C.c_char_p,
                                        C.c_size_t]
    lib.rmb_queries_free.argtypes = [C.c_void_p]
    lib.rmb_queries_free.restype = None
    lib.rmb_probe_int32_peak.argtypes = [C.c_int32, C.POINTER(C.c_double), C.c_char_p, C.c_size_t]
    fp = C.POINTER(C.c_float)
    lib.rmb_sched_set_model.argtypes = [C.c_void_p, fp, C.c_uint32, C.c_char_p, C.c_size_t]
    lib.rmb_sched_log.argtypes = [C.c_void_p, C.c_uint32, u8pp, C.POINTER(C.c_uint32), C.POINTER(fp),
                                  C.POINTER(C.POINTER(C.c_uint32)), C.POINTER(C.c_uint64), C.c_char_p, C.c_size_t]
    lib.rmb_sched_train.argtypes = [C.c_int32, fp, fp, C.c_uint64, C.c_uint32, C.c_uint32, C.c_float, C.c_uint64,
                                    C.c_float, fp, fp, C.c_char_p, C.c_size_t]
    lib.rmb_sched_grad.argtypes = [C.c_int32, fp, fp, fp, C.c_uint32, fp, fp, C.c_char_p, C.c_size_t]
    lib.rmb_sched_predict.argtypes = [C.c_int32, fp, fp, C.c_uint64, fp, C.c_char_p, C.c_size_t]
    return lib


def device_name(device: int = 0) -> tuple[str, int]:
    """(name, SM count) of a CUDA device, through the CUDA runtime the library links."""
    import torch
    pr = torch.cuda.get_device_properties(device)
    return pr.name, pr.multi_processor_count


def int32_peak_tops(device: int = 0) -> float:
    """Sustained int32 add/max throughput of the device (Tops/s), measured by the library."""
    v = C.c_double()
    err = C.create_string_buffer(256)
    _check(lib().rmb_probe_int32_peak(device, C.byref(v), err, 256), err)
    return v.value


_LIB: C.CDLL | None = None


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        _LIB = load_library()
    return _LIB


def _check(rc: int, err: C.Array) -> None:
    if rc != 0:
        raise RmbError(rc, err.value.decode(errors="replace"))


def encode(ascii_seq: bytes | np.ndarray) -> np.ndarray:
    """encoding.rs:125 encode_iupac: ASCII -> sentinel-wrapped BLASTNA."""
    b = bytes(ascii_seq) if not isinstance(ascii_seq, np.ndarray) else ascii_seq.tobytes()
    out = np.empty(len(b) + 2, dtype=np.uint8)
    lib().rmb_encode_iupac(b, len(b), out.ctypes.data_as(C.POINTER(C.c_uint8)))
    return out


def read_fasta_records(text: str) -> list[tuple[str, str, bytes]]:
    """seq/fasta.rs:83-150 FastaReader: (id, defline, sequence) per record; the defline is the
    header after '>' with only its line ending removed."""
    recs, head, buf = [], None, []
    for line in text.split("\n"):
        line = line.rstrip("\r")
        if line.startswith(">"):
            if head is not None:
                recs.append((head.split()[0], head, "".join(buf).encode()))
            head = line[1:]
            buf = []
        elif line.strip():
            buf.append(line.strip())
    if head is not None:
        recs.append((head.split()[0], head, "".join(buf).encode()))
    return recs


def read_fasta(text: str) -> list[tuple[str, bytes]]:
    """seq/fasta.rs:83 FastaReader: (id, sequence) per record."""
    recs, name, buf = [], None, []
    for line in text.splitlines():
        if line.startswith(">"):
            if name is not None:
                recs.append((name, "".join(buf).encode()))
            name = line[1:].split()[0]
            buf = []
        elif line.strip():
            buf.append(line.strip())
    if name is not None:
        recs.append((name, "".join(buf).encode()))
    return recs


@dataclass
class ScoreMatrix:
    scores: np.ndarray  # int32 (16, 16), scores[q][s]
    freqs: np.ndarray   # float64 (16,)
    lambda_: float
    name: str
    text: str | None = None  # the file text (its "# KARLIN" line feeds the E-value statistics)

    @classmethod
    def from_text(cls, text: str, name: str = "") -> "ScoreMatrix":
        sc = (C.c_int32 * 256)()
        fr = (C.c_double * 16)()
        lam = C.c_double()
        err = C.create_string_buffer(512)
        _check(lib().rmb_matrix_parse(text.encode(), sc, fr, C.byref(lam), err, 512), err)
        return cls(np.frombuffer(sc, dtype=np.int32).reshape(16, 16).copy(), np.frombuffer(fr).copy(),
                   lam.value, name, text)

    @classmethod
    def from_file(cls, path: str) -> "ScoreMatrix":
        return cls.from_text(Path(path).read_text(), path)


@dataclass
class SearchParams:
    """options.rs:12-104 (with rmblastn's CLI defaults, main.rs:128-281)."""
    gap_open: int = 20
    gap_extend: int = 5
    word_size: int = 11
    xdrop_ungap: int = 20
    xdrop_gap: int = 30
    xdrop_gap_final: int = 100
    min_raw_gapped_score: int = 0
    complexity_adjust: bool = False
    dust: bool = False
    mask_level: int = -1
    ungapped_cutoff: int = -1
    device: int = 0
    # 0: automatic kernel choice; 1: every preliminary DP on the warp-cooperative kernel
    kernels: int = 0
    # 0: FIFO record queue; 1: learned, the predicted-costliest records first; 2: learned, all in
    # descending predicted cost (Searcher.set_schedule_model)
    schedule: int = 0
    # 0: batched (persistent kernels with device work queues); 1: plain (one launch per stage,
    # one work item per thread in arrival order)
    pipeline: int = 0
    # --evalue threshold (0: off) and the -matrix_lambda/-matrix_k/-matrix_alpha/-matrix_beta
    # statistics overrides (zeros: unset)
    evalue: float = 0.0
    matrix_lambda: float = 0.0
    matrix_k: float = 0.0
    matrix_alpha: float = 0.0
    matrix_beta: float = 0.0

    def _c(self, ka=(-1.0, -1.0, -1.0, 0.0, 0.0)) -> _Params:
        return _Params(self.gap_open, self.gap_extend, self.word_size, self.xdrop_ungap, self.xdrop_gap,
                       self.xdrop_gap_final, self.min_raw_gapped_score, int(self.complexity_adjust), int(self.dust),
                       self.mask_level, self.ungapped_cutoff, self.device, self.schedule, self.kernels,
                       self.pipeline, *ka,
                       self.evalue)


class SubjectDb:
    """seq/mod.rs:155-291: subjects decoded once, ambiguity codes CRandom-resolved."""

    def __init__(self, ids: list[str], plus: list[np.ndarray], masks: list[np.ndarray | None],
                 deflines: list[str] | None = None):
        self.ids, self.plus, self.masks = ids, plus, masks
        self.deflines = deflines  # full FASTA headers (None for a .2bit database: ids only)

    @classmethod
    def from_records(cls, recs: list[tuple[str, bytes | np.ndarray]]) -> "SubjectDb":
        ids, plus, masks = [], [], []
        for name, seq in recs:
            raw = encode(seq)
            n = len(raw) - 2
            p = np.empty_like(raw)
            m = np.zeros(max(n, 1), dtype=np.uint8)
            has = C.c_int32()
            lib().rmb_resolve_subject(raw.ctypes.data_as(C.POINTER(C.c_uint8)), n,
                                      p.ctypes.data_as(C.POINTER(C.c_uint8)), m.ctypes.data_as(C.POINTER(C.c_uint8)),
                                      C.byref(has))
            ids.append(name)
            plus.append(p)
            masks.append(m[:n] if has.value else None)
        return cls(ids, plus, masks)

    @classmethod
    def from_fasta(cls, text: str) -> "SubjectDb":
        recs = read_fasta_records(text)
        db = cls.from_records([(i, s) for i, _, s in recs])
        db.deflines = [d for _, d, _ in recs]
        return db

    @classmethod
    def from_twobit(cls, path: str | Path) -> "SubjectDb":
        """seq/twobit.rs: a UCSC .2bit database (either byte order), its N blocks CRandom-resolved
        with n_mask = N, soft-mask blocks ignored."""
        d = Path(path).read_bytes()
        magic = int.from_bytes(d[0:4], "little")
        order = "little" if magic == 0x1A412743 else "big" if magic == 0x4327411A else None
        if order is None:
            raise ValueError("not a .2bit file (bad signature)")
        r32 = lambda p: int.from_bytes(d[p:p + 4], order)
        count, pos = r32(8), 16
        index = []
        for _ in range(count):
            nl = d[pos]
            name = d[pos + 1:pos + 1 + nl].decode()
            pos += 1 + nl
            index.append((name, r32(pos)))
            pos += 4
        ucsc = np.array([3, 1, 0, 2], dtype=np.uint8)  # UCSC T, C, A, G -> BLASTNA
        dt = np.dtype(np.uint32).newbyteorder("<" if order == "little" else ">")
        ids, plus, masks = [], [], []
        for name, off in index:
            n, nb = r32(off), r32(off + 4)
            starts = np.frombuffer(d, dtype=dt, count=nb, offset=off + 8).astype(np.uint32)
            sizes = np.frombuffer(d, dtype=dt, count=nb, offset=off + 8 + 4 * nb).astype(np.uint32)
            mb = r32(off + 8 + 8 * nb)
            dna_off = off + 8 + 8 * nb + 4 + 8 * mb + 4
            packed = np.frombuffer(d, dtype=np.uint8, count=(n + 3) // 4, offset=dna_off)
            codes = np.stack([(packed >> s) & 3 for s in (6, 4, 2, 0)], axis=1).ravel()[:n]
            p = np.full(n + 2, 15, dtype=np.uint8)
            p[1:n + 1] = ucsc[codes]
            m = np.zeros(max(n, 1), dtype=np.uint8)
            if nb:
                lib().rmb_resolve_twobit_n(n, nb, starts.ctypes.data_as(C.POINTER(C.c_uint32)),
                                           sizes.ctypes.data_as(C.POINTER(C.c_uint32)),
                                           p.ctypes.data_as(C.POINTER(C.c_uint8)), m.ctypes.data_as(C.POINTER(C.c_uint8)))
            ids.append(name)
            plus.append(p)
            masks.append(m[:n] if nb else None)
        return cls(ids, plus, masks)

    def select(self, gilist: list[str]) -> "SubjectDb":
        """main.rs:1444-1470: the subjects named in a gilist (a bare number also names "gi|n"),
        in database order."""
        keep = set()
        for e in (x.strip() for x in gilist):
            if not e:
                continue
            if e.isdigit():
                keep.add("gi|" + e)
            keep.add(e)
        idx = [i for i, n in enumerate(self.ids) if n in keep]
        return SubjectDb([self.ids[i] for i in idx], [self.plus[i] for i in idx], [self.masks[i] for i in idx],
                         [self.deflines[i] for i in idx] if self.deflines else None)

    def total_letters(self) -> int:
        return sum(len(p) - 2 for p in self.plus)


def _ptr_array(arrs: list[np.ndarray | None]):
    t = (C.POINTER(C.c_uint8) * len(arrs))()
    for i, a in enumerate(arrs):
        t[i] = a.ctypes.data_as(C.POINTER(C.c_uint8)) if a is not None else C.POINTER(C.c_uint8)()
    return t


class Results:
    """rmb_results: HSPs per query in the reference's output order."""

    def __init__(self, searcher: "Searcher", ptr, query_ids: list[str]):
        self._s, self._p, self.query_ids = searcher, ptr, query_ids
        self._lib = lib()  # held for __del__, which can run after the module's globals are gone
        r = ptr.contents
        self.n_hsps = int(r.n_hsps)
        c = r.counters
        self.counters = {f: getattr(c, f) for f, _ in _Counters._fields_}

    def hsps(self) -> list[dict]:
        r = self._p.contents
        out = []
        for q in range(r.n_queries):
            for k in range(r.query_off[q], r.query_off[q + 1]):
                h = r.hsps[k]
                out.append({f: getattr(h, f) for f, _ in _Hsp._fields_} | {"query": q})
        return out

    def pairwise(self, queries: list[np.ndarray], query_deflines: list[str], db_name: str, parts: int = 3,
                 db_mtime: int = -1) -> str:
        """rmb_format_pairwise: outfmt 0 for these results (header and footer by `parts`)."""
        s = self._s
        n = len(query_deflines)
        qp = _ptr_array(queries) if queries else None
        ql = (C.c_uint32 * max(n, 1))(*[len(q) - 2 for q in queries]) if queries else (C.c_uint32 * max(n, 1))()
        qd = (C.c_char_p * max(n, 1))(*[d.encode() for d in query_deflines])
        sd = (C.c_char_p * len(s.db.ids))(*[d.encode() for d in s.db.deflines]) if s.db.deflines else None
        txt = C.c_void_p()
        size = C.c_size_t()
        err = C.create_string_buffer(512)
        _check(lib().rmb_format_pairwise(s._ctx, self._p, qp, ql, qd, sd, db_name.encode(), C.c_int64(db_mtime),
                                         parts, C.byref(txt), C.byref(size), err, 512), err)
        try:
            return C.string_at(txt.value, size.value).decode()
        finally:
            lib().rmb_text_free(txt)

    def tabular(self, outfmt: str) -> str:
        ids = (C.c_char_p * max(1, len(self.query_ids)))(*[i.encode() for i in self.query_ids])
        txt = C.c_void_p()
        n = C.c_size_t()
        err = C.create_string_buffer(512)
        _check(lib().rmb_format_tabular(self._s._ctx, self._p, ids, outfmt.encode(), C.byref(txt), C.byref(n), err,
                                        512), err)
        try:
            return C.string_at(txt.value, n.value).decode()
        finally:
            lib().rmb_text_free(txt)

    def __del__(self):
        if getattr(self, "_p", None):
            self._lib.rmb_results_free(self._p)
            self._p = None


class ResidentQueries:
    def __init__(self, h: C.c_void_p, n: int):
        self._h, self.n = h, n
        self._lib = lib()

    def free(self):
        if getattr(self, "_h", None):
            self._lib.rmb_queries_free(self._h)
            self._h = None

    def __del__(self):
        self.free()


SCHED_NF, SCHED_H, SCHED_NET, SCHED_NPARAM = 12, 64, 5057, 5081


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def sched_init(features: np.ndarray, seed: int = 0, targets: np.ndarray | None = None) -> np.ndarray:
    """Initial parameters of the schedule network (He-normal weights, zero hidden biases, the
    output bias at the targets' mean when given) and the normalisation of the given raw features
    (mean, 1/std), in the rmb_sched layout."""
    rng = np.random.default_rng(seed)
    p = np.zeros(SCHED_NPARAM, dtype=np.float32)
    o = 0
    p[o:o + SCHED_NF * SCHED_H] = rng.normal(0, np.sqrt(2.0 / SCHED_NF), SCHED_NF * SCHED_H)
    o += SCHED_NF * SCHED_H + SCHED_H
    p[o:o + SCHED_H * SCHED_H] = rng.normal(0, np.sqrt(2.0 / SCHED_H), SCHED_H * SCHED_H)
    o += SCHED_H * SCHED_H + SCHED_H
    p[o:o + SCHED_H] = rng.normal(0, np.sqrt(1.0 / SCHED_H), SCHED_H)
    if targets is not None and len(targets):
        p[o + SCHED_H] = float(np.mean(targets))
    f = np.asarray(features, dtype=np.float64)
    sd = f.std(axis=0)
    p[SCHED_NET:SCHED_NET + SCHED_NF] = f.mean(axis=0)
    p[SCHED_NET + SCHED_NF:] = np.where(sd > 1e-6, 1.0 / np.maximum(sd, 1e-6), 1.0)
    return p


def sched_train(features: np.ndarray, targets: np.ndarray, params: np.ndarray, epochs: int = 4, batch: int = 8192,
                lr: float = 2e-3, seed: int = 0, val_fraction: float = 0.1, device: int = 0):
    """rmb_sched_train: returns (trained parameters, per-epoch training MSE, held-out RMSE)."""
    f = np.ascontiguousarray(features, dtype=np.float32)
    t = np.ascontiguousarray(targets, dtype=np.float32)
    p = np.ascontiguousarray(params, dtype=np.float32).copy()
    stats = np.zeros(epochs + 1, dtype=np.float32)
    err = C.create_string_buffer(512)
    _check(lib().rmb_sched_train(device, _fptr(f), _fptr(t), len(t), epochs, batch, lr, seed, val_fraction, _fptr(p),
                                 _fptr(stats), err, 512), err)
    return p, stats[:epochs].copy(), float(stats[epochs])


def sched_grad(params: np.ndarray, features: np.ndarray, targets: np.ndarray, device: int = 0):
    """rmb_sched_grad: (MSE, gradient in the parameter layout) on the given rows."""
    f = np.ascontiguousarray(features, dtype=np.float32)
    t = np.ascontiguousarray(targets, dtype=np.float32)
    p = np.ascontiguousarray(params, dtype=np.float32)
    g = np.zeros(SCHED_NET, dtype=np.float32)
    loss = C.c_float()
    err = C.create_string_buffer(512)
    _check(lib().rmb_sched_grad(device, _fptr(p), _fptr(f), _fptr(t), len(t), _fptr(g), C.byref(loss), err, 512), err)
    return float(loss.value), g


def sched_predict(params: np.ndarray, features: np.ndarray, device: int = 0) -> np.ndarray:
    """rmb_sched_predict: the inference kernel's predicted log1p cells for raw features."""
    f = np.ascontiguousarray(features, dtype=np.float32)
    p = np.ascontiguousarray(params, dtype=np.float32)
    y = np.zeros(len(f), dtype=np.float32)
    err = C.create_string_buffer(512)
    _check(lib().rmb_sched_predict(device, _fptr(p), _fptr(f), len(f), _fptr(y), err, 512), err)
    return y


def ka_resolve(matrix_name: str, gap_open: int, gap_extend: int, matrix_text: str | None = None,
               cli: tuple[float, float, float, float] | None = None) -> tuple[tuple[float, ...], int]:
    """rmb_ka_resolve: (lambda, K, H, alpha, beta) and the source (0 none, 1 table, 2 command
    line, 3 matrix comment) of the E-value statistics, as the reference's ka_stats::resolve."""
    ka = (C.c_double * 5)()
    src = C.c_int32()
    err = C.create_string_buffer(512)
    c = (C.c_double * 4)(*cli) if cli else None
    _check(lib().rmb_ka_resolve(matrix_name.encode(), matrix_text.encode() if matrix_text is not None else None,
                                gap_open, gap_extend, c, ka, C.byref(src), err, 512), err)
    return tuple(ka), src.value


class Searcher:
    """One search context on one GPU: parameters, matrix and the resident library."""

    def __init__(self, params: SearchParams, matrix: ScoreMatrix, db: SubjectDb):
        self.params, self.matrix, self.db = params, matrix, db
        ctx = C.c_void_p()
        err = C.create_string_buffer(512)
        sc = matrix.scores.astype(np.int32).ravel()
        fr = matrix.freqs.astype(np.float64)
        cli = (params.matrix_lambda, params.matrix_k, params.matrix_alpha, params.matrix_beta)
        self.ka, self.ka_source = ka_resolve(matrix.name, params.gap_open, params.gap_extend, matrix.text, cli)
        _check(lib().rmb_ctx_create(C.byref(params._c(self.ka)), sc.ctypes.data_as(C.POINTER(C.c_int32)),
                                    fr.ctypes.data_as(C.POINTER(C.c_double)), matrix.lambda_,
                                    matrix.name.encode(), C.byref(ctx), err, 512), err)
        self._ctx = ctx
        self._lib = lib()
        n = len(db.ids)
        lens = (C.c_uint32 * n)(*[len(p) - 2 for p in db.plus])
        ids = (C.c_char_p * n)(*[i.encode() for i in db.ids])
        _check(lib().rmb_db_load(ctx, n, _ptr_array(db.plus), lens, _ptr_array(db.masks), ids, err, 512), err)

    def _queries(self, queries: list[np.ndarray]):
        n = len(queries)
        return n, _ptr_array(queries), (C.c_uint32 * max(n, 1))(*[len(q) - 2 for q in queries])

    def search(self, queries: list[np.ndarray], query_ids: list[str] | None = None) -> Results:
        n, qp, ql = self._queries(queries)
        res = C.POINTER(_Results)()
        err = C.create_string_buffer(1024)
        _check(lib().rmb_search_batch(self._ctx, n, qp, ql, C.byref(res), err, 1024), err)
        return Results(self, res, query_ids or [f"query{i}" for i in range(n)])

    def set_schedule_model(self, params: np.ndarray) -> None:
        """rmb_sched_set_model: the cost network for searches with schedule=1."""
        p = np.ascontiguousarray(params, dtype=np.float32)
        err = C.create_string_buffer(512)
        _check(lib().rmb_sched_set_model(self._ctx, _fptr(p), p.size, err, 512), err)

    def schedule_log(self, queries: list[np.ndarray]) -> tuple[np.ndarray, np.ndarray]:
        """rmb_sched_log: (raw features n x 12, DP cells n) of the records of one FIFO search."""
        n, qp, ql = self._queries(queries)
        f = C.POINTER(C.c_float)()
        c = C.POINTER(C.c_uint32)()
        m = C.c_uint64()
        err = C.create_string_buffer(1024)
        _check(lib().rmb_sched_log(self._ctx, n, qp, ql, C.byref(f), C.byref(c), C.byref(m), err, 1024), err)
        try:
            k = m.value
            feats = np.ctypeslib.as_array(f, shape=(max(k, 1) * SCHED_NF,))[:k * SCHED_NF].reshape(k, SCHED_NF).copy()
            cells = np.ctypeslib.as_array(c, shape=(max(k, 1),))[:k].copy()
        finally:
            lib().rmb_text_free(C.cast(f, C.c_void_p))
            lib().rmb_text_free(C.cast(c, C.c_void_p))
        return feats, cells

    def tune(self) -> dict:
        """rmb_tune_get: the context's launch knobs."""
        t = _Tune()
        _check(lib().rmb_tune_get(self._ctx, C.byref(t)), C.create_string_buffer(1))
        return {f: getattr(t, f) for f, _ in _Tune._fields_}

    def set_tune(self, knobs: dict) -> None:
        """rmb_tune_set: launch knobs (unlisted ones keep their current values)."""
        cur = self.tune()
        cur.update(knobs)
        t = _Tune(*[int(cur[f]) for f, _ in _Tune._fields_])
        err = C.create_string_buffer(512)
        _check(lib().rmb_tune_set(self._ctx, C.byref(t), err, 512), err)

    def autotune(self, queries: list[np.ndarray], cache: str | Path | None = None, key: str | None = None) -> dict:
        """rmb_autotune on sample queries: the fastest launch knobs stay on the context.  With a
        cache file, a set stored under `key` (default: the GPU's name and SM count with the
        search parameters) is applied without timing anything, and a new result is stored."""
        import json
        key = key or self.tune_key()
        store = {}
        if cache and Path(cache).exists():
            store = json.loads(Path(cache).read_text())
            if key in store:
                self.set_tune(store[key]["tune"])
                return dict(store[key], cached=True)
        n, qp, ql = self._queries(queries)
        t = _Tune()
        best, dflt = C.c_double(), C.c_double()
        err = C.create_string_buffer(1024)
        _check(lib().rmb_autotune(self._ctx, n, qp, ql, C.byref(t), C.byref(best), C.byref(dflt), err, 1024), err)
        res = {"tune": {f: getattr(t, f) for f, _ in _Tune._fields_}, "best_ms": best.value,
               "default_ms": dflt.value, "sample_queries": n, "sample_bp": int(sum(len(q) - 2 for q in queries))}
        if cache:
            store[key] = res
            Path(cache).write_text(json.dumps(store, indent=1, sort_keys=True) + "\n")
        return dict(res, cached=False)

    def tune_key(self) -> str:
        """GPU model and SM count plus the parameters that shape the work (word size, gaps, X-drops)."""
        name, sms = device_name(self.params.device)
        p = self.params
        return (f"{name}/{sms}sm/w{p.word_size}/g{p.gap_open}.{p.gap_extend}/x{p.xdrop_ungap}.{p.xdrop_gap}."
                f"{p.xdrop_gap_final}/s{p.schedule}")

    def upload(self, queries: list[np.ndarray]) -> "ResidentQueries":
        """rmb_queries_upload: the queries copied into device memory once."""
        n, qp, ql = self._queries(queries)
        h = C.c_void_p()
        err = C.create_string_buffer(1024)
        _check(lib().rmb_queries_upload(self._ctx, n, qp, ql, C.byref(h), err, 1024), err)
        return ResidentQueries(h, n)

    def search_resident(self, rq: "ResidentQueries", query_ids: list[str] | None = None) -> Results:
        res = C.POINTER(_Results)()
        err = C.create_string_buffer(1024)
        _check(lib().rmb_search_resident(self._ctx, rq._h, C.byref(res), err, 1024), err)
        return Results(self, res, query_ids or [f"query{i}" for i in range(rq.n)])

    def stage(self, queries: list[np.ndarray], stage: int) -> np.ndarray:
        n, qp, ql = self._queries(queries)
        rec = C.POINTER(C.c_uint32)()
        nrec = C.c_uint64()
        err = C.create_string_buffer(1024)
        _check(lib().rmb_debug_stage(self._ctx, n, qp, ql, stage, C.byref(rec), C.byref(nrec), err, 1024), err)
        width = (3, 6, 8, 3, 9)[stage]
        try:
            a = np.ctypeslib.as_array(rec, shape=(int(nrec.value) * width,)).copy() if nrec.value else np.zeros(0, np.uint32)
        finally:
            lib().rmb_text_free(C.cast(rec, C.c_void_p))
        return a.reshape(-1, width)

    def close(self):
        if getattr(self, "_ctx", None):
            self._lib.rmb_ctx_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        self.close()
