"""Seeded synthetic genome-vs-TE-library workloads (no public dataset exists for this path).

Model: i.i.d. genome at 41% GC (A=T=0.295, C=G=0.205) with planted copies of library
consensi.  Each copy is a random sub-span (>= 50 bp) of a consensus on a random strand,
Kimura-2P mutated at a drawn divergence (transition:transversion 2:1) with indels of
geometric length (mean 2) at a drawn rate.  N runs of 20-500 bp cover 1% of the genome.

Workloads (sizes in bases):
  small      one 100 kb query, 50 consensi of 300-6,000 bp, 300 planted copies at 5-30%
             divergence, 1-5% indels; word 7.
  plain      1,000 query chunks of 60 kb (45% planted repeats at 2-35% divergence) against
             2,000 consensi with log-normal lengths (median 1.5 kb, 100-12,000, about 5 Mb);
             word 11.
  batched    20,000 query chunks of 1-200 kb (log-normal) against the plain library.
  allvsall   5,000 consensi of 200-10,000 bp (20% derived from others at 10-40% divergence)
             searched against themselves; word 7, masklevel off.

Every generator takes a seed and is deterministic; `scale` shrinks the query side for tests.
The query chunks of plain and batched each come from their own random stream (seed, chunk
index), so any batch of chunks can be made on its own and in parallel.
"""
from __future__ import annotations

import numpy as np

BASES = np.frombuffer(b"ACGT", dtype=np.uint8)
COMP = np.zeros(256, dtype=np.uint8)
for a, b in zip(b"ACGTN", b"TGCAN"):
    COMP[a] = b
FREQ = np.array([0.295, 0.205, 0.205, 0.295])
# transitions: A<->G, C<->T ; transversions: the other two
TRANSITION = {ord("A"): ord("G"), ord("G"): ord("A"), ord("C"): ord("T"), ord("T"): ord("C")}
TRANSVERSIONS = {
    ord("A"): (ord("C"), ord("T")), ord("G"): (ord("C"), ord("T")),
    ord("C"): (ord("A"), ord("G")), ord("T"): (ord("A"), ord("G")),
}
_TI = np.zeros(256, dtype=np.uint8)
_TV = np.zeros((256, 2), dtype=np.uint8)
for k, v in TRANSITION.items():
    _TI[k] = v
for k, v in TRANSVERSIONS.items():
    _TV[k] = v

MATRIX_TEXT = """# FREQS A 0.295 C 0.205 G 0.205 T 0.295
    A    C    G    T    N
A   9  -15   -8  -15   -1
C -15   10  -15   -8   -1
G  -8  -15   10  -15   -1
T -15   -8  -15    9   -1
N  -1   -1   -1   -1   -1
"""
MATRIX_NAME = "synthetic41gc.matrix"


def random_dna(rng: np.random.Generator, n: int) -> np.ndarray:
    return BASES[rng.choice(4, size=n, p=FREQ)]


def revcomp(s: np.ndarray) -> np.ndarray:
    return COMP[s[::-1]]


def mutate(rng: np.random.Generator, s: np.ndarray, div: float, indel: float) -> np.ndarray:
    """Kimura-2P substitutions at rate `div` (ts:tv 2:1) and geometric indels at rate `indel`."""
    s = s.copy()
    sub = rng.random(len(s)) < div
    ts = rng.random(len(s)) < 2.0 / 3.0
    pick = rng.integers(0, 2, len(s))
    idx = np.nonzero(sub & ts)[0]
    s[idx] = _TI[s[idx]]
    idx = np.nonzero(sub & ~ts)[0]
    s[idx] = _TV[s[idx], pick[idx]]
    if indel <= 0:
        return s
    ev = np.nonzero(rng.random(len(s)) < indel)[0]
    if len(ev) == 0:
        return s
    # every event's length and kind, and the bases of all insertions, drawn at once
    lens = rng.geometric(0.5, len(ev))
    is_ins = rng.random(len(ev)) < 0.5
    ins_bases = random_dna(rng, int(lens[is_ins].sum()))
    out = []
    prev = 0
    used = 0
    for p, ln, ins in zip(ev.tolist(), lens.tolist(), is_ins.tolist()):
        if p < prev:
            continue  # inside an earlier deletion
        out.append(s[prev:p])
        if ins:
            out.append(ins_bases[used:used + ln])
            used += ln
            prev = p
        else:
            prev = p + ln
    out.append(s[prev:])
    return np.concatenate(out)


def library(rng: np.random.Generator, n: int, lengths: np.ndarray) -> list[np.ndarray]:
    return [random_dna(rng, int(L)) for L in lengths]


def plant(rng: np.random.Generator, genome: np.ndarray, lib: list[np.ndarray], target_frac: float | None,
          n_copies: int | None, div_range: tuple[float, float], indel_range: tuple[float, float]) -> np.ndarray:
    """Overwrite genome spans with mutated library fragments, keeping the genome length."""
    g = genome
    L = len(g)
    planted = 0
    copies = 0
    goal = target_frac * L if target_frac is not None else None
    while (goal is not None and planted < goal) or (n_copies is not None and copies < n_copies):
        c = lib[int(rng.integers(len(lib)))]
        if len(c) < 50:
            continue
        flen = int(rng.integers(50, len(c) + 1))
        st = int(rng.integers(0, len(c) - flen + 1))
        frag = c[st:st + flen]
        if rng.random() < 0.5:
            frag = revcomp(frag)
        frag = mutate(rng, frag, float(rng.uniform(*div_range)), float(rng.uniform(*indel_range)))
        if len(frag) >= L:
            continue
        pos = int(rng.integers(0, L - len(frag)))
        g[pos:pos + len(frag)] = frag
        planted += len(frag)
        copies += 1
    return g


def add_n_runs(rng: np.random.Generator, g: np.ndarray, frac: float = 0.01) -> np.ndarray:
    covered = 0
    while covered < frac * len(g):
        ln = int(rng.integers(20, 501))
        if ln >= len(g):
            break
        pos = int(rng.integers(0, len(g) - ln))
        g[pos:pos + ln] = ord("N")
        covered += ln
    return g


def lognormal_lengths(rng: np.random.Generator, n: int, median: float, total: float, lo: int, hi: int) -> np.ndarray:
    mean = total / n
    sigma = float(np.sqrt(2.0 * np.log(max(mean / median, 1.0000001))))
    x = rng.lognormal(np.log(median), sigma, n)
    return np.clip(np.round(x), lo, hi).astype(np.int64)


def to_fasta(names: list[str], seqs: list[np.ndarray]) -> str:
    parts = []
    for n, s in zip(names, seqs):
        b = s.tobytes().decode()
        parts.append(">" + n + "\n" + "\n".join(b[i:i + 80] for i in range(0, len(b), 80)) + "\n")
    return "".join(parts)


def _chunk(args) -> tuple[str, np.ndarray]:
    """Query chunk i of a genome-vs-library workload, from its own random stream."""
    name, seed, i, lib = args
    rng = np.random.default_rng([seed, i])
    if name == "plain":
        qlen = 60_000
    else:
        qlen = int(np.clip(np.round(rng.lognormal(np.log(20_000), 1.0)), 1_000, 200_000))
    g = random_dna(rng, qlen)
    g = plant(rng, g, lib, 0.45, None, (0.02, 0.35), (0.01, 0.05))
    g = add_n_runs(rng, g)
    return f"chunk{i}", g


_POOL_LIB = None


def _init_pool(lib):
    global _POOL_LIB
    _POOL_LIB = lib


def _chunk_pooled(args):
    name, seed, i = args
    return _chunk((name, seed, i, _POOL_LIB))


def genome_library(seed: int | None = None) -> list[np.ndarray]:
    """The 2,000-consensus library of the plain and batched workloads (log-normal lengths,
    median 1.5 kb, 100-12,000 bp, about 5 Mb)."""
    lrng = np.random.default_rng(0x524D42 + 1 if seed is None else seed)
    lens = lognormal_lengths(lrng, 2000, 1500.0, 5_000_000.0, 100, 12_000)
    return library(lrng, 2000, lens)


def chunk_count(name: str, scale: float = 1.0) -> int:
    return max(1, int(round({"plain": 1000, "batched": 20_000}[name] * scale)))


def query_chunks(name: str, lib: list[np.ndarray], start: int, stop: int, seed: int | None = None,
                 workers: int = 0) -> list[tuple[str, np.ndarray]]:
    """Chunks start..stop-1 of a plain or batched workload's query set.  Every chunk has its
    own random stream (seed, chunk index), so a batch of chunks is the same whichever other
    chunks are made, and `workers` > 1 makes them in that many processes."""
    base = 0x524D42 + {"plain": 1, "batched": 2}[name] if seed is None else seed
    idx = range(start, stop)
    if workers > 1 and stop - start > 8:
        import multiprocessing as mp
        # spawn: the callers may already hold a CUDA context, which a forked child must not touch
        with mp.get_context("spawn").Pool(workers, initializer=_init_pool, initargs=(lib,)) as pool:
            return pool.map(_chunk_pooled, [(name, base, i) for i in idx], chunksize=4)
    return [_chunk((name, base, i, lib)) for i in idx]


def workload(name: str, seed: int | None = None, scale: float = 1.0, workers: int = 0):
    """Returns (queries, library, params) with sequences as uint8 ASCII arrays.

    `scale` < 1 keeps the library and the per-query shapes but generates fewer queries
    (or a shorter query for `small`), for tests and bounded CPU samples.
    """
    base = {"small": 0, "plain": 1, "batched": 2, "allvsall": 4}[name]
    rng = np.random.default_rng(0x524D42 + base if seed is None else seed)
    common = dict(gap_open=20, gap_extend=5, complexity_adjust=1, dust=0)
    if name == "small":
        lib = library(rng, 50, rng.integers(300, 6001, 50))
        qlen = max(1000, int(100_000 * scale))
        g = random_dna(rng, qlen)
        g = plant(rng, g, lib, None, max(1, int(300 * scale)), (0.05, 0.30), (0.01, 0.05))
        g = add_n_runs(rng, g)
        params = dict(common, word_size=7, mask_level=80)
        return [("genome", g)], [(f"cons{i}", s) for i, s in enumerate(lib)], params
    if name in ("plain", "batched"):
        lib = genome_library(seed)
        qs = query_chunks(name, lib, 0, chunk_count(name, scale), seed, workers)
        params = dict(common, word_size=11, mask_level=80)
        return qs, [(f"cons{i}", s) for i, s in enumerate(lib)], params
    if name == "allvsall":
        n = max(2, int(round(5000 * scale)))
        lens = rng.integers(200, 10_001, n)
        lib = []
        for i in range(n):
            if i > 10 and rng.random() < 0.2:
                src = lib[int(rng.integers(len(lib)))]
                d = rng.uniform(0.35, 0.40) if rng.random() < 0.25 else rng.uniform(0.10, 0.40)
                s = mutate(rng, src, float(d), 0.02)
                # segmental rearrangement: swap two halves
                cut = int(rng.integers(1, max(2, len(s) - 1)))
                s = np.concatenate([s[cut:], s[:cut]])
                lib.append(s)
            else:
                lib.append(random_dna(rng, int(lens[i])))
        recs = [(f"cons{i}", s) for i, s in enumerate(lib)]
        params = dict(common, word_size=7, mask_level=-1)
        return recs, recs, params
    raise ValueError(name)


# RepeatMasker's search settings (NCBIBlastSearchEngine): the cutoffs and X-drops it passes
# to rmblastn with every search; every workload runs with them.
RM_FLAGS = dict(min_raw_gapped_score=200, xdrop_ungap=400, xdrop_gap=100, xdrop_gap_final=200)
# rmblastn's own defaults for the flags the workloads leave unset.
DEFAULT_FLAGS = dict(min_raw_gapped_score=0, xdrop_ungap=20, xdrop_gap=30, xdrop_gap_final=100)
