#!/usr/bin/env python
"""Benchmark of the B200 rmblastn search core on the genome-vs-TE-library workloads.

Default workload ("batched", the learned-schedule configuration): 20,000 query chunks of 1-200 kb
(log-normal, median 20 kb; 45% planted repeats at 2-35% divergence, 1% N runs; about 630 Mb)
against 2,000 synthetic consensi (about 5 Mb), word 11, gap costs 20/5, complexity adjustment,
masklevel 80, dust off, RepeatMasker's cutoffs and X-drops (min_raw_gapped_score 200,
xdrop_ungap 400, xdrop_gap 100, xdrop_gap_final 200).  The chunks go to the GPU in batches of
1,000; a step is one batch through the full path (lookup tables, scan, extensions, dedup,
prelim DP, interval-tree filters, traceback DP, complexity adjustment, purges, masklevel, hit
order), and the steps cycle through the batches, so 20 timed steps are the whole query set.

The measured arm is the batched pipeline (persistent kernels with device work queues) with the
learned record order.  On the same steps the bench also times
  plain          the plain GPU pipeline (one launch per stage, one work item per thread, FIFO):
                 `vs_plain` is the measured arm over it
  batched_fifo   the batched pipeline with the FIFO record order: the learned order's own gain
  value  query Mbp/s with queries and library resident in HBM (rmb_search_resident)
  e2e    the measured arm through rmb_search_batch from host buffers plus the outfmt-6 text of
         every HSP (host->device query copy and device->host results inside the timed region)

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload batched|plain|small|allvsall] [--schedule learned|fifo]
                    [--pipeline batched|plain]
Multi-GPU (weak scaling): each rank searches its own query chunks (the workload's chunk stream
continued past the other ranks') against the full library; no collective is on the data path.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

FIELDS = "6 score perc_sub qseqid qstart qend sseqid sstart send"
OPS_PER_CELL = 11  # int32 add/sub/max/compare per DP cell in search/gapped.rs:234-262
# DRAM bytes (read + write) per ungapped record of k_prelim_stream, from one ncu capture of
# `bench.py --workload plain --scale 0.01` (1.31 M records, 80.1 MB); the traffic is per record
# (the 48-byte geometry read, the 28-byte result write, sequence words), so a launch's traffic
# is this times its records
PRELIM_STREAM_DRAM_BYTES_PER_RECORD = 61.0
# copy bandwidth of this pool's B200s measured earlier, used when MEASURED_PEAKS.json is absent
HBM_FALLBACK_GBS = 6650.0
BATCH_CHUNKS = 1000


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="batched", choices=["batched", "plain", "small", "allvsall"])
    ap.add_argument("--scale", type=float, default=1.0, help="fraction of the query set (tests/profiling)")
    ap.add_argument("--batch-chunks", type=int, default=BATCH_CHUNKS, help="query chunks per step (batched)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU baseline sample budget")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-compare", action="store_true", help="skip the plain and FIFO comparison arms")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch knobs")
    ap.add_argument("--lanes", type=int, choices=[1, 2], default=None,
                    help="pipeline lanes of the measured arm (default: the library's, 2)")
    ap.add_argument("--dust", action="store_true", help="mask the queries with DUST (the reference's default)")
    ap.add_argument("--schedule", choices=["fifo", "learned", "learned-full"], default=None,
                    help="prelim DP record order: FIFO; learned (the predicted-costliest records first); "
                         "learned-full (all in descending predicted cost).  Default: learned for the batched "
                         "workload, else FIFO")
    ap.add_argument("--pipeline", choices=["batched", "plain"], default="batched")
    ap.add_argument("--sched-model", default=None, help="schedule network JSON (default: the committed one)")
    a = ap.parse_args(argv)
    if a.schedule is None:
        a.schedule = "learned" if a.workload == "batched" and a.pipeline == "batched" else "fifo"
    if a.schedule != "fifo" and a.pipeline == "plain":
        ap.error("the learned order feeds the batched pipeline's queue")
    return a


TUNE_SAMPLE_CHUNKS = 200


def workload(args, rank: int):
    """(batches of (id, ASCII chunk), library, params, total chunks, tuning sample) of this rank.
    Batched and plain chunk streams are per-chunk seeded, so rank r takes the stream's chunks
    after ranks 0 .. r-1 and shares the library; only the batches the run reaches are made.  The
    autotuner's sample is the stream's next chunks after every rank's (never a timed chunk)."""
    from rmblast_b200 import synth
    if args.workload in ("plain", "batched"):
        lib = synth.genome_library()
        n = synth.chunk_count(args.workload, args.scale)
        step = min(args.batch_chunks, n) if args.workload == "batched" else n
        nb = (n + step - 1) // step
        need = min(nb, args.warmup + args.steps)
        base = rank * n
        workers = os.cpu_count() or 1
        qs = synth.query_chunks(args.workload, lib, base, base + min(n, need * step), workers=workers)
        batches = [qs[i:i + step] for i in range(0, len(qs), step)]
        db = [(f"cons{i}", s) for i, s in enumerate(lib)]
        _, _, prm = synth.workload(args.workload, scale=1e-9)
        total = n
        tail = max(int(os.environ.get("WORLD_SIZE", 1)), 1) * n
        sample = synth.query_chunks(args.workload, lib, tail, tail + min(TUNE_SAMPLE_CHUNKS, max(step // 5, 1)),
                                    workers=workers)
    else:
        qs, db, prm = synth.workload(args.workload, scale=args.scale)
        batches, total = [qs], len(qs)
        sample = qs[:max(1, len(qs) // 20)]
    p = dict(prm, **synth.RM_FLAGS)
    if args.dust:
        p["dust"] = 1
    return batches, db, p, total, sample


def config_of(args, p, total_chunks, batches, db, world) -> dict:
    """The workload's description, the same in both arms' JSON lines."""
    per_step = [sum(len(s) for _, s in b) for b in batches]
    return {"workload": args.workload, "chunks": total_chunks, "chunks_per_step": len(batches[0]),
            "mean_step_bp": round(statistics.mean(per_step)), "library": len(db),
            "library_bp": int(sum(len(s) for _, s in db)), "word_size": p["word_size"],
            "flags": f"gapopen {p['gap_open']} gapextend {p['gap_extend']} "
                     f"{'complexity_adjust ' if p.get('complexity_adjust') else ''}"
                     f"masklevel {p['mask_level']} dust {'yes' if p.get('dust') else 'no'} "
                     f"min_raw_gapped_score {p['min_raw_gapped_score']} xdrop_ungap {p['xdrop_ungap']} "
                     f"xdrop_gap {p['xdrop_gap']} xdrop_gap_final {p['xdrop_gap_final']}",
            "pipeline": args.pipeline, "schedule": args.schedule,
            "l2": "inputs larger than L2 (each step's lookup tables and hit arrays are GBs)",
            "parallelism": f"{world} independent ranks, query chunks sharded by rank"}


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while the timed region runs."""

    def __init__(self, index: int):
        self.index, self.rows, self.proc = index, [], None

    def __enter__(self):
        cmd = ["nvidia-smi", "-i", str(self.index), "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
               "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
               "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
               "--format=csv,noheader,nounits", "-lms", "200"]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 7:
                self.rows.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def cpu_model() -> str:
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline(qs, db, p, budget_s: float, start: int = 0):
    """The C++ restatement of the reference CPU path (oracle) on all host cores, over the queries
    of the same workload from `start` on until the time budget is spent (at least two queries).
    Returns the baseline figure, the oracle's outfmt-6 text of the sampled queries (the parity
    witness), its stage counters (reference-counted DP cells) and the sampled query ids."""
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_ref as O
    from rmblast_b200 import synth
    threads = os.cpu_count() or 1
    dbf = synth.to_fasta([n for n, _ in db], [s for _, s in db])
    bases, secs, n = 0, 0.0, 0
    texts, ctr = [], {}
    for name, s in qs[start:]:
        qf = synth.to_fasta([name], [s])
        txt, c, t = O.search_text(qf, dbf, synth.MATRIX_TEXT, synth.MATRIX_NAME, p, FIELDS, threads=threads)
        texts.append(txt)
        for k, v in c.items():
            ctr[k] = ctr.get(k, 0) + v
        bases += len(s)
        secs += t
        n += 1
        if secs >= budget_s and n >= 2:
            break
    cb = {"value": bases / secs / 1e6, "unit": "Mbp/s", "cores": threads, "kind": "port", "cpu_model": cpu_model(),
          "sample": f"queries {qs[start][0]}..{qs[start + n - 1][0]} ({bases} bp) vs the full library, "
                    f"{secs:.1f} s, C++ restatement of the reference CPU path (mt-mode 0 split by subject, "
                    f"{threads} threads)"}
    return cb, "".join(texts), ctr, [name for name, _ in qs[start:start + n]]


def parity_witness(gpu_text: str, oracle_text: str, sample_ids: list[str]) -> dict:
    """The GPU run's outfmt-6 lines of the sampled queries (qseqid is the third field) against
    the oracle's text for the same queries, byte for byte."""
    keep = set(sample_ids)
    got = "".join(ln for ln in gpu_text.splitlines(True) if ln.split("\t", 3)[2] in keep)
    return {"queries": len(sample_ids), "lines": oracle_text.count("\n"), "identical": got == oracle_text,
            "against": "oracle (C++ restatement of the reference CPU path), same queries and flags",
            "fields": FIELDS}


def reference_arm(args, rank, world):
    """The reference CPU path on the host cores (the oracle: the reference is Rust and cannot be
    built here), each step a bounded sample of the same workload's queries, consecutive steps
    taking consecutive queries."""
    if rank != 0:
        return
    batches, db, p, total, _ = workload(args, 0)
    qs = [q for b in batches for q in b]
    per_step = max(2.0, 60.0 / max(1, args.steps + args.warmup))
    vals, start, first = [], 0, None
    cb_i = None
    for i in range(args.warmup + args.steps):
        cb_i, _, _, sample = cpu_baseline(qs, db, p, per_step, start)
        start = (start + len(sample)) % len(qs)
        if i >= args.warmup:
            vals.append(cb_i["value"])
            first = first or sample[0]
    v = statistics.mean(vals)
    threads = os.cpu_count() or 1
    cb = dict(cb_i, value=v,
              sample=f"{args.steps} steps of ~{per_step:.1f} s, each the next queries of the workload from "
                     f"{first} on, against the full library; C++ restatement of the reference CPU path "
                     f"(mt-mode 0 split by subject, {threads} threads)",
              spread={"min": min(vals), "max": max(vals), "stdev": statistics.stdev(vals) if len(vals) > 1 else 0.0})
    line = {"metric": "query Mbp/s", "value": v, "unit": "Mbp/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded genome/TE-library model)",
            "impl": "reference", "config": config_of(args, p, total, batches, db, world), "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "Mbp/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def scan_roofline(n_queries: float, db, c: dict, peaks: dict) -> dict:
    """The seed scan against HBM: algorithmic bytes = every query reads the whole packed library
    (a byte per 4 bases) and every word hit writes 8 bytes; the library (~1.2 MB packed) stays
    in L2, so DRAM carries far less and the stage is bound by its random probes into the query
    tables, not by bandwidth."""
    packed = sum((len(s) + 3) // 4 for _, s in db)
    algo = n_queries * packed + 8 * c["word_hits"]
    ms = c["gpu_ms_scan"]
    gbs = algo / (ms * 1e-3) / 1e9 if ms > 0 else None
    peak = peaks.get("hbm_gbs")
    return {"kernel": "k_scan (one staged pass) + k_scan_gather", "bound": "L2 probes", "algorithmic_bytes": algo,
            "ms": ms, "achieved_gbs": gbs, "hbm_peak_gbs": peak, "frac_of_hbm": gbs / peak if gbs and peak else None}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    # the query chunks are made (in spawned processes) before this process touches CUDA
    batches, db, p, total, tune_sample = workload(args, rank)
    import torch
    from rmblast_b200 import api, build, synth
    build.build()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    m = api.ScoreMatrix.from_text(synth.MATRIX_TEXT, synth.MATRIX_NAME)
    sdb = api.SubjectDb.from_records(db)
    compare = not args.no_compare and args.workload in ("batched", "plain") and args.pipeline == "batched"
    model = None
    if args.schedule != "fifo":
        from rmblast_b200 import train_sched
        model = train_sched.load_model(Path(args.sched_model) if args.sched_model else train_sched.MODEL_PATH)

    def searcher(pipeline: str, schedule: str):
        sp = api.SearchParams(gap_open=p["gap_open"], gap_extend=p["gap_extend"], word_size=p["word_size"],
                              xdrop_ungap=p["xdrop_ungap"], xdrop_gap=p["xdrop_gap"],
                              xdrop_gap_final=p["xdrop_gap_final"], min_raw_gapped_score=p["min_raw_gapped_score"],
                              complexity_adjust=bool(p["complexity_adjust"]), mask_level=p["mask_level"],
                              dust=bool(p.get("dust", 0)), device=local,
                              schedule={"fifo": 0, "learned": 1, "learned-full": 2}[schedule],
                              pipeline=1 if pipeline == "plain" else 0)
        s = api.Searcher(sp, m, sdb)
        if schedule != "fifo":
            s.set_schedule_model(model)
        return s

    enc = [[api.encode(x) for _, x in b] for b in batches]
    ids = [[n for n, _ in b] for b in batches]
    bases = [sum(len(x) for _, x in b) for b in batches]
    nb = len(batches)
    warm = [k % nb for k in range(args.warmup)]
    timed = [(args.warmup + k) % nb for k in range(args.steps)]
    timed_bases = sum(bases[b] for b in timed) / args.steps  # per step

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        if not dist:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def resident_arm(s, clocks=None):
        """K timed steps with every batch resident in HBM: (ms per step, mean counters)."""
        rq = [s.upload(e) for e in enc]
        # the largest step first, so the grow-only device buffers reach their size untimed
        s.search_resident(rq[max(range(nb), key=lambda i: bases[i])])
        for b in warm:
            s.search_resident(rq[b], ids[b])
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ctrs = []
        cm = ClockSampler(local) if clocks is not None else None
        if cm:
            cm.__enter__()
        barrier()
        ev0.record()
        for b in timed:
            ctrs.append(s.search_resident(rq[b], ids[b]).counters)
        ev1.record()
        barrier()
        if cm:
            cm.__exit__()
            clocks.update(cm.summary())
        for r in rq:
            r.free()
        cc = {k: sum(x[k] for x in ctrs) / len(ctrs) for k in ctrs[0]}
        return max_over_ranks(ev0.elapsed_time(ev1) / args.steps), cc

    def kernel_pass(s) -> dict:
        """The timed steps again on one pipeline lane, untimed: each stage's device time alone (two
        lanes' kernels overlap, so their event times include each other)."""
        knobs = s.tune()
        s.set_tune(dict(knobs, lanes=1))
        rq = [s.upload(enc[b]) for b in timed]
        kc = [s.search_resident(r).counters for r in rq]
        for r in rq:
            r.free()
        s.set_tune(knobs)
        return {key: sum(x[key] for x in kc) / len(kc) for key in kc[0]}

    def arm_summary(ms: float, kc: dict) -> dict:
        """An arm's throughput (its timed steps) and its stages' device times (one lane)."""
        return {"value": timed_bases * world / (ms * 1e-3) / 1e6, "ms_per_step": ms, "prelim_ms": kc["gpu_ms_prelim"],
                "gcups_computed": kc["so_cells"] / (kc["gpu_ms_prelim"] * 1e-3) / 1e9 if kc["gpu_ms_prelim"] else None,
                "stage_ms": {key: round(kc[key], 3) for key in ("gpu_ms_scan", "gpu_ms_ungapped", "gpu_ms_dedup",
                                                              "gpu_ms_prelim", "gpu_ms_sched", "gpu_ms_traceback")}}

    # ---- the measured arm: autotuned launch knobs (batched pipeline), resident, then end to end
    s = searcher(args.pipeline, args.schedule)
    tuned = None
    if args.pipeline == "batched" and not args.no_autotune:
        tuned = s.autotune([api.encode(x) for _, x in tune_sample])
    if args.lanes:
        s.set_tune(dict(s.tune(), lanes=args.lanes))
    clk = {}
    ms_step, c = resident_arm(s, clk)
    # the context's query buffers (device and pinned host) grow to the largest step untimed
    big = max(range(nb), key=lambda i: bases[i])
    for b in [big] + warm[:max(1, args.warmup // 2)]:
        s.search(enc[b], ids[b]).tabular(FIELDS)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    h2d = d2h = 0
    barrier()
    e0.record()
    for b in timed:
        txt = s.search(enc[b], ids[b]).tabular(FIELDS)
        h2d += sum(len(e) for e in enc[b])
        d2h += len(txt)
    e1.record()
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
    # the measured arm's text of the first timed step: the parity witness and the arms' check
    b0 = timed[0]
    text_b0 = s.search(enc[b0], ids[b0]).tabular(FIELDS)

    peak_int = api.int32_peak_tops(local)
    # the kernels alone (one lane): the roofline, GCUPS and stage times come from these
    knobs = s.tune() if args.pipeline == "batched" else {"lanes": 1}
    k = kernel_pass(s) if args.pipeline == "batched" else c
    prelim_ms = k["gpu_ms_prelim"]
    so_cells = k["so_cells"]
    # the dominant kernel: k_prelim_stream (one launch per sub-batch), timed alone with CUDA events
    main_ms, main_cells = k["gpu_ms_prelim_main"], k["so_cells_main"]
    if main_ms <= 0:  # parameters outside the thread kernel's range: the warp kernel does it all
        main_ms, main_cells = prelim_ms, so_cells
    achieved = main_cells * OPS_PER_CELL / (main_ms * 1e-3) / 1e12 if main_ms > 0 else 0.0
    traffic = (PRELIM_STREAM_DRAM_BYTES_PER_RECORD * k["prelim_dp"]
               if PRELIM_STREAM_DRAM_BYTES_PER_RECORD and k["gpu_ms_prelim_main"] > 0 else None)
    peaks, peak_source = {"hbm_gbs": HBM_FALLBACK_GBS}, "fallback"
    pk = ROOT / "MEASURED_PEAKS.json"
    if pk.exists():
        peaks, peak_source = json.loads(pk.read_text()), "measured"
    line = {
        "metric": "query Mbp/s", "value": timed_bases * world / (ms_step * 1e-3) / 1e6, "unit": "Mbp/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded genome/TE-library model)",
        "config": config_of(args, p, total, batches, db, world),
        # DP cells the GPU computed (gapped.rs:188 counting) per second of the stage; the reference-
        # counted figures (gcups_reference) follow from the oracle's cells on the CPU sample
        "gcups_computed": so_cells / (prelim_ms * 1e-3) / 1e9 if prelim_ms > 0 else None,
        "traceback_gcups_computed": (k["tb_cells"] / (k["gpu_ms_traceback"] * 1e-3) / 1e9
                                     if k["gpu_ms_traceback"] > 0 else None),
        "scan_roofline": scan_roofline(sum(len(enc[b]) for b in timed) / args.steps, db, k, peaks),
        # device time per stage on one lane (the kernels alone), and the lanes' sum in the timed run
        # (gpu_ms_sched: the learned order's features, network and order, a part of gpu_ms_prelim)
        "stage_ms": {key: round(k[key], 3) for key in ("gpu_ms_lookup", "gpu_ms_scan", "gpu_ms_ungapped",
                                                      "gpu_ms_dedup", "gpu_ms_prelim", "gpu_ms_sched",
                                                      "gpu_ms_traceback", "ms_host_2a", "ms_host_2b")},
        "lanes": knobs.get("lanes", 1),
        # wall-clock per stage on the host (device work, syncs and host steps together)
        "wall_ms": {k: round(c[k], 3) for k in ("ms_lookup", "ms_scan", "ms_ungapped", "ms_dedup", "ms_prelim_dp",
                                                 "ms_host_2a", "ms_traceback", "ms_host_2b")},
        "counts": {k: int(c[k]) for k in ("word_hits", "ungapped", "prelim_dp", "prelims", "tb_dp", "finals",
                                          "so_cells", "tb_cells")},
        "roofline": {"kernel": "k_prelim_stream (score-only X-drop DP)", "bound": "int32", "achieved": achieved,
                     "peak": peak_int, "unit": "Tops/s", "frac": achieved / peak_int if peak_int else None,
                     "traffic": traffic, "kernel_ms": main_ms, "cells": main_cells,
                     "hbm": {"achieved_gbs": traffic / (main_ms * 1e-3) / 1e9 if traffic else None,
                             "peak_gbs": peaks.get("hbm_gbs"), "peak_source": peak_source,
                             "frac": (traffic / (main_ms * 1e-3) / 1e9 / peaks["hbm_gbs"]
                                      if traffic and peaks.get("hbm_gbs") else None)},
                     "note": f"{OPS_PER_CELL} int32 ops per DP cell (the reference's cell step) x cells of the "
                             "records k_prelim_stream completed / its event time; peak = rmb_probe_int32_peak "
                             "(dependent int32 add/max throughput of this GPU) measured in this run; the kernel "
                             "is bound by integer issue, not by HBM (hbm.frac) or tensor cores"},
        "gpu_launches": int(c["launches"] * args.steps),
        "clocks": clk,
        "e2e": {"value": timed_bases * world / (e2e_ms * 1e-3) / 1e6, "unit": "Mbp/s",
                "h2d_bytes_per_step": h2d // args.steps, "d2h_bytes_per_step": d2h // args.steps,
                "ms_per_step": e2e_ms},
    }
    if tuned is not None:
        line["autotune"] = {"knobs": tuned["tune"], "tuned_ms": tuned["best_ms"], "default_ms": tuned["default_ms"],
                            "sample": f"{tuned['sample_queries']} chunks ({tuned['sample_bp']} bp) of the workload's "
                                      "stream past the timed ones; device ms of the ungapped, dedup and prelim stages"}
    if model is not None and not args.sched_model:
        from rmblast_b200 import train_sched
        info = json.loads(train_sched.MODEL_PATH.read_text()).get("info", {})
        line["schedule_model"] = {"test_rmse_log_cells": info.get("test_rmse_log_cells"),
                                  "test_mean_predictor_rmse": info.get("test_mean_predictor_rmse"),
                                  "test_spearman": info.get("test_ranking", {}).get("spearman")}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb, otext, octr, sample_ids = cpu_baseline(batches[b0], db, p, args.cpu_seconds)
        line["cpu_baseline"] = cb
        line["parity"] = parity_witness(text_b0, otext, sample_ids)
        # the GPU's DP cells on the same sample: it runs the prelim DP of every ungapped record and
        # the traceback of every post-purge prelim, while the reference skips the records already
        # contained in an earlier HSP (search/engine.rs:1333-1345, 1491-1509)
        n = len(sample_ids)
        rs = s.search(enc[b0][:n], ids[b0][:n])
        spec_so = rs.counters["so_cells"] / octr["so_cells"] if octr.get("so_cells") else None
        spec_tb = rs.counters["tb_cells"] / octr["tb_cells"] if octr.get("tb_cells") else None
        line["speculative_cell_ratio"] = {"prelim": spec_so, "traceback": spec_tb,
                                          "sample": f"the {n} queries of cpu_baseline"}
        if spec_so and line["gcups_computed"]:
            line["gcups_reference"] = line["gcups_computed"] / spec_so
        if spec_tb and line["traceback_gcups_computed"]:
            line["traceback_gcups_reference"] = line["traceback_gcups_computed"] / spec_tb
    s.close()
    # ---- the comparison arms on the same steps
    if compare:
        me = arm_summary(ms_step, k)
        arms = {"measured": me}
        s = searcher("plain", "fifo")
        ms, cc = resident_arm(s)
        arms["plain"] = arm_summary(ms, cc)  # the plain pipeline runs one lane
        arms["plain"]["identical_output_first_step"] = s.search(enc[b0], ids[b0]).tabular(FIELDS) == text_b0
        s.close()
        line["vs_plain"] = {"value": me["value"] / arms["plain"]["value"],
                            "gcups_computed": (me["gcups_computed"] / arms["plain"]["gcups_computed"]
                                               if arms["plain"]["gcups_computed"] else None),
                            "prelim_stage": arms["plain"]["prelim_ms"] / me["prelim_ms"] if me["prelim_ms"] else None}
        if args.schedule != "fifo":
            s = searcher("batched", "fifo")
            if tuned is not None:
                s.set_tune(tuned["tune"])
            ms, cc = resident_arm(s)
            arms["batched_fifo"] = arm_summary(ms, kernel_pass(s))
            arms["batched_fifo"]["identical_output_first_step"] = s.search(enc[b0], ids[b0]).tabular(FIELDS) == text_b0
            s.close()
            line["learned_vs_fifo"] = {"value": me["value"] / arms["batched_fifo"]["value"],
                                       "prelim_stage": (arms["batched_fifo"]["prelim_ms"] / me["prelim_ms"]
                                                        if me["prelim_ms"] else None)}
        line["arms"] = arms
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
