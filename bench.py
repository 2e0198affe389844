#!/usr/bin/env python
"""Benchmark of the B200 rmblastn search core on the genome-vs-TE-library workloads.

Default workload ("plain", one GPU): 1,000 query chunks of 60 kb (60 Mb, 45% planted repeats at
2-35% divergence, 1% N runs) against 2,000 synthetic consensi (about 5 Mb), word 11, gap costs
20/5, complexity adjustment, masklevel 80, dust off, RepeatMasker's cutoffs and X-drops
(min_raw_gapped_score 200, xdrop_ungap 400, xdrop_gap 100, xdrop_gap_final 200).

A step is one search of the whole query set through the full path (lookup tables, scan,
extensions, dedup, prelim DP, interval-tree filters, traceback DP, complexity adjustment,
purges, masklevel, hit order).
  value  query Mbp/s with queries and library resident in HBM (rmb_search_resident)
  e2e    the same through rmb_search_batch from host buffers plus the outfmt-6 text of every
         HSP (host->device query copy and device->host results inside the timed region)

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Multi-GPU (weak scaling): each rank searches its own query set of the same size (seeded by
rank) against the full library; no collective is on the data path.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

FIELDS = "6 score perc_sub qseqid qstart qend sseqid sstart send"
OPS_PER_CELL = 11  # int32 add/sub/max/compare per DP cell in search/gapped.rs:234-262
# DRAM bytes (read + write) per ungapped record of k_prelim_stream, from one ncu capture of
# `bench.py --scale 0.01` (1.31 M records, 80.1 MB); the traffic is per record (the
# 48-byte geometry read, the 28-byte result write, sequence words), so a launch's traffic is
# this times its records
PRELIM_STREAM_DRAM_BYTES_PER_RECORD = 61.0
# copy bandwidth of this pool's B200s measured earlier, used when MEASURED_PEAKS.json is absent
HBM_FALLBACK_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="plain", choices=["plain", "small", "batched", "allvsall"])
    ap.add_argument("--scale", type=float, default=1.0, help="fraction of the query set (tests/profiling)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU baseline sample budget")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--dust", action="store_true", help="mask the queries with DUST (the reference's default)")
    ap.add_argument("--schedule", choices=["fifo", "learned"], default="fifo",
                    help="prelim DP record order: FIFO, or the learned cost order (rmblast_b200/sched_mlp.json)")
    ap.add_argument("--sched-model", default=None, help="schedule network JSON (default: the committed one)")
    return ap.parse_args()


def workload(name: str, scale: float, rank: int, dust: bool = False):
    from rmblast_b200 import synth
    seed = None if rank == 0 else 0x524D42 + 1000 + rank
    qs, db, prm = synth.workload(name, seed=seed, scale=scale)
    if name in ("plain", "batched") and rank:
        # every rank shares the library of the workload; only the query set changes
        _, db, _ = synth.workload(name, scale=1e-9)
    p = dict(prm, **synth.RM_FLAGS)
    if dust:
        p["dust"] = 1
    return qs, db, p


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


def cpu_baseline(qs, db, p, budget_s: float):
    """The C++ restatement of the reference CPU path (oracle) on all host cores, over the first
    queries of the same workload until the time budget is spent (at least two queries)."""
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_ref as O
    from rmblast_b200 import synth
    threads = os.cpu_count() or 1
    dbf = synth.to_fasta([n for n, _ in db], [s for _, s in db])
    bases, secs, n = 0, 0.0, 0
    for name, s in qs:
        qf = synth.to_fasta([name], [s])
        _, _, t = O.search_text(qf, dbf, synth.MATRIX_TEXT, synth.MATRIX_NAME, p, FIELDS, threads=threads)
        bases += len(s)
        secs += t
        n += 1
        if secs >= budget_s and n >= 2:
            break
    return {"value": bases / secs / 1e6, "unit": "Mbp/s", "cores": threads, "kind": "port", "cpu_model": cpu_model(),
            "sample": f"{n} of {len(qs)} queries ({bases} bp) vs the full library, {secs:.1f} s, C++ restatement "
                      f"of the reference CPU path (mt-mode 0 split by subject, {threads} threads)"}


def reference_arm(args, rank, world):
    if rank != 0:
        return
    qs, db, p = workload(args.workload, args.scale, 0, args.dust)
    # each step is a bounded sample of the same workload
    per_step = max(2.0, 60.0 / max(1, args.steps + args.warmup))
    vals = []
    cb = None
    for i in range(args.warmup + args.steps):
        cb = cpu_baseline(qs, db, p, per_step)
        if i >= args.warmup:
            vals.append(cb["value"])
    v = statistics.mean(vals)
    line = {"metric": "query Mbp/s", "value": v, "unit": "Mbp/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded genome/TE-library model)",
            "impl": "reference",
            "config": {"workload": args.workload, "queries": len(qs), "query_bp": sum(len(s) for _, s in qs),
                       "library": len(db), "word_size": p["word_size"]},
            "cpu_baseline": dict(cb, value=v), "e2e": {"value": v, "unit": "Mbp/s", "h2d_bytes_per_step": 0,
                                                        "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def scan_roofline(n_queries: int, sdb, c: dict, peaks: dict) -> dict:
    """The seed scan against HBM: algorithmic bytes = every query reads the whole packed library
    (a byte per 4 bases) and every word hit writes 8 bytes; the library (~1.2 MB packed) stays
    in L2, so DRAM carries far less and the stage is bound by its random probes into the query
    tables, not by bandwidth."""
    packed = sum((len(p) - 2 + 3) // 4 for p in sdb.plus)
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
    import numpy as np
    import torch
    from rmblast_b200 import api, build, synth
    build.build()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    qs, db, p = workload(args.workload, args.scale, rank, args.dust)
    m = api.ScoreMatrix.from_text(synth.MATRIX_TEXT, synth.MATRIX_NAME)
    sp = api.SearchParams(gap_open=p["gap_open"], gap_extend=p["gap_extend"], word_size=p["word_size"],
                          xdrop_ungap=p["xdrop_ungap"], xdrop_gap=p["xdrop_gap"], xdrop_gap_final=p["xdrop_gap_final"],
                          min_raw_gapped_score=p["min_raw_gapped_score"], complexity_adjust=bool(p["complexity_adjust"]),
                          mask_level=p["mask_level"], dust=bool(p.get("dust", 0)), device=local,
                          schedule=1 if args.schedule == "learned" else 0)
    sdb = api.SubjectDb.from_records(db)
    s = api.Searcher(sp, m, sdb)
    if args.schedule == "learned":
        from rmblast_b200 import train_sched
        s.set_schedule_model(train_sched.load_model(Path(args.sched_model) if args.sched_model else
                                                    train_sched.MODEL_PATH))
    enc = [api.encode(x) for _, x in qs]
    ids = [n for n, _ in qs]
    bases = sum(len(x) for _, x in qs)
    h2d = int(sum(len(e) for e in enc))

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

    # ---- value: resident inputs
    rq = s.upload(enc)
    for _ in range(args.warmup):
        r = s.search_resident(rq, ids)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ctrs = []
    with ClockSampler(local) as clk:
        barrier()
        ev0.record()
        for _ in range(args.steps):
            r = s.search_resident(rq, ids)
            ctrs.append(r.counters)
        ev1.record()
        barrier()
    ms_total = ev0.elapsed_time(ev1)
    ms_step = max_over_ranks(ms_total / args.steps)
    n_hsps = r.n_hsps
    rq.free()
    # ---- e2e: host buffers in, outfmt-6 text out
    for _ in range(max(1, args.warmup // 2)):
        r2 = s.search(enc, ids)
        txt = r2.tabular(FIELDS)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record()
    d2h = 0
    for _ in range(args.steps):
        r2 = s.search(enc, ids)
        txt = r2.tabular(FIELDS)
        d2h = len(txt)
    e1.record()
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)

    c = {k: statistics.mean(x[k] for x in ctrs) for k in ctrs[0]}
    peak_int = api.int32_peak_tops(local)
    prelim_ms = c["gpu_ms_prelim"]
    so_cells = c["so_cells"]
    # the dominant kernel: k_prelim_stream (one launch per step), timed alone with CUDA events
    main_ms, main_cells = c["gpu_ms_prelim_main"], c["so_cells_main"]
    if main_ms <= 0:  # parameters outside the thread kernel's range: the warp kernel does it all
        main_ms, main_cells = prelim_ms, so_cells
    achieved = main_cells * OPS_PER_CELL / (main_ms * 1e-3) / 1e12 if main_ms > 0 else 0.0
    traffic = (PRELIM_STREAM_DRAM_BYTES_PER_RECORD * c["prelim_dp"]
               if PRELIM_STREAM_DRAM_BYTES_PER_RECORD and c["gpu_ms_prelim_main"] > 0 else None)
    value = bases * world / (ms_step * 1e-3) / 1e6
    peaks, peak_source = {"hbm_gbs": HBM_FALLBACK_GBS}, "fallback"
    pk = ROOT / "MEASURED_PEAKS.json"
    if pk.exists():
        peaks, peak_source = json.loads(pk.read_text()), "measured"
    line = {
        "metric": "query Mbp/s", "value": value, "unit": "Mbp/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded genome/TE-library model)",
        "config": {"workload": args.workload, "queries_per_gpu": len(qs), "query_bp_per_gpu": bases,
                   "library": len(db), "library_bp": sdb.total_letters(), "word_size": p["word_size"],
                   "flags": f"gapopen {p['gap_open']} gapextend {p['gap_extend']} "
                            f"{'complexity_adjust ' if p.get('complexity_adjust') else ''}"
                            f"masklevel {p['mask_level']} dust {'yes' if p.get('dust') else 'no'} "
                            f"min_raw_gapped_score {p['min_raw_gapped_score']} xdrop_ungap {p['xdrop_ungap']} "
                            f"xdrop_gap {p['xdrop_gap']} xdrop_gap_final {p['xdrop_gap_final']}",
                   "l2": "inputs larger than L2 (lookup tables and hit arrays are GBs per step)",
                   "parallelism": f"{world} independent ranks, queries sharded by rank",
                   "schedule": args.schedule},
        "gcups": so_cells / (prelim_ms * 1e-3) / 1e9 if prelim_ms > 0 else None,
        "traceback_gcups": c["tb_cells"] / (c["gpu_ms_traceback"] * 1e-3) / 1e9 if c["gpu_ms_traceback"] > 0 else None,
        "scan_roofline": scan_roofline(len(qs), sdb, c, peaks),
        "stage_ms": dict({k: round(c[k], 3) for k in ("gpu_ms_lookup", "gpu_ms_scan", "gpu_ms_ungapped",
                                                      "gpu_ms_dedup", "gpu_ms_prelim", "gpu_ms_traceback",
                                                      "ms_host_2a", "ms_host_2b")},
                         # DUST runs once per uploaded query set: its time is the e2e search's
                         gpu_ms_dust_e2e=round(r2.counters["gpu_ms_dust"], 3)),
        "counts": {k: int(c[k]) for k in ("word_hits", "ungapped", "prelim_dp", "prelims", "tb_dp", "finals",
                                          "so_cells", "tb_cells")},
        "hsps": n_hsps,
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
        "gpu_launches": int(c["launches"]) * args.steps,
        "clocks": clk.summary(),
        "e2e": {"value": bases * world / (e2e_ms * 1e-3) / 1e6, "unit": "Mbp/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(qs, db, p, args.cpu_seconds)
    if rank == 0:
        print(json.dumps(line), flush=True)
    s.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
