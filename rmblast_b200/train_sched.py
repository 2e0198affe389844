"""Trains the learned schedule's cost network on the GPU and writes rmblast_b200/sched_mlp.json.

    python -m rmblast_b200.train_sched [--scale 0.08] [--epochs 4] [--out PATH]

Training pairs come from a FIFO search (rmb_sched_log) of a plain-shaped workload drawn from its
own seed, so neither its genome nor its library is the benchmark's: each ungapped record's 12
features and the DP cells the thread kernel spent on it (target log1p(cells)).  The network is
trained by the library's own kernels (rmb_sched_train: Adam, FP32 with BF16-rounded weights) and
the file records its held-out RMSE next to that of the constant (mean) predictor.
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np

MODEL_PATH = Path(__file__).resolve().parent / "sched_mlp.json"
TRAIN_SEED, TEST_SEED = 0x524D42 + 500, 0x524D42 + 600


def ranking_stats(pred: np.ndarray, cells: np.ndarray) -> dict:
    """How well predictions rank records by cost: Spearman correlation, the share of the true
    costliest 1% found in the predicted top 5%, and the share of all cells in the predicted top 5%
    (the true top 5%'s share beside it)."""
    n = len(cells)
    rp = np.empty(n); rp[np.argsort(pred, kind="stable")] = np.arange(n)
    rc = np.empty(n); rc[np.argsort(cells, kind="stable")] = np.arange(n)
    k1, k5 = max(1, n // 100), max(1, n // 20)
    top_true1 = np.argsort(-cells, kind="stable")[:k1]
    top_pred5 = np.argsort(-pred, kind="stable")[:k5]
    in_pred5 = np.zeros(n, bool); in_pred5[top_pred5] = True
    tot = float(cells.sum())
    return {"spearman": round(float(np.corrcoef(rp, rc)[0, 1]), 4),
            "recall_true_top1_in_pred_top5": round(float(in_pred5[top_true1].mean()), 4),
            "cells_share_pred_top5": round(float(cells[top_pred5].sum()) / tot, 4),
            "cells_share_true_top5": round(float(np.sort(cells)[::-1][:k5].sum()) / tot, 4)}


def queue_makespan(cells: np.ndarray, order: np.ndarray, workers: int) -> int:
    """The finishing time, in DP cells, of `workers` lanes that each take the next record of one
    queue (in `order`) when their last one is done -- the record queue of k_prelim_stream, with a
    record's time taken as its cells.  Records are handed out in queue order to whichever lane is
    free first (list scheduling), the lanes all starting at 0."""
    import heapq
    c = np.asarray(cells, dtype=np.int64)[np.asarray(order)]
    w = min(workers, len(c))
    if w == 0:
        return 0
    free = [int(x) for x in c[:w]]
    heapq.heapify(free)
    for x in c[w:].tolist():
        heapq.heapreplace(free, free[0] + x)
    return max(free)


def cost_bins(pred: np.ndarray) -> np.ndarray:
    """rmb_sched.cuh sched_bin: 64 bins a quarter of a log-cell wide (0 for <= 0, 63 from 15.75)."""
    b = np.asarray(pred, dtype=np.float32) * np.float32(4.0)
    return np.where(b <= 0, 0, np.where(b >= 63, 63, np.trunc(np.clip(b, 0, 63)))).astype(np.int64)


def front_loaded_order(pred: np.ndarray, front_div: int = 32) -> np.ndarray:
    """The queue order of schedule 1 (k_sched_cut + the partition in rmb_kernels.cu) on the host:
    the records in the costliest of 64 predicted-cost bins, as many bins as hold at most
    n / front_div records, in arrival order, then the rest in reverse arrival order."""
    pred = np.asarray(pred, dtype=np.float32)
    b = cost_bins(pred)
    hist = np.bincount(b, minlength=64)
    limit, acc, cut = len(pred) // front_div, 0, 64
    for k in range(63, -1, -1):
        if acc + hist[k] > limit:
            break
        acc += hist[k]
        cut = k
    sel = b >= cut
    idx = np.arange(len(pred))
    return np.concatenate([idx[sel], idx[~sel][::-1]])


def load_model(path: Path = MODEL_PATH) -> np.ndarray:
    """The committed network parameters (rmb_sched layout) for Searcher.set_schedule_model."""
    return np.asarray(json.loads(path.read_text())["params"], dtype=np.float32)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scale", type=float, default=0.08, help="fraction of the plain workload's 1,000 queries")
    ap.add_argument("--epochs", type=int, default=4)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--out", default=str(MODEL_PATH))
    ap.add_argument("--test-scale", type=float, default=0.02)
    args = ap.parse_args()
    from rmblast_b200 import api, build, synth
    build.build()
    qs, db, prm = synth.workload("plain", seed=TRAIN_SEED, scale=args.scale)
    p = dict(prm, **synth.RM_FLAGS)
    m = api.ScoreMatrix.from_text(synth.MATRIX_TEXT, synth.MATRIX_NAME)
    sp = api.SearchParams(gap_open=p["gap_open"], gap_extend=p["gap_extend"], word_size=p["word_size"],
                          xdrop_ungap=p["xdrop_ungap"], xdrop_gap=p["xdrop_gap"], xdrop_gap_final=p["xdrop_gap_final"],
                          min_raw_gapped_score=p["min_raw_gapped_score"], complexity_adjust=True,
                          mask_level=p["mask_level"], device=args.device)
    s = api.Searcher(sp, m, api.SubjectDb.from_records(db))
    # the test set: another seed's workload (its own genome and library)
    tq, tdb, _ = synth.workload("plain", seed=TEST_SEED, scale=args.test_scale)
    st = api.Searcher(sp, m, api.SubjectDb.from_records(tdb))
    t_feats, t_cells = st.schedule_log([api.encode(x) for _, x in tq])
    t0 = time.time()
    feats, cells = s.schedule_log([api.encode(x) for _, x in qs])
    t_log = time.time() - t0
    target = np.log1p(cells.astype(np.float64)).astype(np.float32)
    p0 = api.sched_init(feats, args.seed, target)
    t0 = time.time()
    params, mse, rmse = api.sched_train(feats, target, p0, epochs=args.epochs, batch=args.batch, lr=args.lr,
                                        seed=args.seed, val_fraction=0.1, device=args.device)
    t_train = time.time() - t0
    t_target = np.log1p(t_cells.astype(np.float64))
    t_pred = api.sched_predict(params, t_feats, device=args.device).astype(np.float64)
    info = {
        "workload": f"plain, seed {TRAIN_SEED:#x}, {len(qs)} queries of 60 kb vs its own 2,000-consensus library",
        "pairs": int(len(cells)), "epochs": args.epochs, "batch": args.batch, "lr": args.lr, "seed": args.seed,
        "train_mse_per_epoch": [round(float(x), 5) for x in mse],
        "heldout_rmse_log_cells": round(rmse, 4),
        "mean_predictor_rmse_log_cells": round(float(target.std()), 4),
        "test_workload": f"plain, seed {TEST_SEED:#x}, {len(tq)} queries, {len(t_cells)} records",
        "test_rmse_log_cells": round(float(np.sqrt(np.mean((t_pred - t_target) ** 2))), 4),
        "test_mean_predictor_rmse": round(float(t_target.std()), 4),
        "test_ranking": ranking_stats(t_pred, t_cells.astype(np.float64)),
        "log_seconds": round(t_log, 2), "train_seconds": round(t_train, 2),
    }
    Path(args.out).write_text(json.dumps({"info": info, "params": [float(x) for x in params]}) + "\n")
    print(json.dumps(info))


if __name__ == "__main__":
    main()
