"""Host side of the learned schedule, without a GPU: the parameter layout the C ABI expects,
the initial parameters, the committed model file and the ranking statistics of the training
script."""
import json

import numpy as np

from rmblast_b200 import api, train_sched

NF, H, NET, NPARAM = api.SCHED_NF, api.SCHED_H, api.SCHED_NET, api.SCHED_NPARAM


def test_layout_matches_the_header():
    text = (api.LIB_PATH.parent.parent.parent / "include" / "rmb_gpu.h").read_text()
    assert f"#define RMB_SCHED_NET {NET}" in text and f"#define RMB_SCHED_NPARAM {NPARAM}" in text
    assert NET == NF * H + H + H * H + H + H + 1 and NPARAM == NET + 2 * NF


def test_init_normalises_and_centres_the_output():
    rng = np.random.default_rng(0)
    f = rng.normal([1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12], 2.0, (5000, NF)).astype(np.float32)
    f[:, 7] = 1.0  # a constant feature (the strand of a one-strand set) keeps a unit scale
    t = rng.normal(7.5, 0.3, 5000)
    p = api.sched_init(f, 1, t)
    mean, istd = p[NET:NET + NF], p[NET + NF:]
    np.testing.assert_allclose(mean, f.mean(axis=0), rtol=1e-5, atol=1e-5)
    assert istd[7] == 1.0
    z = (f - mean) * istd
    np.testing.assert_allclose(np.delete(z.std(axis=0), 7), 1.0, rtol=1e-3)
    assert abs(p[NET - 1] - t.mean()) < 1e-5  # output bias
    assert np.all(p[NF * H:NF * H + H] == 0)  # hidden biases start at zero
    assert np.array_equal(p, api.sched_init(f, 1, t))  # seeded


def test_committed_model():
    d = json.loads(train_sched.MODEL_PATH.read_text())
    p = train_sched.load_model()
    assert p.shape == (NPARAM,) and np.isfinite(p).all()
    info = d["info"]
    assert info["pairs"] > 1_000_000
    assert info["heldout_rmse_log_cells"] < info["mean_predictor_rmse_log_cells"]


def test_ranking_stats():
    rng = np.random.default_rng(2)
    cells = rng.lognormal(7.0, 0.5, 20000)
    perfect = train_sched.ranking_stats(np.log(cells), cells)
    assert perfect["spearman"] > 0.999 and perfect["recall_true_top1_in_pred_top5"] == 1.0
    assert perfect["cells_share_pred_top5"] == perfect["cells_share_true_top5"]
    chance = train_sched.ranking_stats(rng.normal(size=20000), cells)
    assert abs(chance["spearman"]) < 0.05 and chance["recall_true_top1_in_pred_top5"] < 0.15


def test_queue_makespan_list_scheduling():
    """The queue simulation behind the schedule's gain test: lanes take records in queue order,
    each record going to the lane that is free first."""
    cells = np.array([5, 1, 1, 1, 1, 1])
    assert train_sched.queue_makespan(cells, np.arange(6), 2) == 5  # 5 | 1+1+1+1+1
    assert train_sched.queue_makespan(cells, np.arange(6)[::-1], 2) == 7  # the long record last
    assert train_sched.queue_makespan(cells, np.arange(6), 1) == 10
    assert train_sched.queue_makespan(cells, np.arange(6), 64) == 5
    rng = np.random.default_rng(3)
    c = rng.integers(1, 1000, 5000)
    # longest first is never worse than 4/3 of the optimum; any order is within 2x the lower bound
    lb = max(c.sum() / 16, c.max())
    assert train_sched.queue_makespan(c, np.argsort(-c, kind="stable"), 16) <= 4 / 3 * lb + 1
    assert train_sched.queue_makespan(c, np.arange(5000), 16) <= 2 * lb


def test_front_loaded_order():
    """Schedule 1's queue on the host: the costliest bins (at most n / 32 records) first in arrival
    order, the others after them in reverse arrival order."""
    rng = np.random.default_rng(5)
    pred = rng.normal(7.0, 1.0, 4096).astype(np.float32)
    order = train_sched.front_loaded_order(pred)
    assert sorted(order.tolist()) == list(range(4096))
    b = train_sched.cost_bins(pred)
    hist = np.bincount(b, minlength=64)
    cut = 64
    while cut > 0 and hist[cut - 1:].sum() <= 4096 // 32:
        cut -= 1
    nf = int((b >= cut).sum())
    front, back = order[:nf], order[nf:]
    assert 0 < len(front) <= 4096 // 32
    assert (np.diff(front) > 0).all() and (np.diff(back) < 0).all()
    assert b[front].min() > b[back].max()
    assert train_sched.cost_bins(np.array([-1.0, 0.0, 0.3, 2.26, 15.8, 99.0])).tolist() == [0, 0, 1, 9, 63, 63]
