"""The learned schedule of the preliminary DP (rmb_sched.cuh, rmb_sched.cu).

* The inference kernel (BF16 mma, FP32 accumulation) against a torch CPU restatement of the same
  network with the same roundings (BF16 weights, inputs and hidden activations).
* The training kernels' loss and gradient against torch autograd (FP32, BF16-rounded weights).
* Training on logged (features, cells) pairs lowers the loss and predicts held-out cells better
  than the mean does.
* A search with the learned cost order gives the same output as the FIFO queue: the network only
  orders work.
"""
import numpy as np
import pytest

from rmblast_b200 import api, build, synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

NF, H, NET = api.SCHED_NF, api.SCHED_H, api.SCHED_NET


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def _bf16(x):
    return torch.as_tensor(x, dtype=torch.float32).to(torch.bfloat16).to(torch.float32)


def _unpack(p):
    p = torch.as_tensor(p, dtype=torch.float32)
    o = 0
    w1 = p[o:o + NF * H].reshape(NF, H); o += NF * H
    b1 = p[o:o + H]; o += H
    w2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    w3 = p[o:o + H]; o += H
    b3 = p[o]; o += 1
    return w1, b1, w2, b2, w3, b3, p[o:o + NF], p[o + NF:o + 2 * NF]


def _random_case(n, seed):
    rng = np.random.default_rng(seed)
    f = rng.normal(2.0, 1.5, (n, NF)).astype(np.float32)
    p = api.sched_init(f, seed)
    p[:NET] += rng.normal(0, 0.05, NET).astype(np.float32)  # non-zero biases too
    t = rng.normal(6.0, 2.0, n).astype(np.float32)
    return f, p, t


def test_predict_kernel_matches_torch():
    f, p, _ = _random_case(1000, 1)  # 31 full warps and a ragged one
    got = api.sched_predict(p, f)
    w1, b1, w2, b2, w3, b3, mean, istd = _unpack(p)
    x = _bf16((torch.as_tensor(f) - mean) * istd)
    h1 = _bf16(torch.relu(x @ _bf16(w1) + b1))
    h2 = _bf16(torch.relu(h1 @ _bf16(w2) + b2))
    want = (h2 @ _bf16(w3) + b3).numpy()
    # same roundings; FP32 sums in another order can flip a BF16 rounding of a hidden unit
    np.testing.assert_allclose(got, want, rtol=1e-2, atol=2e-2)
    assert np.corrcoef(got, want)[0, 1] > 0.9999


def test_grad_matches_torch_autograd():
    f, p, t = _random_case(777, 2)
    loss, g = api.sched_grad(p, f, t)
    w1, b1, w2, b2, w3, b3, mean, istd = _unpack(p)
    ws = [_bf16(w1).requires_grad_(), _bf16(b1).requires_grad_(), _bf16(w2).requires_grad_(),
          _bf16(b2).requires_grad_(), _bf16(w3).requires_grad_(), _bf16(b3).requires_grad_()]
    x = (torch.as_tensor(f) - mean) * istd
    h1 = torch.relu(x @ ws[0] + ws[1])
    h2 = torch.relu(h1 @ ws[2] + ws[3])
    y = h2 @ ws[4] + ws[5]
    ref = ((y - torch.as_tensor(t)) ** 2).mean()
    ref.backward()
    want = torch.cat([w.grad.reshape(-1) for w in ws]).numpy()
    assert abs(loss - ref.item()) <= 1e-4 * abs(ref.item())
    np.testing.assert_allclose(g, want, rtol=1e-3, atol=1e-4 * np.abs(want).max())


def _searcher(p, schedule=0):
    m = api.ScoreMatrix.from_text(synth.MATRIX_TEXT, synth.MATRIX_NAME)
    return m, api.SearchParams(gap_open=p["gap_open"], gap_extend=p["gap_extend"], word_size=p["word_size"],
                               xdrop_ungap=p["xdrop_ungap"], xdrop_gap=p["xdrop_gap"],
                               xdrop_gap_final=p["xdrop_gap_final"],
                               min_raw_gapped_score=p["min_raw_gapped_score"], complexity_adjust=True,
                               mask_level=p["mask_level"], schedule=schedule)


@pytest.fixture(scope="module")
def logged():
    # (features, cells) of a FIFO search on a separately seeded plain workload
    qs, db, prm = synth.workload("plain", seed=0x524D42 + 700, scale=0.02)
    p = dict(prm, **synth.RM_FLAGS)
    m, sp = _searcher(p)
    s = api.Searcher(sp, m, api.SubjectDb.from_records(db))
    f, c = s.schedule_log([api.encode(x) for _, x in qs])
    return f, c


def test_logged_pairs_are_the_searchs_records(logged):
    f, c = logged
    assert len(f) == len(c) > 100_000 and f.shape[1] == NF
    assert np.isfinite(f).all() and (c > 0).all()


def test_training_beats_the_mean(logged):
    f, c = logged
    t = np.log1p(c.astype(np.float64)).astype(np.float32)
    p0 = api.sched_init(f, 3, t)
    p, mse, rmse = api.sched_train(f, t, p0, epochs=4, batch=8192, lr=1e-3, seed=3, val_fraction=0.1)
    assert mse[-1] < mse[0] and mse[-1] < float(t.var())
    # held out: below the mean's RMSE (the std).  Most records here cost about the same (an
    # X-drop walk through unrelated sequence; log-cell std ~0.3), so the margin is small
    assert rmse < float(t.std())
    assert np.isfinite(p).all()
    # and the inference kernel ranks records by cost better than chance
    pred = api.sched_predict(p, f)
    rank = lambda x: np.argsort(np.argsort(x, kind="stable"), kind="stable")  # noqa: E731
    assert np.corrcoef(rank(pred), rank(c))[0, 1] > 0.05


def test_learned_order_gives_the_fifo_output(logged):
    f, c = logged
    t = np.log1p(c.astype(np.float64)).astype(np.float32)
    p, _, _ = api.sched_train(f, t, api.sched_init(f, 4, t), epochs=1, batch=8192, seed=4)
    qs, db, prm = synth.workload("plain", scale=0.01)
    prm = dict(prm, **synth.RM_FLAGS)
    enc = [api.encode(x) for _, x in qs]
    ids = [n for n, _ in qs]
    fields = "6 score perc_sub qseqid qstart qend sseqid sstart send"
    outs = []
    for schedule, params in ((0, None), (1, p), (1, api.sched_init(f, 5))):
        m, sp = _searcher(prm, schedule)
        s = api.Searcher(sp, m, api.SubjectDb.from_records(db))
        if params is not None:
            s.set_schedule_model(params)
        r = s.search(enc, ids)
        outs.append((r.tabular(fields), r.counters["so_cells"]))
    assert outs[0][0] and outs[1] == outs[0] and outs[2] == outs[0]


def test_learned_schedule_needs_a_model():
    qs, db, prm = synth.workload("small", scale=0.05)
    m, sp = _searcher(dict(prm, **synth.RM_FLAGS), 1)
    s = api.Searcher(sp, m, api.SubjectDb.from_records(db))
    with pytest.raises(api.RmbError):
        s.search([api.encode(x) for _, x in qs])


def test_learned_order_shortens_the_record_queue():
    """What the trained network gains over the FIFO queue, measured without timing noise: the DP
    cells of every record of a workload the network never saw (rmb_sched_log), the records taken
    by as many lanes as the persistent DP grid gives each lane on the full plain workload (~1,160
    records a lane), in FIFO order and in the network's descending predicted cost.  The learned
    order finishes earlier: its makespan is shorter than FIFO's (the true-cost order, longest first,
    is printed beside them as the reference point).  Inputs are seeded and the network fixed, so the
    comparison is deterministic."""
    from rmblast_b200 import train_sched
    qs, db, prm = synth.workload("plain", seed=train_sched.TEST_SEED + 7, scale=0.01)
    p = dict(prm, **synth.RM_FLAGS)
    sp = api.SearchParams(gap_open=p["gap_open"], gap_extend=p["gap_extend"], word_size=p["word_size"],
                          xdrop_ungap=p["xdrop_ungap"], xdrop_gap=p["xdrop_gap"], xdrop_gap_final=p["xdrop_gap_final"],
                          min_raw_gapped_score=p["min_raw_gapped_score"], complexity_adjust=True,
                          mask_level=p["mask_level"])
    s = api.Searcher(sp, api.ScoreMatrix.from_text(synth.MATRIX_TEXT, synth.MATRIX_NAME),
                     api.SubjectDb.from_records(db))
    feats, cells = s.schedule_log([api.encode(x) for _, x in qs])
    s.close()
    pred = api.sched_predict(train_sched.load_model(), feats)
    lanes = max(1, len(cells) // 1160)
    fifo = train_sched.queue_makespan(cells, np.arange(len(cells)), lanes)
    learned = train_sched.queue_makespan(cells, np.argsort(-pred, kind="stable"), lanes)
    ideal = train_sched.queue_makespan(cells, np.argsort(-cells.astype(np.int64), kind="stable"), lanes)
    # the library's default learned layout: the predicted-costliest 1/32 first, the rest reversed
    front = train_sched.front_loaded_order(pred)
    loaded = train_sched.queue_makespan(cells, front, lanes)
    print(f"records {len(cells)} lanes {lanes} makespan fifo {fifo} learned {learned} front-loaded {loaded} "
          f"true-cost order {ideal}")
    assert learned < fifo and loaded < fifo
