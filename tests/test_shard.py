"""Query sharding over two ranks on the CPU (gloo): the joined text of the per-rank searches is
the single-run text.  The per-shard search here is the oracle (this test needs no GPU); on GPUs
each rank calls its own Searcher in the same place."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from rmblast_b200 import shard, synth

FIELDS = "6 score perc_sub qseqid qstart qend sseqid sstart send"


def test_shard_bounds_cover_and_balance():
    lens = [100, 5, 7, 300, 20, 20, 90, 1, 1, 60]
    for world in (1, 2, 3, 4, 12):
        b = shard.shard_bounds(lens, world)
        assert len(b) == world and b[0][0] == 0 and b[-1][1] == len(lens)
        assert all(x[1] == y[0] for x, y in zip(b, b[1:]))
    b = shard.shard_bounds([10] * 8, 2)
    assert b == [(0, 4), (4, 8)]
    with pytest.raises(ValueError):
        shard.shard_bounds(lens, 0)


def _workload():
    qs, db, prm = synth.workload("plain", scale=0.004)  # 4 queries of 60 kb
    p = dict(prm, **synth.RM_FLAGS)
    dbf = synth.to_fasta([n for n, _ in db], [s for _, s in db])
    return qs, dbf, p


def _oracle_search(dbf, p):
    import oracle_ref as O

    def run(queries, ids):
        if not queries:
            return ""
        qf = synth.to_fasta(ids, queries)
        txt, _, _ = O.search_text(qf, dbf, synth.MATRIX_TEXT, synth.MATRIX_NAME, p, FIELDS, threads=2)
        return txt
    return run


def _rank(rank, world, port, out_path):
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(__file__))
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        qs, dbf, p = _workload()
        txt = shard.search_sharded(_oracle_search(dbf, p), [s for _, s in qs], [n for n, _ in qs])
        if rank == 0:
            with open(out_path, "w") as f:
                f.write(txt)
        else:
            assert txt is None
    finally:
        dist.destroy_process_group()


def test_two_ranks_give_the_single_run_text(tmp_path):
    import oracle_ref as O
    O.build_oracle()
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = tmp_path / "sharded.tsv"
    mp.start_processes(_rank, args=(2, port, str(out)), nprocs=2, join=True, start_method="spawn")
    qs, dbf, p = _workload()
    want = _oracle_search(dbf, p)([s for _, s in qs], [n for n, _ in qs])
    assert want.count("\n") > 10
    assert out.read_text() == want
