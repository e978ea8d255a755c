"""Sharded batches through the engine: batch.run_sharded with batch.engine_runner, i.e. each
rank packs its share of the graphs and runs it with lv_run_batch, then the per-graph results
are gathered on the host over gloo. Results must equal one lv_run_batch call over all graphs
and the oracle's single-graph runs.

World size 1 runs in this process inside a one-rank gloo group. World size 2 runs two spawned
processes that both use cuda:0: their kernels never wait on one another (each runs its own
independent batch; the only exchange is the host-side object gather), so sharing one GPU is
safe. The reference has no batching or multi-GPU path (main.cu:19-39)."""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _graph_set(graphs):
    return [graphs.chung_lu_mean(n, 2.1, 8, seed=i) for i, n in enumerate((400, 1200, 700, 300, 2000, 5000))] + \
           [graphs.rmat(12, 8, seed=3), graphs.planted_partition(n=3000, n_comm=30, smin=20, smax=300,
                                                                  mean_degree=10, seed=4)]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _check_against_batch_and_oracle(lv, graphs, oracle, labels, qs, ks):
    import importlib
    batch = importlib.import_module("louvain-fast-move-cuda_b200.batch")
    gs = _graph_set(graphs)
    e = lv.Engine(0)
    offs, row, col, w = batch.pack(gs)
    out, bq, bk, _ = e.run_batch(offs, row, col, w)
    e.close()
    ref = batch.unpack(out, offs)
    for i, g in enumerate(gs):
        np.testing.assert_array_equal(np.asarray(labels[i]), ref[i])
        assert ks[i] == bk[i]
        assert abs(qs[i] - bq[i]) <= 1e-12
        o = oracle.Oracle(g)
        o.louvain()
        np.testing.assert_array_equal(np.asarray(labels[i]), o.best())
        assert ks[i] == o.n_best
        assert abs(qs[i] - o.modularity) <= 1e-12


def test_sharded_engine_world1(lv, graphs, oracle):
    import importlib
    import torch.distributed as dist
    batch = importlib.import_module("louvain-fast-move-cuda_b200.batch")
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1)
    try:
        e = lv.Engine(0)
        labels, qs, ks = batch.run_sharded(_graph_set(graphs), batch.engine_runner(e), 0, 1)
        e.close()
        dist.barrier()
    finally:
        dist.destroy_process_group()
    _check_against_batch_and_oracle(lv, graphs, oracle, labels, qs, ks)


def _rank_main(rank, world, port, q):
    import importlib
    import sys
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    lv = importlib.import_module("louvain-fast-move-cuda_b200")
    graphs = importlib.import_module("louvain-fast-move-cuda_b200.graphs")
    batch = importlib.import_module("louvain-fast-move-cuda_b200.batch")
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        e = lv.Engine(0)
        labels, qs, ks = batch.run_sharded(_graph_set(graphs), batch.engine_runner(e), rank, world)
        e.close()
        q.put((rank, [np.asarray(l).tolist() for l in labels], qs.tolist(), ks.tolist()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_sharded_engine_world2_gloo(lv, graphs, oracle):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=600) for _ in procs]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res.sort()
    assert res[0][1:] == res[1][1:], "both ranks gathered the same results"
    _check_against_batch_and_oracle(lv, graphs, oracle, res[0][1], res[0][2], res[0][3])
