"""Host-side logic without a GPU: graph generators and canonical CSR, batch packing, and
dealing graphs to ranks with results gathered over a world-size-2 gloo process group (the
per-rank runner here is the CPU oracle standing in for the device)."""
import os
import socket

import numpy as np
import pytest


def _check_canonical(g):
    assert g.row_ptr[0] == 0 and np.all(np.diff(g.row_ptr) > 0), "no isolated vertex"
    src = g.src()
    assert np.all(src != g.col), "no self-loop"
    # rows sorted by destination, no duplicate pair
    key = src.astype(np.int64) * (g.n + 1) + g.col
    assert np.all(np.diff(key) > 0)
    # symmetric: (u,v) present iff (v,u) present, with the same weight
    rkey = g.col.astype(np.int64) * (g.n + 1) + src
    order = np.argsort(rkey)
    np.testing.assert_array_equal(rkey[order], key)
    if g.w is not None:
        np.testing.assert_array_equal(g.w[order], g.w)


@pytest.mark.parametrize("make", ["chung_lu_bounded", "chung_lu_mean", "rmat", "planted"])
def test_generators_canonical_and_deterministic(make, graphs):
    f = {
        "chung_lu_bounded": lambda s: graphs.chung_lu_bounded(3000, 2.0, 1, 99, seed=s),
        "chung_lu_mean": lambda s: graphs.chung_lu_mean(3000, 2.1, 8, seed=s),
        "rmat": lambda s: graphs.rmat(11, 16, seed=s),
        "planted": lambda s: graphs.planted_partition(n=3000, n_comm=20, smin=50, smax=400, seed=s),
    }[make]
    a, b, c = f(1), f(1), f(2)
    _check_canonical(a)
    np.testing.assert_array_equal(a.row_ptr, b.row_ptr)
    np.testing.assert_array_equal(a.col, b.col)
    assert a.E != c.E or not np.array_equal(a.col, c.col)


def test_rmat_quadrant_rates(graphs):
    u, v = graphs.rmat_pairs(10, 64, seed=3)
    top = 1 << 9
    q = np.array([np.mean((u < top) & (v < top)), np.mean((u < top) & (v >= top)),
                  np.mean((u >= top) & (v < top)), np.mean((u >= top) & (v >= top))])
    np.testing.assert_allclose(q, [0.57, 0.19, 0.19, 0.05], atol=0.01)


def test_planted_partition_mixing(graphs):
    g = graphs.planted_partition(n=20000, n_comm=100, smin=100, smax=1000, mean_degree=20, mu=0.3, seed=1)
    src = g.src()
    inter = np.mean(g.truth[src] != g.truth[g.col])
    assert 0.25 < inter < 0.35
    assert g.w.min() >= 0.1 and g.w.max() <= 1.5


def test_pack_unpack_roundtrip(lv, graphs):
    batch = __import__("importlib").import_module("louvain-fast-move-cuda_b200.batch")
    gs = [graphs.chung_lu_mean(n, 2.1, 8, seed=n) for n in (300, 500, 900)]
    offs, row, col, w = batch.pack(gs)
    assert row[-1] == sum(g.E for g in gs) and offs[-1] == sum(g.n for g in gs)
    for i, g in enumerate(gs):
        lo, hi = offs[i], offs[i + 1]
        np.testing.assert_array_equal(row[lo:hi + 1] - row[lo], g.row_ptr)
        np.testing.assert_array_equal(col[row[lo]:row[hi]] - lo, g.col)


def test_deal_balances_and_is_deterministic(lv):
    batch = __import__("importlib").import_module("louvain-fast-move-cuda_b200.batch")
    rng = np.random.default_rng(0)
    sizes = rng.integers(100, 100000, 500)
    for world in (1, 2, 3, 8):
        shares = batch.deal(sizes, world)
        assert sorted(i for s in shares for i in s) == list(range(500))
        loads = [sizes[s].sum() for s in shares]
        assert max(loads) - min(loads) <= sizes.max()
        assert shares == batch.deal(sizes, world)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import importlib
    import sys
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "oracle"))
    import oracle as O
    graphs = importlib.import_module("louvain-fast-move-cuda_b200.graphs")
    batch = importlib.import_module("louvain-fast-move-cuda_b200.batch")
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    gs = [graphs.chung_lu_mean(n, 2.1, 8, seed=i) for i, n in enumerate((400, 1200, 700, 300, 2000))]

    def run_batch(sub):
        labs, qs, ks = [], [], []
        for g in sub:
            o = O.Oracle(g)
            o.louvain()
            labs.append(o.best()); qs.append(o.modularity); ks.append(o.n_best)
        return labs, qs, ks

    labels, qs, ks = batch.run_sharded(gs, run_batch, rank, world)
    q.put((rank, [l.tolist() for l in labels], qs.tolist(), ks.tolist()))
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_batch_gloo_world2(lv):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert res[0][1:] == res[1][1:], "both ranks gathered the same results"
    # and they equal a single-process run
    import importlib
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
    import oracle as O
    graphs = importlib.import_module("louvain-fast-move-cuda_b200.graphs")
    gs = [graphs.chung_lu_mean(n, 2.1, 8, seed=i) for i, n in enumerate((400, 1200, 700, 300, 2000))]
    for i, g in enumerate(gs):
        o = O.Oracle(g)
        o.louvain()
        assert res[0][1][i] == o.best().tolist()
        assert res[0][3][i] == o.n_best
