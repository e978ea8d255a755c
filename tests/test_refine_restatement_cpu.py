"""The C oracle's refinement (oracle/louvain_oracle.c, refine_partition) against the independent
Python restatement in refine_restatement.py: after a level's local moving, the refined
partition the oracle aggregates by is the restatement's, label for label, in every mode and
with a pass limit, on the reference's fixture and small generated graphs."""
import numpy as np
import pytest

import refine_restatement as R


def _graphs(graphs, golden):
    return {"fixture": golden.load_fixture(),
            "chung_lu_3000": graphs.chung_lu_bounded(3000, 2.0, 1, 99, seed=11),
            "rmat10": graphs.rmat(10, 16, seed=2)}


@pytest.mark.parametrize("name", ["fixture", "chung_lu_3000", "rmat10"])
@pytest.mark.parametrize("mode", [1, 0, 2])
def test_oracle_refine_equals_restatement(name, mode, oracle, graphs, golden):
    g = _graphs(graphs, golden)[name]
    o = oracle.Oracle(g, mode=mode, refine=True)
    o.optimization_run()
    row, col, w = o.graph()
    comm, a, k = o.comm(), o.totals(), o.k()
    labels = R.refine(row.tolist(), col.tolist(), w.tolist(), k.tolist(), comm.tolist(), a.tolist(),
                      o.total_weight, mode=mode)
    o.aggregation_run(True)
    np.testing.assert_array_equal(o.best(), R.renumber(labels))
    assert o.refine_passes >= 1


def test_oracle_refine_second_level_and_pass_limit(oracle, graphs):
    """The restatement also agrees at level 1 (an aggregated graph with self-loops and integer
    weights above 1) and under refine_passes = 1."""
    g = graphs.chung_lu_bounded(3000, 2.0, 1, 99, seed=12)
    for cap in (0, 1):
        o = oracle.Oracle(g, mode=1, refine=True, refine_passes=cap)
        o.optimization_run()
        o.aggregation_run(True)          # level 0 -> 1 (refined)
        best0 = o.best()
        o.optimization_run()
        row, col, w = o.graph()
        comm, a, k = o.comm(), o.totals(), o.k()
        assert np.any(w > 1)
        labels = R.refine(row.tolist(), col.tolist(), w.tolist(), k.tolist(), comm.tolist(),
                          a.tolist(), o.total_weight, mode=1, max_passes=cap)
        o.aggregation_run(True)
        np.testing.assert_array_equal(o.best(), R.renumber(labels)[best0])


def _random_graph(seed: int, n: int, p: float, loops: bool):
    """A random symmetric CSR with integer weights 1..3 and optional self-loop entries."""
    from importlib import import_module
    CSRGraph = import_module("louvain-fast-move-cuda_b200.graphs").CSRGraph
    rng = np.random.default_rng(seed)
    src, dst, wts = [], [], []
    for u in range(n):
        for v in range(u + 1, n):
            if rng.random() < p:
                w = float(rng.integers(1, 4))
                src += [u, v]
                dst += [v, u]
                wts += [w, w]
        if loops and rng.random() < 0.2:
            src.append(u)
            dst.append(u)
            wts.append(float(rng.integers(1, 4)))
    # every vertex needs an entry: chain the isolated ones to their successor
    deg = np.bincount(np.array(src, dtype=np.int64), minlength=n) if src else np.zeros(n, int)
    for u in range(n):
        if deg[u] == 0:
            v = (u + 1) % n
            src += [u, v]
            dst += [v, u]
            wts += [1.0, 1.0]
    order = np.lexsort((np.array(dst), np.array(src)))
    s = np.array(src, dtype=np.int64)[order]
    d = np.array(dst, dtype=np.int32)[order]
    w = np.array(wts, dtype=np.float32)[order]
    row = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(s, minlength=n), out=row[1:])
    return CSRGraph(n=n, row_ptr=row, col=d, w=w, name=f"random_{seed}")


def test_oracle_refine_equals_restatement_random(oracle):
    """Many small random graphs (n 3..60, densities 0.05..0.5, integer weights, self-loops),
    every mode: the oracle's refined partition is the restatement's."""
    hyp = pytest.importorskip("hypothesis")
    st = hyp.strategies

    @hyp.settings(max_examples=60, deadline=None, derandomize=True)
    @hyp.given(seed=st.integers(0, 10**6), n=st.integers(3, 60), p=st.floats(0.05, 0.5),
               loops=st.booleans(), mode=st.sampled_from([0, 1, 2, 3]))
    def check(seed, n, p, loops, mode):
        g = _random_graph(seed, n, p, loops)
        o = oracle.Oracle(g, mode=mode, refine=True)
        o.optimization_run()
        row, col, w = o.graph()
        labels = R.refine(row.tolist(), col.tolist(), w.tolist(), o.k().tolist(), o.comm().tolist(),
                          o.totals().tolist(), o.total_weight, mode=mode)
        o.aggregation_run(True)
        np.testing.assert_array_equal(o.best(), R.renumber(labels))

    check()


@pytest.mark.parametrize("case", ["chung_lu_1500", "rmat9", "random_a", "random_b"])
@pytest.mark.parametrize("mode", [1, 0])
def test_oracle_refined_run_equals_restatement(case, mode, oracle, graphs):
    """The whole refined run -- passes, refinement, continuation rule, the end-of-run return to
    the previous level's partition -- in the restatement gives the oracle's final partition and
    modularity."""
    g = {"chung_lu_1500": lambda: graphs.chung_lu_bounded(1500, 2.0, 1, 40, seed=3),
         "rmat9": lambda: graphs.rmat(9, 8, seed=5),
         "random_a": lambda: _random_graph(11, 60, 0.08, True),
         "random_b": lambda: _random_graph(12, 80, 0.05, False)}[case]()
    o = oracle.Oracle(g, mode=mode, refine=True)
    o.louvain()
    best, q = R.louvain_refined(g.row_ptr.tolist(), g.col.tolist(), g.weights_or_ones.tolist(), mode=mode)
    np.testing.assert_array_equal(o.best(), best)
    assert q == o.modularity


@pytest.mark.parametrize("seed,n,p,loops", [(23, 60, 0.06, False), (30, 30, 0.2, True)])
@pytest.mark.parametrize("mode", [1, 0])
def test_oracle_refined_run_returns_previous_partition(seed, n, p, loops, mode, oracle):
    """Graphs whose last level ends below the previous level's end: both return the previous
    level's partition and its modularity."""
    g = _random_graph(seed, n, p, loops)
    info = {}
    best, q = R.louvain_refined(g.row_ptr.tolist(), g.col.tolist(), g.weights_or_ones.tolist(),
                                mode=mode, info=info)
    assert info["reverted"] and info["levels"] >= 2
    o = oracle.Oracle(g, mode=mode, refine=True)
    o.louvain()
    np.testing.assert_array_equal(o.best(), best)
    assert q == o.modularity


def test_oracle_plain_run_equals_restatement_random(oracle):
    """The unrefined run too, on random small graphs in every mode: the restatement's final
    partition and modularity are the oracle's (which the reference's own goldens pin)."""
    hyp = pytest.importorskip("hypothesis")
    st = hyp.strategies

    @hyp.settings(max_examples=40, deadline=None, derandomize=True)
    @hyp.given(seed=st.integers(0, 10**6), n=st.integers(3, 60), p=st.floats(0.05, 0.5),
               loops=st.booleans(), mode=st.sampled_from([0, 1, 2, 3]), fast=st.booleans())
    def check(seed, n, p, loops, mode, fast):
        g = _random_graph(seed, n, p, loops)
        o = oracle.Oracle(g, mode=mode, fast_first=fast)
        o.louvain()
        best, q = R.louvain_plain(g.row_ptr.tolist(), g.col.tolist(), g.weights_or_ones.tolist(),
                                  mode=mode, fast_first=fast)
        np.testing.assert_array_equal(o.best(), best)
        assert q == o.modularity

    check()
