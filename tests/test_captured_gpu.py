"""The captured run (use_graphs = 1: the level loop as one CUDA graph with device-side
conditional nodes) against the host-driven run (use_graphs = 0: host reads sizes and loop
conditions back between launches). Same kernels, same order of work, so the results are
identical: communities bit-exact, modularity bit-identical, the same numbers of levels,
passes and communities, and the same per-pass trace. Forced-small degree bins put most rows
in the global-table bin, so the arena grows between levels and the captured run has to stop
and resume (graph_launches > 1) -- the result must not change.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SMALL_BINS = [1, 2, 3, 4, 5, 6, 7]


@pytest.fixture(scope="module")
def cases(graphs, golden):
    return {
        "fixture": golden.load_fixture(),
        "rmat12": graphs.rmat(12, 8, seed=3),
        "rmat16": graphs.rmat(16, 16, seed=1),
        "chung_lu_40000": graphs.chung_lu_mean(40000, seed=7),
        "planted_weighted": graphs.planted_partition(20000, 40, seed=5),
    }


def _pair(lv, **kw):
    return lv.Engine(0, use_graphs=False, **kw), lv.Engine(0, use_graphs=True, **kw)


def _same(r0, r1):
    c0, q0, s0 = r0
    c1, q1, s1 = r1
    assert np.array_equal(c0, c1)
    assert q0 == q1
    assert (s0.levels, s0.iterations, s0.n_communities) == (s1.levels, s1.iterations, s1.n_communities)
    assert s0.graph_launches == 0 and s1.graph_launches >= 1
    assert s1.kernel_launches > 0 and s1.ms_optimization_kernels > 0


@pytest.mark.parametrize("key", ["fixture", "rmat12", "rmat16", "chung_lu_40000", "planted_weighted"])
def test_captured_equals_host_driven(key, cases, lv):
    g = cases[key]
    e0, e1 = _pair(lv)
    _same(e0.run_graph(g), e1.run_graph(g))
    # a second call reuses the context's memory pool and captures again
    _same(e0.run_graph(g), e1.run_graph(g))
    e0.close()
    e1.close()


@pytest.mark.parametrize("key", ["rmat12", "rmat16", "chung_lu_40000"])
def test_captured_arena_growth_resumes(key, cases, lv):
    g = cases[key]
    e0, e1 = _pair(lv, bin_max_degree=SMALL_BINS + [0])
    r0, r1 = e0.run_graph(g), e1.run_graph(g)
    _same(r0, r1)
    e0.close()
    e1.close()


def test_captured_arena_growth_happens(cases, lv):
    """At least one of the forced-small-bin runs stops to grow its arena and resumes."""
    e1 = lv.Engine(0, use_graphs=True, bin_max_degree=SMALL_BINS + [0])
    launches = [e1.run_graph(cases[k])[2].graph_launches for k in ("rmat12", "rmat16", "chung_lu_40000")]
    e1.close()
    assert max(launches) > 1, launches


def test_captured_batch_equals_host_driven(lv, graphs):
    import importlib
    batch = importlib.import_module("louvain-fast-move-cuda_b200.batch")
    gs = [graphs.chung_lu_mean(n, seed=n) for n in (200, 1000, 5000, 300, 20000, 700)]
    gs += [graphs.rmat(s, 8, seed=s) for s in (8, 11, 13)]
    offs, row, col, w = batch.pack(gs)
    e0, e1 = _pair(lv)
    c0, q0, k0, s0 = e0.run_batch(offs, row, col)
    c1, q1, k1, s1 = e1.run_batch(offs, row, col)
    assert np.array_equal(c0, c1) and np.array_equal(q0, q1) and np.array_equal(k0, k1)
    assert s1.graph_launches >= 1
    e0.close()
    e1.close()


def test_captured_trace_equals_host_driven(cases, lv):
    g = cases["rmat16"]
    e0, e1 = _pair(lv)
    c0 = e0.community(g)
    c1 = e1.community(g)
    c0.louvain()
    c1.louvain()
    t0, t1 = c0.trace(), c1.trace()
    assert len(t0) == len(t1) > 0
    assert np.array_equal(t0, t1)
    assert np.array_equal(c0.best(), c1.best())
    c0.close()
    c1.close()
    e0.close()
    e1.close()
