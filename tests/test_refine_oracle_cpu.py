"""The oracle's refinement (refine=True) on the CPU: the refined partition of a level is nested
in the level's partition and every refined community is connected; results do not depend on
the thread count; the refined run ends with no disconnected community on the reference's
fixture and never below the plain run's modularity on these graphs."""
import numpy as np
import pytest

from test_refine_gpu import _components_ok


def _disconnected(g, best):
    import scipy.sparse as sp
    from scipy.sparse.csgraph import connected_components
    A = sp.csr_matrix((np.ones(g.col.size), g.col, g.row_ptr), shape=(g.n, g.n))
    bad = 0
    for c in np.unique(best):
        idx = np.flatnonzero(best == c)
        if idx.size > 1 and connected_components(A[idx][:, idx], directed=False)[0] > 1:
            bad += 1
    return bad


@pytest.mark.parametrize("which", ["fixture", "rmat12", "chung_lu"])
def test_refined_partition_nested_connected(which, oracle, graphs, golden):
    g = {"fixture": lambda: golden.load_fixture(),
         "rmat12": lambda: graphs.rmat(12, 16, seed=3),
         "chung_lu": lambda: graphs.chung_lu_bounded(6000, 2.0, 1, 99, seed=6)}[which]()
    o = oracle.Oracle(g, mode=1, refine=True)
    o.optimization_run()
    coarse = o.comm()
    o.aggregation_run(True)
    ref = o.best()
    assert o.refine_passes > 0
    assert np.unique(ref).size == o.n < g.n
    _components_ok(g, ref, coarse)


def test_refine_thread_count_independent(oracle, graphs):
    g = graphs.rmat(13, 16, seed=5)
    runs = []
    for nt in (1, 4):
        o = oracle.Oracle(g, mode=1, refine=True, nthreads=nt)
        o.louvain()
        runs.append((o.best(), o.modularity, o.refine_passes, o.trace()))
    np.testing.assert_array_equal(runs[0][0], runs[1][0])
    assert runs[0][1] == runs[1][1] and runs[0][2] == runs[1][2]
    np.testing.assert_array_equal(runs[0][3], runs[1][3])


def test_refine_quality_on_fixture_and_generators(oracle, graphs, golden):
    for g in (golden.load_fixture(), graphs.chung_lu_bounded(10000, 2.0, 1, 99, seed=4),
              graphs.rmat(13, 16, seed=1)):
        plain = oracle.Oracle(g, mode=1)
        plain.louvain()
        ref = oracle.Oracle(g, mode=1, refine=True)
        ref.louvain()
        assert ref.modularity >= plain.modularity
    fx = golden.load_fixture()
    o = oracle.Oracle(fx, mode=1, refine=True)
    o.louvain()
    assert _disconnected(fx, o.best()) == 0


def test_refine_off_is_the_plain_run(oracle, graphs):
    g = graphs.rmat(12, 16, seed=2)
    a = oracle.Oracle(g, mode=1)
    a.louvain()
    b = oracle.Oracle(g, mode=1, refine=False, refine_passes=3, refine_tolerance=0.5)
    b.louvain()
    np.testing.assert_array_equal(a.best(), b.best())
    assert a.modularity == b.modularity and b.refine_passes == 0


@pytest.mark.parametrize("name", ["stars", "ring_of_cliques", "int_weights", "self_loops", "components"])
def test_refined_partition_edge_cases(name, oracle, graphs):
    from test_refine_gpu import _edge_case
    g = _edge_case(name, graphs)
    o = oracle.Oracle(g, mode=1, refine=True)
    o.optimization_run()
    coarse = o.comm()
    o.aggregation_run(True)
    _components_ok(g, o.best(), coarse)
    full = oracle.Oracle(g, mode=1, refine=True)
    full.louvain()
    assert np.unique(full.best()).size == full.n_best


def test_ring_of_cliques_keeps_cliques(oracle, graphs):
    """30 six-cliques in a ring: every final community is a union of whole cliques."""
    from test_refine_gpu import _edge_case
    g = _edge_case("ring_of_cliques", graphs)
    o = oracle.Oracle(g, mode=1, refine=True)
    o.louvain()
    b = o.best()
    for c in range(30):
        assert np.unique(b[6 * c:6 * c + 6]).size == 1
