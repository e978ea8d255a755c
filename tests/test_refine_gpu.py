"""Refinement (lv_config.refine = 1): the CUDA engine against the CPU oracle's restatement of
the same refined pipeline (oracle/louvain_oracle.c, refine_partition / orc_louvain), through
the C ABI.

Bit-exact with integer weights: final partitions, community counts, the per-pass trace
(level, pass, movers, I, S) and the number of refinement passes; modularity equal to 1e-12
(both sides evaluate the same exact I and S). Properties of the refined partition itself:
every refined community lies inside one community of the level's partition and is
connected. The configuration errors (server, resume) are checked too.
"""
import numpy as np
import pytest

from test_engine_gpu import Q_TOL, _pack

pytestmark = pytest.mark.gpu


def _trace_rows(tr):
    return [(int(r["level"]), int(r["iteration"]), int(r["n_moved"]), float(r["internal"]),
             float(r["sum_a2"])) for r in tr]


_ENGINE_ONLY = ("bin_max_degree",)


def _oracle_run(oracle, g, mode=1, **kw):
    kw = {k: v for k, v in kw.items() if k not in _ENGINE_ONLY}
    o = oracle.Oracle(g, mode=mode, refine=True, nthreads=0, **kw)
    o.louvain()
    return o


def _check_full(lv, oracle, g, mode=1, **kw):
    e = lv.Engine(0, mode=mode, refine=True, **kw)
    c = e.community(g)
    st = c.louvain()
    o = _oracle_run(oracle, g, mode, **kw)
    np.testing.assert_array_equal(c.best(), o.best())
    assert c.info().n_best == o.n_best
    assert abs(c.info().modularity - o.modularity) <= Q_TOL
    ot = o.trace()
    te = _trace_rows(c.trace())
    to = _trace_rows(ot)
    if c.info().weights_integer:
        assert te == to
    else:
        # fp32 weights: S is a double sum whose order differs (relative 1e-12, as Q)
        assert [r[:4] for r in te] == [r[:4] for r in to]
        np.testing.assert_allclose([r[4] for r in te], [r[4] for r in to], rtol=1e-12)
    assert st.refine_passes == o.refine_passes
    # the one-shot entry point gives the same result
    best, q, st2 = e.run_graph(g)
    np.testing.assert_array_equal(best, o.best())
    assert abs(q - o.modularity) <= Q_TOL
    assert st2.refine_passes == o.refine_passes and st2.graph_launches == 0
    c.close()
    e.close()
    return o


@pytest.mark.parametrize("mode", [1, 0, 2, 3])
def test_refine_fixture_all_modes(mode, lv, oracle, golden):
    o = _check_full(lv, oracle, golden.load_fixture(), mode)
    assert o.refine_passes > 0 and o.level >= 2


@pytest.mark.parametrize("seed", [1, 2])
def test_refine_rmat(seed, lv, oracle, graphs):
    _check_full(lv, oracle, graphs.rmat(14, 16, seed=seed))


def test_refine_chung_lu(lv, oracle, graphs):
    _check_full(lv, oracle, graphs.chung_lu_bounded(20000, 2.0, 1, 99, seed=4))


def test_refine_hub_kernels(lv, oracle, graphs):
    """Hubs beyond the shared-memory bins: the refinement passes run the global-table
    kernels on the restricted rows too."""
    g = graphs.rmat(16, 16, seed=7)
    assert g.degrees().max() > 8192
    _check_full(lv, oracle, g)


def test_refine_small_bins_and_pass_limit(lv, oracle, graphs):
    g = graphs.chung_lu_bounded(6000, 2.0, 1, 99, seed=8)
    _check_full(lv, oracle, g, bin_max_degree=[1, 2, 3, 4, 5, 6, 8, 0])
    _check_full(lv, oracle, g, refine_passes=1)
    _check_full(lv, oracle, g, refine_tolerance=0.5, threshold=1e-6)


def test_refine_weighted(lv, oracle, graphs):
    """fp32 weights: partitions agree exactly, S and Q to 1e-12 (double sums in another order)."""
    g = graphs.planted_partition(n=4000, n_comm=40, smin=20, smax=400, mean_degree=12, seed=2)
    assert g.w is not None and not np.all(np.floor(g.w) == g.w)
    _check_full(lv, oracle, g)


def test_refine_max_levels(lv, oracle, graphs):
    g = graphs.rmat(13, 16, seed=3)
    for ml in (1, 2, 3):
        o = _check_full(lv, oracle, g, max_levels=ml)
        assert o.level <= ml


def test_refine_batch_equals_single_runs(lv, oracle, graphs, golden):
    gs = [golden.load_fixture(), graphs.chung_lu_bounded(3000, 2.0, 1, 99, seed=11),
          graphs.rmat(10, 16, seed=2), graphs.chung_lu_mean(5000, 2.1, 8, seed=3),
          graphs.rmat(12, 8, seed=5)]
    offs, row, col, w = _pack(gs)
    e = lv.Engine(0, mode=1, refine=True)
    out, qs, ks, st = e.run_batch(offs, row, col, w)
    for i, g in enumerate(gs):
        o = _oracle_run(oracle, g)
        np.testing.assert_array_equal(out[offs[i]:offs[i + 1]], o.best(), err_msg=f"graph {i}")
        assert ks[i] == o.n_best
        assert abs(qs[i] - o.modularity) <= Q_TOL
    e.close()


def _components_ok(g, part, coarse):
    """Every class of `part` lies in one class of `coarse` and induces a connected subgraph."""
    import scipy.sparse as sp
    from scipy.sparse.csgraph import connected_components
    A = sp.csr_matrix((np.ones(g.col.size), g.col, g.row_ptr), shape=(g.n, g.n))
    order = np.argsort(part, kind="stable")
    bounds = np.searchsorted(part[order], np.arange(part.max() + 2))
    for c in range(part.max() + 1):
        idx = order[bounds[c]:bounds[c + 1]]
        if idx.size == 0:
            continue
        assert np.unique(coarse[idx]).size == 1
        if idx.size > 1:
            nc, _ = connected_components(A[idx][:, idx], directed=False)
            assert nc == 1


@pytest.mark.parametrize("which", ["fixture", "chung_lu"])
def test_refined_partition_nested_and_connected(which, lv, oracle, graphs, golden):
    """Phase-level run: after the first level's passes, aggregation with refinement maps each
    vertex to its refined community (the next level's vertex): nested in the level's
    partition, connected, and equal to the oracle's."""
    g = golden.load_fixture() if which == "fixture" else graphs.chung_lu_bounded(8000, 2.0, 1, 99, seed=6)
    e = lv.Engine(0, mode=1, refine=True)
    c = e.community(g)
    o = oracle.Oracle(g, mode=1, refine=True)
    c.optimization_run()
    o.optimization_run()
    coarse, _ = c.partition()
    np.testing.assert_array_equal(coarse, o.comm())
    c.aggregation_run(True)
    o.aggregation_run(True)
    ref = c.best()
    np.testing.assert_array_equal(ref, o.best())
    assert ref.max() + 1 < g.n and np.unique(ref).size == ref.max() + 1
    _components_ok(g, ref, coarse)
    # the contracted graph follows the refined partition
    row_e, col_e, w_e, k_e = c.graph()
    row_o, col_o, w_o = o.graph()
    np.testing.assert_array_equal(row_e, row_o)
    np.testing.assert_array_equal(col_e, col_o)
    np.testing.assert_array_equal(w_e, w_o)
    c.close()
    e.close()


def test_refine_configuration_errors(lv, graphs):
    e = lv.Engine(0, mode=1, refine=True)
    with pytest.raises(lv.LouvainError) as ex:
        lv.Server(e, budget_bytes=1 << 30, slots=2)
    assert ex.value.status == 1
    g = graphs.rmat(10, 8, seed=1)
    e2 = lv.Engine(0, mode=1)
    c = e2.community(g)
    c.optimization_run()
    c.aggregation_run(True)
    ck = c.checkpoint()
    with pytest.raises(lv.LouvainError) as ex:
        e.resume(ck)
    assert ex.value.status == 1
    # both contexts still work
    best, q, _ = e.run_graph(g)
    assert q > 0
    c.close()
    e.close()
    e2.close()


# ---- structured edge cases -------------------------------------------------------------------------
def _with_self_loops(g, every=7, weight=3.0):
    """Adds a self-loop entry of `weight` to every `every`-th vertex (kept sorted by column)."""
    import numpy as np
    from importlib import import_module
    CSRGraph = import_module("louvain-fast-move-cuda_b200.graphs").CSRGraph
    src = g.src()
    w = g.weights_or_ones.astype(np.float32)
    loops = np.arange(0, g.n, every)
    s2 = np.concatenate([src, loops])
    c2 = np.concatenate([g.col.astype(np.int64), loops])
    w2 = np.concatenate([w, np.full(loops.size, weight, dtype=np.float32)])
    order = np.lexsort((c2, s2))
    s2, c2, w2 = s2[order], c2[order], w2[order]
    row = np.zeros(g.n + 1, dtype=np.int64)
    np.cumsum(np.bincount(s2, minlength=g.n), out=row[1:])
    return CSRGraph(n=g.n, row_ptr=row, col=c2.astype(np.int32), w=w2, name=g.name + "_loops")


def _edge_case(name, graphs):
    rng = np.random.default_rng(3)
    if name == "stars":
        u = np.concatenate([np.zeros(200), np.full(150, 201), [0]])
        v = np.concatenate([np.arange(1, 201), np.arange(202, 352), [201]])
        return graphs.canonical_from_pairs(u, v, name="stars")
    if name == "ring_of_cliques":
        us, vs = [], []
        for c in range(30):
            b = 6 * c
            for i in range(6):
                for j in range(i + 1, 6):
                    us.append(b + i)
                    vs.append(b + j)
            us.append(b)
            vs.append((b + 6) % 180)
        return graphs.canonical_from_pairs(np.array(us), np.array(vs), name="ring_of_cliques")
    if name == "int_weights":
        g = graphs.chung_lu_bounded(5000, 2.0, 1, 99, seed=12)
        src = g.src()
        key = np.minimum(src, g.col) * 7919 + np.maximum(src, g.col)
        g.w = (key % 5 + 1).astype(np.float32)  # symmetric integer weights 1..5
        return g
    if name == "self_loops":
        return _with_self_loops(graphs.chung_lu_bounded(4000, 2.0, 1, 99, seed=13))
    if name == "components":
        a = graphs.rmat(10, 8, seed=4)
        b = _edge_case("ring_of_cliques", graphs)
        u = np.concatenate([a.src(), b.src() + a.n])
        v = np.concatenate([a.col, b.col + a.n])
        return graphs.canonical_from_pairs(u, v, name="components")
    raise KeyError(name)


EDGE_CASES = ["stars", "ring_of_cliques", "int_weights", "self_loops", "components"]


@pytest.mark.parametrize("name", EDGE_CASES)
def test_refine_edge_cases(name, lv, oracle, graphs):
    g = _edge_case(name, graphs)
    for mode in (1, 0):
        _check_full(lv, oracle, g, mode)


@pytest.mark.slow
def test_refine_rmat22_matches_oracle(lv, oracle, golden):
    """Full-size workload (R-MAT scale 22, 128.3 M entries, chunking active in the levels'
    passes): the refined run's partition, community count and modularity equal the oracle's."""
    g = golden.case_graph(golden.RMAT22)
    e = lv.Engine(0, mode=1, refine=True)
    best, q, st = e.run_graph(g)
    o = _oracle_run(oracle, g)
    np.testing.assert_array_equal(best, o.best())
    assert st.n_communities == o.n_best
    assert abs(q - o.modularity) <= Q_TOL
    assert st.refine_passes == o.refine_passes
    e.close()
