"""Parity of the CUDA engine (through its C ABI) with the reference and with the oracle.

Bit-exact checks: partitions (communities per vertex), community counts, per-pass
partitions and community totals, contracted graphs (destinations and integer weights per
row), the internal weight I and the squared-total sum S of every pass. Modularity: equal to
1e-12 absolute (integer weights: both sides evaluate the same exact I and S; fp32 weights:
S is a double sum whose order differs, so 1e-12 is the stated tolerance).
"""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

SUMMARY = json.load(open(os.path.join(GOLDEN, "reference_summary.json")))
CASES = sorted(k for k, v in SUMMARY.items()
               if "n_best" in v and os.path.exists(os.path.join(GOLDEN, k + ".npz")))
Q_TOL = 1e-12


@pytest.fixture(scope="module")
def engines(lv):
    cache = {}

    def get(mode=1, **kw):
        key = (mode, tuple(sorted(kw.items())))
        if key not in cache:
            cache[key] = lv.Engine(0, mode=mode, **kw)
        return cache[key]

    yield get
    for e in cache.values():
        e.close()


# ---- against the reference's own outputs ---------------------------------------------------------
@pytest.mark.parametrize("key", CASES)
def test_engine_matches_reference_golden(key, golden, engines):
    rec = SUMMARY[key]
    g = golden.case_graph(rec["case"])
    mode = 1 if rec["mode"] == "SORT" else 0
    best, q, st = engines(mode).run_graph(g)
    z = np.load(os.path.join(GOLDEN, key + ".npz"))
    np.testing.assert_array_equal(best, z["best"])
    assert st.n_communities == rec["n_best"]
    assert abs(q - rec["modularity"]) <= Q_TOL


def _pass_records(tr):
    return [(int(r["level"]), int(r["iteration"]), float(r["internal"]), float(r["sum_a2"]))
            for r in tr]


@pytest.mark.parametrize("key", [k for k in CASES if k.startswith(("fixture", "rmat_s14", "chung_lu_10000_s1"))])
def test_engine_pass_trace_matches_reference_values(key, golden, lv, oracle):
    """Every (I, S) pair the reference printed after each pass equals the engine's."""
    rec = SUMMARY[key]
    g = golden.case_graph(rec["case"])
    mode = 1 if rec["mode"] == "SORT" else 0
    e = lv.Engine(0, mode=mode)
    c = e.community(g)
    c.louvain()
    tr = c.trace()
    o = oracle.Oracle(g, mode=mode)
    o.louvain()
    ot = o.trace()
    assert len(tr) == len(ot)
    for a, b in zip(_pass_records(tr), [(int(r["level"]), int(r["iteration"]), r["internal"], r["sum_a2"]) for r in ot]):
        assert a == b
    np.testing.assert_array_equal(c.best(), np.load(os.path.join(GOLDEN, key + ".npz"))["best"])


# ---- pass-by-pass against the oracle ---------------------------------------------------------------
def _lockstep(lv, oracle, g, mode, thr=1e-3, chunk_edges=50_000_000, fast_first=True):
    e = lv.Engine(0, mode=mode, threshold=thr, chunk_edges=chunk_edges, fast_first=fast_first)
    c = e.community(g)
    o = oracle.Oracle(g, mode=mode, threshold=thr, chunk_edges=chunk_edges, fast_first=fast_first)
    levels = 0
    while True:
        q_level = o.modularity
        assert abs(c.info().modularity - q_level) <= Q_TOL
        while True:
            mo, do = o.optimization_step()
            me, de = c.optimization_step()
            comm_e, tot_e = c.partition()
            np.testing.assert_array_equal(comm_e, o.comm())
            np.testing.assert_array_equal(tot_e, o.totals())
            inf = c.info()
            assert me == mo
            assert inf.internal == o.internal
            if inf.weights_integer:
                assert inf.sum_a2 == o.sum_a2
            assert abs(inf.modularity - o.modularity) <= Q_TOL
            if not (do > thr):
                break
        cont = (o.modularity - q_level) > thr
        o.aggregation_run(cont)
        c.aggregation_run(cont)
        levels += 1
        np.testing.assert_array_equal(c.best(), o.best())
        if not cont:
            break
        row_e, col_e, w_e, k_e = c.graph()
        row_o, col_o, w_o = o.graph()
        np.testing.assert_array_equal(row_e, row_o)
        np.testing.assert_array_equal(col_e, col_o)
        np.testing.assert_array_equal(w_e, w_o)
        np.testing.assert_array_equal(k_e, o.k())
    return levels


@pytest.mark.parametrize("mode", [1, 0, 2, 3])
def test_lockstep_fixture_all_modes(mode, lv, oracle, golden):
    g = golden.load_fixture()
    assert _lockstep(lv, oracle, g, mode) >= 2


@pytest.mark.parametrize("seed", [1, 2])
def test_lockstep_rmat(seed, lv, oracle, graphs):
    g = graphs.rmat(13, 16, seed=seed)
    _lockstep(lv, oracle, g, 1)
    _lockstep(lv, oracle, g, 0)


def test_lockstep_chunk_early_return(lv, oracle, graphs):
    """STEP_ROUND emulation at a small chunk size: passes end at the first empty chunk."""
    g = graphs.rmat(12, 16, seed=3)
    for chunk in (3000, 20000):
        _lockstep(lv, oracle, g, 1, chunk_edges=chunk)
        _lockstep(lv, oracle, g, 0, chunk_edges=chunk)


def test_lockstep_threshold_1e6(lv, oracle, graphs):
    g = graphs.chung_lu_bounded(10000, 2.0, 1, 99, seed=4)
    _lockstep(lv, oracle, g, 1, thr=1e-6)


def test_lockstep_no_fast_pass(lv, oracle, graphs):
    g = graphs.chung_lu_bounded(5000, 2.0, 1, 99, seed=5)
    _lockstep(lv, oracle, g, 1, fast_first=False)


def test_lockstep_weighted(lv, oracle, graphs):
    """fp32 weights (no reference counterpart): double sums, one fp32 rounding per
    contracted weight; exact here because the weight range keeps every sum exact."""
    g = graphs.planted_partition(n=4000, n_comm=40, smin=20, smax=400, mean_degree=12, seed=2)
    assert g.w is not None and not np.all(np.floor(g.w) == g.w)
    _lockstep(lv, oracle, g, 1)


def test_hub_bins_and_global_tables(lv, oracle, graphs):
    """A graph whose hubs exceed the shared-memory bins (degree > 8192) so the global
    hash-table arena and block-per-vertex kernels run, in every pass and the contraction."""
    g = graphs.rmat(16, 16, seed=7)
    assert g.degrees().max() > 8192
    _lockstep(lv, oracle, g, 1)


def test_small_bins_forced(lv, oracle, graphs):
    """Tiny bin thresholds push most vertices into block and global-table kernels."""
    g = graphs.chung_lu_bounded(6000, 2.0, 1, 99, seed=8)
    e = lv.Engine(0, mode=1, bin_max_degree=[1, 2, 3, 4, 5, 6, 8, 0])
    best, q, st = e.run_graph(g)
    o = oracle.Oracle(g, mode=1)
    o.louvain()
    np.testing.assert_array_equal(best, o.best())


# ---- larger graphs -------------------------------------------------------------------------------
def test_rmat18_matches_oracle(lv, oracle, graphs, engines):
    g = graphs.rmat(18, 16, seed=1)
    for mode in (1, 0):
        best, q, st = engines(mode).run_graph(g)
        o = oracle.Oracle(g, mode=mode, nthreads=0)
        o.louvain()
        np.testing.assert_array_equal(best, o.best())
        assert abs(q - o.modularity) <= Q_TOL


@pytest.mark.slow
def test_rmat22_matches_reference(lv, graphs, golden, engines):
    """Full-size workload (R-MAT scale 22, 128.3M entries, chunking active): the engine's
    partition hash, community count and modularity equal the reference's own run."""
    g = golden.case_graph(golden.RMAT22)
    assert golden.graph_digest(g) == SUMMARY["rmat_s22_ef16__SORT"]["digest"]
    for mode in ("SORT", "HASH"):
        rec = SUMMARY[f"rmat_s22_ef16__{mode}"]
        best, q, st = engines(1 if mode == "SORT" else 0).run_graph(g)
        assert hashlib.sha256(best.astype(np.int32).tobytes()).hexdigest()[:16] == rec["best_sha"]
        assert st.n_communities == rec["n_best"]
        assert abs(q - rec["modularity"]) <= Q_TOL


# ---- batch -------------------------------------------------------------------------------------------
def _pack(gs):
    offs = [0]
    rows = [np.zeros(1, dtype=np.int64)]
    cols, ws = [], []
    eoff = 0
    for g in gs:
        rows.append(g.row_ptr[1:] + eoff)
        cols.append(g.col.astype(np.int64) + offs[-1])
        ws.append(g.weights_or_ones)
        eoff += g.E
        offs.append(offs[-1] + g.n)
    return (np.array(offs, dtype=np.int64), np.concatenate(rows), np.concatenate(cols).astype(np.int32),
            np.concatenate(ws).astype(np.float32))


def test_batch_equals_single_runs(lv, oracle, graphs, golden, engines):
    gs = [golden.load_fixture(), graphs.chung_lu_bounded(3000, 2.0, 1, 99, seed=11),
          graphs.rmat(10, 16, seed=2), graphs.chung_lu_mean(5000, 2.1, 8, seed=3),
          golden.case_graph(golden.CASES[-1]), graphs.rmat(12, 8, seed=5)]
    offs, row, col, w = _pack(gs)
    for mode in (1, 0):
        out, qs, ks, st = engines(mode).run_batch(offs, row, col, w)
        for i, g in enumerate(gs):
            o = oracle.Oracle(g, mode=mode)
            o.louvain()
            np.testing.assert_array_equal(out[offs[i]:offs[i + 1]], o.best(), err_msg=f"graph {i}")
            assert ks[i] == o.n_best
            assert abs(qs[i] - o.modularity) <= Q_TOL


def test_batch_many_small(lv, oracle, graphs, engines):
    rng = np.random.default_rng(5)
    gs = [graphs.chung_lu_mean(int(n), 2.1, 8, seed=int(s))
          for n, s in zip(np.exp(rng.uniform(np.log(200), np.log(3000), 64)).astype(int), range(64))]
    offs, row, col, w = _pack(gs)
    out, qs, ks, st = engines(1).run_batch(offs, row, col, w)
    for i in range(0, 64, 7):
        o = oracle.Oracle(gs[i], mode=1)
        o.louvain()
        np.testing.assert_array_equal(out[offs[i]:offs[i + 1]], o.best())
        assert abs(qs[i] - o.modularity) <= Q_TOL


# ---- API behaviour -------------------------------------------------------------------------------------
def test_device_buffers_and_determinism(lv, graphs, engines):
    import torch
    g = graphs.rmat(14, 16, seed=9)
    e = engines(1)
    best_h, q_h, _ = e.run_graph(g)
    row = torch.from_numpy(g.row_ptr).cuda()
    col = torch.from_numpy(g.col).cuda()
    out = torch.empty(g.n, dtype=torch.int32, device="cuda")
    _, q_d, _ = e.run_csr(g.n, row, col, None, out=out)
    np.testing.assert_array_equal(out.cpu().numpy(), best_h)
    assert q_d == q_h
    for _ in range(2):
        b2, q2, _ = e.run_graph(g)
        np.testing.assert_array_equal(b2, best_h)
        assert q2 == q_h


def test_reference_facade(lv, golden):
    g = lv.GraphHost.from_csr(golden.load_fixture())
    C = lv.ModularityAlgorithms.Louvain(g, lv.MODE.SORT)
    rec = SUMMARY["fixture_power_law_10000__SORT"]
    assert C.n_of_best_communities == rec["n_best"]
    assert abs(C.modularity - rec["modularity"]) <= Q_TOL


@pytest.mark.parametrize("bad", ["col_range", "empty_row", "zero_weight", "fraction_int", "negative_row"])
def test_invalid_input_rejected_and_context_survives(bad, lv, graphs):
    g = graphs.chung_lu_bounded(500, 2.0, 1, 20, seed=1)
    row, col = g.row_ptr.copy(), g.col.copy()
    w = None
    kw = {}
    if bad == "col_range":
        col[5] = g.n + 3
    elif bad == "empty_row":
        row = np.concatenate([row[:3], [row[3]], row[3:]])  # vertex 3 gets no entries
        col = col.copy()
    elif bad == "zero_weight":
        w = np.ones(g.E, dtype=np.float32)
        w[7] = 0.0
    elif bad == "fraction_int":
        w = np.ones(g.E, dtype=np.float32)
        w[7] = 1.5
        kw = {"weight_mode": lv.WEIGHTS_INTEGER}
    elif bad == "negative_row":
        row = row.copy()
        row[4] = -1
    e = lv.Engine(0, **kw)
    n = row.size - 1
    with pytest.raises(lv.LouvainError) as ei:
        e.run_csr(n, row, col, w)
    assert ei.value.status in (1, 2)
    best, q, st = e.run_graph(g)  # the context still works
    assert st.n_communities > 0
