"""lv_autotune: picks one of its candidate degree-bin tables by timing full runs of a sample,
installs it in the context, and never changes results (integer weights: every table computes
the same exact sums, so partitions and modularity are bit-identical to the built-in table's).
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CANDIDATES = {
    (4, 8, 16, 32, 128, 512, 4096), (4, 8, 16, 32, 128, 512, 8192), (4, 8, 16, 32, 128, 512, 2048),
    (8, 16, 32, 64, 128, 512, 4096), (2, 4, 8, 16, 64, 512, 4096), (4, 8, 16, 32, 64, 256, 4096),
    (4, 8, 16, 32, 128, 1024, 4096), (8, 16, 32, 64, 256, 1024, 4096), (8, 16, 32, 64, 128, 512, 2048),
}


def test_autotune_batch_sample_then_full_batch(lv, graphs):
    batch = importlib.import_module("louvain-fast-move-cuda_b200.batch")
    gs = [graphs.chung_lu_mean(n, seed=n) for n in (300, 2000, 9000, 500, 30000, 1200)]
    gs += [graphs.rmat(s, 8, seed=s) for s in (10, 13)]
    offs, row, col, w = batch.pack(gs)
    plain = lv.Engine(0)
    ref = plain.run_batch(offs, row, col)
    tuned = lv.Engine(0)
    sample = batch.pack(gs[::2])
    bins, ms = tuned.autotune(sample[0], sample[1], sample[2], trials=2)
    assert tuple(bins[:7]) in CANDIDATES and bins[7] == 0 and ms > 0
    got = tuned.run_batch(offs, row, col)
    assert np.array_equal(ref[0], got[0])
    assert np.array_equal(ref[1], got[1]) and np.array_equal(ref[2], got[2])
    plain.close()
    tuned.close()


def test_autotune_single_graph(lv, graphs):
    g = graphs.rmat(15, 16, seed=2)
    plain = lv.Engine(0)
    c0, q0, _ = plain.run_graph(g)
    tuned = lv.Engine(0)
    bins, ms = tuned.autotune(np.array([0, g.n], dtype=np.int64), g.row_ptr, g.col, trials=1)
    assert tuple(bins[:7]) in CANDIDATES
    c1, q1, _ = tuned.run_graph(g)
    assert np.array_equal(c0, c1) and q0 == q1
    plain.close()
    tuned.close()


def test_autotune_rejects_bad_arguments(lv, graphs):
    g = graphs.rmat(8, 8, seed=1)
    e = lv.Engine(0)
    with pytest.raises(lv.LouvainError):
        e.autotune(np.array([0, g.n], dtype=np.int64), g.row_ptr, g.col, trials=0)
    # the context still runs afterwards
    e.run_graph(g)
    e.close()
