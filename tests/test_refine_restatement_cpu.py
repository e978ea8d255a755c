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
