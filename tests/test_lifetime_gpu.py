"""Object lifetimes of the Python binding: an Engine closed (or collected) before the objects
made on it -- phase-level communities, ingested graphs, servers -- closes them first, so no
call reaches a destroyed context; closing them again afterwards is a no-op, and a fresh
engine works."""
import gc

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_engine_closes_dependants_first(lv, graphs):
    g = graphs.rmat(11, 8, seed=3)
    e = lv.Engine(0, mode=1)
    c = e.community(g)
    c.optimization_run()
    ing = e.ingest(b"0 1\n1 2\n2 0\n")
    srv = lv.Server(e, budget_bytes=1 << 30, slots=2)
    e.close()
    for obj in (c, ing, srv):
        assert obj._h is None
        obj.close()  # no-op
    e.close()
    e2 = lv.Engine(0, mode=1)
    best, q, _ = e2.run_graph(g)
    assert q > 0 and best.size == g.n
    e2.close()


def test_collection_in_any_order(lv, graphs):
    g = graphs.rmat(10, 8, seed=4)
    for drop_engine_first in (True, False):
        e = lv.Engine(0, mode=1)
        c = e.community(g)
        c.louvain()
        ref = c.best().copy()
        if drop_engine_first:
            e.close()
            del e
            gc.collect()
            del c
        else:
            del c
            gc.collect()
            e.close()
            del e
        gc.collect()
    e = lv.Engine(0, mode=1)
    c = e.community(g)
    c.louvain()
    np.testing.assert_array_equal(c.best(), ref)
    e.close()
