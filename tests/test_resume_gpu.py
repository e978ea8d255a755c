"""Checkpoint / resume at a level start (lv_community_resume): a run stopped after its first
(or second) level, exported through the getters and resumed in a fresh context, finishes with
the same final partition, community count and modularity as the uninterrupted run, and the
passes it runs after the resume produce the same trace records (integer weights: bit-exact).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cases(graphs, golden):
    return {"fixture": golden.load_fixture(), "rmat16": graphs.rmat(16, 16, seed=1),
            "chung_lu_40000": graphs.chung_lu_mean(40000, seed=7)}


@pytest.mark.parametrize("key", ["fixture", "rmat16", "chung_lu_40000"])
@pytest.mark.parametrize("stop_after", [1, 2])
def test_resume_equals_uninterrupted(key, stop_after, cases, lv):
    g = cases[key]
    e = lv.Engine(0)
    full = e.community(g)
    full.louvain()
    best_full, trace_full, q_full = full.best(), full.trace(), full.info().modularity
    levels_full = int(trace_full["level"].max()) + 1
    if levels_full <= stop_after:
        pytest.skip(f"{key} has only {levels_full} levels")
    part = e.community(g)
    for _ in range(stop_after):
        part.optimization_run()
        part.aggregation_run(True)
    ck = part.checkpoint()
    done = len(part.trace())
    part.close()
    assert ck["level"] == stop_after and ck["iterations"] == done

    e2 = lv.Engine(0)
    r = e2.resume(ck)
    r.louvain()
    assert np.array_equal(r.best(), best_full)
    assert r.info().modularity == q_full
    assert np.array_equal(r.trace(), trace_full[done:])
    r.close()
    full.close()
    e.close()
    e2.close()


def test_resume_rejects_bad_checkpoint(cases, lv):
    g = cases["fixture"]
    e = lv.Engine(0)
    c = e.community(g)
    c.optimization_run()
    c.aggregation_run(True)
    ck = c.checkpoint()
    bad = dict(ck, best=np.full_like(ck["best"], ck["row_ptr"].size + 5))
    with pytest.raises(lv.LouvainError) as ex:
        e.resume(bad)
    assert ex.value.status == 2
    frac = dict(ck, w=ck["w"] + 0.5)
    with pytest.raises(lv.LouvainError):
        e.resume(frac)
    # the context still works
    e.resume(ck).close()
    c.close()
    e.close()
