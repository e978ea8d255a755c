"""The serving loop (lv_server_*): each request's result is the same alone and in the mix.

Requests of uneven sizes are submitted together to a server with several slots, so they are
admitted while others run and overlap on the device; every result must equal the same graph
run alone through lv_run_csr: communities bit-exact and modularity bit-identical (integer
weights: the totals, I and S are exact integers, so the tolerance is 0). A weighted request
(fp32 weights) is held to the engine's stated 1e-12 modularity tolerance, communities exact.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BIG = 64 << 30


@pytest.fixture(scope="module")
def mix(graphs, golden):
    gs = [golden.load_fixture()]
    gs += [graphs.rmat(s, 8, seed=s) for s in (9, 12, 14, 16)]
    gs += [graphs.chung_lu_mean(n, seed=n) for n in (300, 5000, 40000)]
    gs += [graphs.planted_partition(20000, 40, seed=5)]
    return gs


@pytest.fixture(scope="module")
def alone(lv, mix):
    e = lv.Engine(0)
    res = [e.run_graph(g)[:2] for g in mix]
    e.close()
    return res


def _check(results, alone, mix):
    for i, (g, (comm, q, lat)) in enumerate(zip(mix, results)):
        ref_comm, ref_q = alone[i]
        assert np.array_equal(comm, ref_comm), f"request {i} ({g.name}) partition differs"
        tol = 0.0 if g.w is None else 1e-12
        assert abs(q - ref_q) <= tol, (i, g.name, q, ref_q)
        assert lat >= 0.0


def _collect(srv, ids):
    srv.drain()
    out = [srv.poll(r) for r in ids]
    assert all(o is not None for o in out)
    return out


def test_server_mix_equals_alone(lv, mix, alone):
    e = lv.Engine(0)
    srv = lv.Server(e, BIG, slots=4)
    # every graph twice, interleaved, so requests overlap with copies of themselves and others
    order = list(range(len(mix))) * 2
    ids = [srv.submit(mix[i]) for i in order]
    out = _collect(srv, ids)
    _check(out, [alone[i] for i in order], [mix[i] for i in order])
    assert srv.progress() == (len(order), 0, 0)
    srv.close()
    e.close()


def test_server_budget_admits_one_at_a_time(lv, mix, alone):
    # a budget that fits the largest request but never two of them: admission serialises
    e = lv.Engine(0)
    biggest = max(g.E * 16 + g.n * 124 for g in mix) + (2 << 20)
    srv = lv.Server(e, biggest + biggest // 2, slots=8)
    ids = [srv.submit(g) for g in mix]
    out = _collect(srv, ids)
    _check(out, alone, mix)
    srv.close()
    e.close()


def test_server_rejects_request_over_budget(lv, mix):
    e = lv.Engine(0)
    srv = lv.Server(e, 1 << 20, slots=2)
    with pytest.raises(lv.LouvainError) as ex:
        srv.submit(mix[4])
    assert ex.value.status == 7  # LV_ERR_BUDGET
    srv.close()
    e.close()


def test_server_poll_before_done_and_unknown_id(lv, mix):
    e = lv.Engine(0)
    srv = lv.Server(e, BIG, slots=1)
    ids = [srv.submit(g) for g in mix[:3]]
    first = srv.poll(ids[-1])  # the last of three on one slot is normally still queued
    srv.drain()
    res = [srv.poll(r) for r in (ids if first is None else ids[:-1])]
    assert all(r is not None for r in res)
    with pytest.raises(lv.LouvainError):
        srv.poll(ids[0])  # already collected
    srv.close()
    e.close()
