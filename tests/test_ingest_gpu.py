"""GPU edge-list ingest (lv_ingest_*) against the CPU restatement of the reference's loader
(oracle/edge_list.py, graph.cu:17-87): node and link counts, min_id and the CSR bit-exact, on
the reference's own fixture written as text and on inputs with every case the loader handles
(duplicate pairs in both orders, self-loops, tabs, CRLF, several pairs per line, header lines,
negative and offset ids, an unpaired last token, a non-integer token ending the input), plus
the two errors (no pair, ids not contiguous). A Louvain run on the ingested graph equals the
run on the same CSR uploaded from the host.
"""
import numpy as np
import pytest

import edge_list as O

pytestmark = pytest.mark.gpu


def _check(lv, engine, text, skip_line=0):
    n, nl, mn, row, col = O.graph_host_csr(text, skip_line)
    g = engine.ingest(text, skip_line)
    assert (g.n_nodes, g.n_links, g.min_id, g.entries) == (n, nl, mn, 2 * nl)
    csr = g.csr()
    assert np.array_equal(csr.row_ptr, row)
    assert np.array_equal(csr.col, col)
    return g, csr


@pytest.fixture(scope="module")
def engine(lv):
    e = lv.Engine(0)
    yield e
    e.close()


def test_ingest_fixture_text(lv, engine, golden):
    g0 = golden.load_fixture()
    text = b"% header line\n" + g0.edge_list_text().encode()
    g, csr = _check(lv, engine, text, skip_line=1)
    # no self-loops in the fixture: the same graph the host parser gives
    assert np.array_equal(csr.row_ptr, g0.row_ptr) and np.array_equal(csr.col, g0.col)
    comm, q, st = g.run()
    c2, q2, _ = engine.run_graph(csr)
    assert np.array_equal(comm, c2) and q == q2
    g.close()


def test_ingest_corner_cases(lv, engine):
    text = (b"# two header lines\n# second\n"
            b"1000 1001\n1001 1000\r\n1002\t1000 1003 1003\n"   # duplicate, CRLF, tab, self-loop
            b"  1004 1001   1002 1004\n1004 1002\n"             # several pairs per line, duplicate
            b"1005 1000 1003")                                  # unpaired last token
    g, csr = _check(lv, engine, text, skip_line=2)
    assert g.min_id == 1000 and g.n_nodes == 6
    g.close()
    # negative ids, and a non-integer token ending the input before an out-of-range id
    text = b"-3 -2\n-2 -1\n-1 -3\n0 -3\nend 99999 5\n"
    g, _ = _check(lv, engine, text)
    assert g.min_id == -3 and g.n_nodes == 4 and g.n_links == 4
    g.close()


def test_ingest_rmat_raw_pairs(lv, engine, graphs):
    u, v = graphs.rmat_pairs(12, 8, seed=4)   # raw: duplicates and self-loops included
    ids = np.unique(np.concatenate([u, v]))
    remap = np.searchsorted(ids, np.concatenate([u, v]))  # contiguous ids
    a, b = remap[: u.size], remap[u.size:]
    text = "\n".join(f"{x} {y}" for x, y in zip(a.tolist(), b.tolist())).encode()
    g, _ = _check(lv, engine, text)
    g.close()


def test_ingest_errors(lv, engine):
    with pytest.raises(lv.LouvainError) as ex:
        engine.ingest(b"x y\n")
    assert ex.value.status == 2
    with pytest.raises(lv.LouvainError) as ex:
        engine.ingest(b"0 1\n1 5\n")   # ids 0, 1, 5: not contiguous
    assert ex.value.status == 2
    # the context still works
    g, _ = _check(lv, engine, b"0 1\n1 2\n")
    g.close()


def test_ingest_every_row_class(lv, engine):
    """Rows of every size class the device sort treats differently (one entry per lane, eight
    and 32 per lane, a block, a bitmap over the row's id range), each with duplicate pairs in
    both orders and, for some hubs, the hub's own self-loop pair (kept twice in its row)."""
    rng = np.random.default_rng(7)
    n = 20000
    pairs = [np.stack([np.arange(n - 1), np.arange(1, n)], 1)]  # a path keeps the ids contiguous
    for hub, deg, loop in ((10, 20, False), (11, 200, True), (12, 900, False), (13, 3000, True),
                           (14, 9000, True), (15, 15000, False)):
        nb = rng.choice(n, size=deg, replace=False)
        pairs.append(np.stack([np.full(deg, hub), nb], 1))
        dup = nb[: deg // 3]
        pairs.append(np.stack([dup, np.full(dup.size, hub)], 1))  # the same pairs reversed
        if loop:
            pairs.append(np.array([[hub, hub], [hub, hub]]))
    p = np.concatenate(pairs)
    p = p[rng.permutation(len(p))]
    text = "\n".join(f"{a} {b}" for a, b in p.tolist()).encode()
    g, csr = _check(lv, engine, text)
    deg = np.diff(csr.row_ptr)
    assert deg.max() > 4096 and ((deg > 1024) & (deg <= 4096)).any() and ((deg > 256) & (deg <= 1024)).any()
    g.close()


def test_ingest_rmat16_raw_pairs(lv, engine, graphs):
    """Raw R-MAT pairs at scale 16 (1 M pairs with duplicates and self-loops): hub rows far above
    4,096 entries, as in the benchmark's scale-22 input."""
    u, v = graphs.rmat_pairs(16, 16, seed=2)
    ids = np.unique(np.concatenate([u, v]))
    remap = np.searchsorted(ids, np.concatenate([u, v]))
    a, b = remap[: u.size], remap[u.size:]
    text = graphs.edge_list_bytes(a, b)
    g, csr = _check(lv, engine, text)
    assert np.diff(csr.row_ptr).max() > 4096
    g.close()
