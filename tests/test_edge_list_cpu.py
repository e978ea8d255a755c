"""The CPU restatement of the reference's edge-list loader (oracle/edge_list.py): on the
reference's bundled fixture it gives the fixture's stored CSR, and a hand-worked input gives
the entries graph.cu:17-87 emits (self-loop pair twice, duplicates once, ids from min_id)."""
import numpy as np
import pytest

import edge_list as O


def test_loader_fixture(golden):
    g = golden.load_fixture()
    n, nl, mn, row, col = O.graph_host_csr(b"header\n" + g.edge_list_text().encode(), skip_line=1)
    assert (n, nl) == (g.n, g.m) and mn == 0
    assert np.array_equal(row, g.row_ptr) and np.array_equal(col, g.col)


def test_loader_hand_worked():
    # pairs: (5,6) twice in both orders, self-loop (7,7), (6,7); an unpaired "5" at the end
    n, nl, mn, row, col = O.graph_host_csr(b"5 6\n6 5\t7 7\r\n6 7 5")
    assert (n, nl, mn) == (3, 3, 5)
    # entries by (source, destination): 0-1, 1-0, 1-2, 2-1, 2-2, 2-2
    assert row.tolist() == [0, 1, 3, 6]
    assert col.tolist() == [1, 0, 2, 1, 2, 2]


def test_loader_stops_at_non_integer_and_errors():
    assert O.parse_tokens(b"1 2 3 x 4 5").tolist() == [1, 2]
    assert O.parse_tokens(b"1 2 +3 4 9999999999 1").tolist() == [1, 2, 3, 4]
    with pytest.raises(O.LoaderError):
        O.graph_host_csr(b"a b")
    with pytest.raises(O.LoaderError):
        O.graph_host_csr(b"0 1 1 3")
