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


def _independent_loader(text: bytes, skip_line: int):
    """A second statement of graph.cu:17-87 for the fuzz test: drop `skip_line` lines, read
    whitespace-separated integers two at a time up to the first other token, keep distinct
    unordered pairs, emit each in both directions, renumber from the smallest id."""
    lines = text.split(b"\n")
    rest = b"\n".join(lines[skip_line:]) if skip_line < len(lines) else b""
    vals = []
    for tok in rest.split():
        t = tok[1:] if tok[:1] in (b"+", b"-") else tok
        if not t.isdigit():
            break
        x = int(tok)
        if not -2**31 <= x < 2**31:
            break
        vals.append(x)
    vals = vals[: len(vals) // 2 * 2]
    if not vals:
        return None
    pairs = {(min(a, b), max(a, b)) for a, b in zip(vals[0::2], vals[1::2])}
    ids = sorted(set(vals))
    if ids[-1] - ids[0] + 1 != len(ids):
        return None
    mn = ids[0]
    ent = sorted([(a - mn, b - mn) for a, b in pairs] + [(b - mn, a - mn) for a, b in pairs])
    n = len(ids)
    row = [0] * (n + 1)
    for s, _ in ent:
        row[s + 1] += 1
    for i in range(n):
        row[i + 1] += row[i]
    return n, len(pairs), mn, row, [d for _, d in ent]


def test_loader_fuzz_against_independent_statement():
    hyp = pytest.importorskip("hypothesis")
    st = hyp.strategies
    seps = st.sampled_from([b" ", b"\t", b"\n", b"\r\n", b"  ", b" \n"])

    @hyp.settings(max_examples=200, deadline=None, derandomize=True)
    @hyp.given(base=st.integers(-50, 50), span=st.integers(1, 12),
               pairs=st.lists(st.tuples(st.integers(0, 11), st.integers(0, 11)), min_size=1, max_size=40),
               sep=seps, header=st.integers(0, 2), tail=st.sampled_from([b"", b" 7", b" x 3 4", b" +2 -1"]))
    def check(base, span, pairs, sep, header, tail):
        toks = []
        for a, b in pairs:
            toks += [str(base + a % span).encode(), str(base + b % span).encode()]
        text = b"# h\n" * header + sep.join(toks) + tail
        want = _independent_loader(text, header)
        if want is None:
            with pytest.raises(O.LoaderError):
                O.graph_host_csr(text, header)
            return
        n, nl, mn, row, col = O.graph_host_csr(text, header)
        assert (n, nl, mn) == want[:3]
        assert row.tolist() == want[3] and col.tolist() == want[4]

    check()
