"""CPU restatement of the reference's edge-list loader -- test infrastructure only.

GraphHost(name, weighted = false, skip_line) (graph.cu:17-87) with GraphDevice's ordering
(graph.cuh:60-91), as the symmetric CSR the engine's lv_ingest_* builds on the GPU:

* `skip_line` lines are dropped (std::getline, graph.cu:21-24);
* the rest is read as integers two at a time (`while (f >> a >> b)`, graph.cu:35) until the
  first token that is not an integer; an unpaired last token is dropped;
* distinct unordered pairs (min, max) are the edges (graph.cu:38-43), self-loop pairs included;
  the distinct ids are the nodes (graph.cu:36-37), min_id the smallest (graph.cu:82);
* every edge is emitted in both directions with weight 1 (graph.cu:68-79), so a self-loop pair
  gives two (u, u) entries; GraphDevice renumbers by id - min_id (graph.cuh:66-85), which needs
  contiguous ids, and sorts entries by (source, destination) (graph.cuh:60).

A token is an optional sign and decimal digits in int32 range. (A token such as "12abc" ends the
input before it; iostream would still read its leading digits.)
"""
from __future__ import annotations

import re

import numpy as np

_INT = re.compile(rb"^[+-]?[0-9]+$")


class LoaderError(ValueError):
    pass


def parse_tokens(text: bytes, skip_line: int = 0) -> np.ndarray:
    """The integers the reference's loop reads, in order (an even count)."""
    pos = 0
    for _ in range(skip_line):
        nl = text.find(b"\n", pos)
        if nl < 0:
            pos = len(text)
            break
        pos = nl + 1
    vals = []
    for tok in text[pos:].split():
        if not _INT.match(tok):
            break
        v = int(tok)
        if v < -2**31 or v > 2**31 - 1:
            break
        vals.append(v)
    vals = vals[: len(vals) // 2 * 2]
    return np.array(vals, dtype=np.int64)


def graph_host_csr(text: bytes, skip_line: int = 0):
    """(n_nodes, n_links, min_id, row_ptr int64[n+1], col int32[2 n_links])."""
    vals = parse_tokens(text, skip_line)
    if vals.size == 0:
        raise LoaderError("Error during parsing: no node found")  # graph.cu:52-55
    a, b = vals[0::2], vals[1::2]
    lo, hi = np.minimum(a, b), np.maximum(a, b)
    ids = np.unique(vals)
    min_id = int(ids[0])
    if ids[-1] - ids[0] + 1 != ids.size:
        raise LoaderError("vertex IDs are not contiguous")
    pairs = np.unique(np.stack([lo - min_id, hi - min_id], axis=1), axis=0)
    src = np.concatenate([pairs[:, 0], pairs[:, 1]])
    dst = np.concatenate([pairs[:, 1], pairs[:, 0]])
    order = np.lexsort((dst, src))
    src, dst = src[order], dst[order]
    n = int(ids.size)
    row_ptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(src, minlength=n), out=row_ptr[1:])
    return n, int(pairs.shape[0]), min_id, row_ptr, dst.astype(np.int32)
