"""Batched graphs: packing into one CSR, and dealing independent graphs across GPUs.

A batch is many independent graphs packed into one CSR (vertex ranges given by an offset
table, column IDs global), which lv_run_batch processes in one device-driven sequence. Across
GPUs the graphs need no exchange at all: they are dealt to ranks by edge count (longest
processing time first onto the least-loaded rank), each rank runs its share as one batch, and
the per-graph results are gathered on the host. The reference has no batching and no
multi-GPU code (one graph per ModularityAlgorithms::Louvain call, main.cu:19-39).
"""
from __future__ import annotations

import heapq
from typing import Callable, List, Sequence, Tuple

import numpy as np


def pack(graphs: Sequence) -> Tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
    """Pack CSRGraphs into (vtx_offsets int64[G+1], row_ptr int64[N+1], col int32[E],
    w float32[E]) with global vertex IDs."""
    G = len(graphs)
    offs = np.zeros(G + 1, dtype=np.int64)
    eoffs = np.zeros(G + 1, dtype=np.int64)
    for i, g in enumerate(graphs):
        offs[i + 1] = offs[i] + g.n
        eoffs[i + 1] = eoffs[i] + g.E
    row = np.empty(int(offs[-1]) + 1, dtype=np.int64)
    col = np.empty(int(eoffs[-1]), dtype=np.int32)
    w = np.empty(int(eoffs[-1]), dtype=np.float32)
    row[0] = 0
    for i, g in enumerate(graphs):
        row[offs[i] + 1: offs[i + 1] + 1] = g.row_ptr[1:] + eoffs[i]
        col[eoffs[i]: eoffs[i + 1]] = g.col + offs[i]
        w[eoffs[i]: eoffs[i + 1]] = g.weights_or_ones
    return offs, row, col, w


def unpack(values: np.ndarray, offs: np.ndarray) -> List[np.ndarray]:
    return [values[offs[i]: offs[i + 1]] for i in range(len(offs) - 1)]


def deal(edge_counts: Sequence[int], world: int) -> List[List[int]]:
    """Greedy longest-processing-time assignment of graphs to `world` ranks by edge count.
    Deterministic: ties go to the lowest rank, graphs of equal size in index order."""
    if world <= 0:
        raise ValueError("world must be positive")
    order = sorted(range(len(edge_counts)), key=lambda i: (-int(edge_counts[i]), i))
    heap = [(0, r) for r in range(world)]
    shares: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shares[r].append(i)
        heapq.heappush(heap, (load + int(edge_counts[i]), r))
    for s in shares:
        s.sort()
    return shares


def run_sharded(graphs: Sequence, run_batch: Callable, rank: int, world: int, group=None):
    """Run this rank's share of `graphs` with `run_batch(list_of_graphs) -> (labels_list,
    modularities, n_communities)` and gather every graph's result on every rank (host-side,
    torch.distributed object collectives; nothing crosses a GPU link). Returns
    (labels per graph, modularity per graph, communities per graph) in input order."""
    shares = deal([g.E for g in graphs], world)
    mine = shares[rank]
    if mine:
        labels, qs, ks = run_batch([graphs[i] for i in mine])
        local = [(i, np.asarray(labels[j]), float(qs[j]), int(ks[j])) for j, i in enumerate(mine)]
    else:
        local = []
    if world > 1:
        import torch.distributed as dist
        gathered = [None] * world
        dist.all_gather_object(gathered, local, group=group)
    else:
        gathered = [local]
    out_l = [None] * len(graphs)
    out_q = np.zeros(len(graphs))
    out_k = np.zeros(len(graphs), dtype=np.int64)
    for part in gathered:
        for i, lab, q, k in part:
            out_l[i], out_q[i], out_k[i] = lab, q, k
    return out_l, out_q, out_k


def engine_runner(engine) -> Callable:
    """A run_batch callable for run_sharded backed by an Engine (lv_run_batch)."""
    def run(gs):
        offs, row, col, w = pack(gs)
        weighted = any(g.w is not None for g in gs)
        out, qs, ks, _ = engine.run_batch(offs, row, col, w if weighted else None)
        return unpack(out, offs), qs, ks
    return run
