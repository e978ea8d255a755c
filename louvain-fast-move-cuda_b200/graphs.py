"""Seeded synthetic graphs and the canonical CSR form the engine consumes.

Every generator returns a ``CSRGraph``: an undirected simple graph stored in both
directions, self-loops removed, duplicate pairs removed, isolated vertices dropped and
the surviving IDs compacted to 0..n-1 in ascending order, rows sorted by destination.
That is the shape the reference's own loader produces (graph.cu:27-82 dedups pairs,
emits both directions, subtracts min_id; graph.cuh:60-91 sorts by (src, dst)), and the
reference requires contiguous IDs with no isolated vertex (graph.cuh:79-91 builds the
degree array with reduce_by_key, which silently skips a vertex without edges).

Generators (all take ``seed``; numpy PCG64 through ``np.random.default_rng``):

* ``chung_lu_bounded``  -- degrees i.i.d. from a discrete power law on [dmin, dmax],
  edges drawn by endpoint sampling proportional to the target degree (the small
  power-law workload: n=10,000, exponent 2.0, degrees in [1, 99]).
* ``chung_lu_mean``     -- classic Chung-Lu weight sequence w_i ~ (i+1)^(-1/(g-1))
  scaled to a mean degree (the batched workload: exponent 2.1, mean degree 8).
* ``rmat``              -- R-MAT with (a, b, c, d) quadrant probabilities, edge factor
  ef, scale s (the single large workload: s=22, ef=16, .57/.19/.19/.05).
* ``planted_partition`` -- power-law community sizes, mixing parameter mu, fp32
  weights drawn from separate intra/inter ranges (the weighted workload).

Canonicalisation runs in numpy; ``to_device_canonical`` gives the same result with
torch on a CUDA device for the scale-22 graph (identical output: both are sort based).
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional

import numpy as np


@dataclasses.dataclass
class CSRGraph:
    """Symmetric CSR: row_ptr int64[n+1], col int32[E], w float32[E] or None (unit)."""

    n: int
    row_ptr: np.ndarray
    col: np.ndarray
    w: Optional[np.ndarray] = None
    name: str = ""
    truth: Optional[np.ndarray] = None  # ground-truth labels (planted partition only)

    @property
    def E(self) -> int:
        return int(self.row_ptr[-1])

    @property
    def m(self) -> int:
        """Undirected edge count (graph.cu:48 ``n_links``)."""
        return self.E // 2

    @property
    def weights_or_ones(self) -> np.ndarray:
        return self.w if self.w is not None else np.ones(self.E, dtype=np.float32)

    def src(self) -> np.ndarray:
        return np.repeat(np.arange(self.n, dtype=np.int32), np.diff(self.row_ptr))

    def degrees(self) -> np.ndarray:
        return np.diff(self.row_ptr)

    def edge_list_text(self) -> str:
        """``u v`` lines with u < v, the reference's unweighted input format (graph.cu:36)."""
        s = self.src()
        keep = s < self.col
        lines = np.char.add(np.char.add(s[keep].astype(str), " "), self.col[keep].astype(str))
        return "\n".join(lines.tolist()) + "\n"


def canonical_from_pairs(u: np.ndarray, v: np.ndarray, w: Optional[np.ndarray] = None,
                         name: str = "", truth: Optional[np.ndarray] = None) -> CSRGraph:
    """Symmetrise, drop self-loops and duplicate pairs (first weight wins), drop isolated
    vertices, compact IDs in ascending order, sort rows by destination."""
    u = np.asarray(u, dtype=np.int64)
    v = np.asarray(v, dtype=np.int64)
    keep = u != v
    u, v = u[keep], v[keep]
    if w is not None:
        w = np.asarray(w, dtype=np.float32)[keep]
    lo = np.minimum(u, v)
    hi = np.maximum(u, v)
    key = (lo << 32) | hi
    if w is None:
        key = np.unique(key)
        wu = None
    else:
        key, first = np.unique(key, return_index=True)
        wu = w[first]
    lo = key >> 32
    hi = key & 0xFFFFFFFF
    ids = np.unique(np.concatenate([lo, hi]))
    if truth is not None:
        truth = np.asarray(truth)[ids]
    lo = np.searchsorted(ids, lo)
    hi = np.searchsorted(ids, hi)
    n = int(ids.size)
    src = np.concatenate([lo, hi])
    dst = np.concatenate([hi, lo])
    k2 = (src << 32) | dst
    if wu is None:
        k2 = np.sort(k2)
        ww = None
    else:
        order = np.argsort(k2, kind="stable")
        k2 = k2[order]
        ww = np.concatenate([wu, wu])[order].astype(np.float32)
    src = (k2 >> 32).astype(np.int64)
    col = (k2 & 0xFFFFFFFF).astype(np.int32)
    counts = np.bincount(src, minlength=n)
    row_ptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=row_ptr[1:])
    return CSRGraph(n=n, row_ptr=row_ptr, col=col, w=ww, name=name, truth=truth)


def _discrete_power_law(rng: np.random.Generator, size: int, exponent: float,
                        dmin: int, dmax: int) -> np.ndarray:
    support = np.arange(dmin, dmax + 1, dtype=np.float64)
    p = support ** (-exponent)
    cdf = np.cumsum(p)
    cdf /= cdf[-1]
    return (np.searchsorted(cdf, rng.random(size)) + dmin).astype(np.int64)


def _endpoint_sample(rng: np.random.Generator, weights: np.ndarray, n_edges: int):
    cdf = np.cumsum(weights, dtype=np.float64)
    cdf /= cdf[-1]
    u = np.searchsorted(cdf, rng.random(n_edges), side="right")
    v = np.searchsorted(cdf, rng.random(n_edges), side="right")
    n = weights.size
    return np.minimum(u, n - 1), np.minimum(v, n - 1)


def chung_lu_bounded(n: int = 10_000, exponent: float = 2.0, dmin: int = 1, dmax: int = 99,
                     seed: int = 1) -> CSRGraph:
    """Chung-Lu graph whose target degrees are i.i.d. discrete power law on [dmin, dmax]."""
    rng = np.random.default_rng(seed)
    deg = _discrete_power_law(rng, n, exponent, dmin, dmax)
    n_edges = int(deg.sum() // 2)
    u, v = _endpoint_sample(rng, deg.astype(np.float64), n_edges)
    return canonical_from_pairs(u, v, name=f"chung_lu_n{n}_g{exponent}_d{dmin}-{dmax}_s{seed}")


def chung_lu_mean(n: int, exponent: float = 2.1, mean_degree: float = 8.0,
                  seed: int = 1) -> CSRGraph:
    """Chung-Lu graph with weight sequence w_i ~ (i+1)^(-1/(exponent-1)), mean degree fixed."""
    rng = np.random.default_rng(seed)
    i = np.arange(n, dtype=np.float64)
    wts = (i + 1.0) ** (-1.0 / (exponent - 1.0))
    wts *= mean_degree * n / wts.sum()
    wts = np.minimum(wts, math.sqrt(wts.sum()))
    n_edges = int(round(mean_degree * n / 2))
    u, v = _endpoint_sample(rng, wts, n_edges)
    perm = rng.permutation(n)  # hubs are not all at low IDs
    return canonical_from_pairs(perm[u], perm[v], name=f"chung_lu_n{n}_g{exponent}_k{mean_degree}_s{seed}")


def rmat_pairs(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19,
               c: float = 0.19, seed: int = 1, chunk: int = 1 << 23):
    """Raw R-MAT endpoint arrays (int64), before canonicalisation."""
    rng = np.random.default_rng(seed)
    n_edges = edge_factor << scale
    us = np.empty(n_edges, dtype=np.int64)
    vs = np.empty(n_edges, dtype=np.int64)
    ab, abc = np.float32(a + b), np.float32(a + b + c)
    fa = np.float32(a)
    for lo in range(0, n_edges, chunk):
        hi = min(lo + chunk, n_edges)
        cnt = hi - lo
        u = np.zeros(cnt, dtype=np.int64)
        v = np.zeros(cnt, dtype=np.int64)
        for _ in range(scale):
            r = rng.random(cnt, dtype=np.float32)
            ubit = r >= ab                       # quadrants c, d
            vbit = ((r >= fa) & (r < ab)) | (r >= abc)  # quadrants b, d
            u = (u << 1) | ubit
            v = (v << 1) | vbit
        us[lo:hi] = u
        vs[lo:hi] = v
    return us, vs


def rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19,
         c: float = 0.19, seed: int = 1) -> CSRGraph:
    """R-MAT graph, unit weights, canonicalised (isolated vertices dropped)."""
    u, v = rmat_pairs(scale, edge_factor, a, b, c, seed)
    return canonical_from_pairs(u, v, name=f"rmat_s{scale}_ef{edge_factor}_s{seed}")


def planted_partition(n: int = 1_000_000, n_comm: int = 1000, exponent: float = 1.5,
                      smin: int = 100, smax: int = 5000, mean_degree: float = 20.0,
                      mu: float = 0.3, w_in=(0.5, 1.5), w_out=(0.1, 0.5),
                      seed: int = 1) -> CSRGraph:
    """Weighted planted partition with power-law community sizes and ground truth."""
    rng = np.random.default_rng(seed)
    sizes = _discrete_power_law(rng, n_comm, exponent, smin, smax).astype(np.float64)
    sizes = np.maximum(np.round(sizes * n / sizes.sum()), 1).astype(np.int64)
    sizes[-1] += n - sizes.sum()
    if sizes[-1] < 1:
        raise ValueError("community size rescaling failed")
    label = np.repeat(np.arange(n_comm, dtype=np.int64), sizes)
    start = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    n_edges = int(round(mean_degree * n / 2))
    n_out = int(round(mu * n_edges))
    n_in = n_edges - n_out
    ui = rng.integers(0, n, n_in)
    ci = label[ui]
    vi = start[ci] + (rng.random(n_in) * sizes[ci]).astype(np.int64)
    uo = rng.integers(0, n, n_out)
    vo = rng.integers(0, n, n_out)
    same = label[uo] == label[vo]
    vo[same] = (vo[same] + sizes[label[vo[same]]] ) % n  # push to another block
    wi = rng.uniform(w_in[0], w_in[1], n_in).astype(np.float32)
    wo = rng.uniform(w_out[0], w_out[1], n_out).astype(np.float32)
    u = np.concatenate([ui, uo])
    v = np.concatenate([vi, vo])
    w = np.concatenate([wi, wo])
    return canonical_from_pairs(u, v, w, name=f"planted_n{n}_c{n_comm}_mu{mu}_s{seed}",
                                truth=label)


def nmi(a: np.ndarray, b: np.ndarray) -> float:
    """Normalised mutual information of two labelings, I(A;B) / sqrt(H(A) H(B)) in nats
    (the geometric normalisation); 1.0 when both labelings have a single class."""
    a = np.unique(np.asarray(a), return_inverse=True)[1].astype(np.int64)
    b = np.unique(np.asarray(b), return_inverse=True)[1].astype(np.int64)
    n = a.size
    if n == 0:
        return 1.0
    pair, cnt = np.unique(a * (int(b.max()) + 1) + b, return_counts=True)
    ca = np.bincount(a).astype(np.float64)
    cb = np.bincount(b).astype(np.float64)
    pa, pb = ca / n, cb / n
    ha = -np.sum(pa * np.log(pa))
    hb = -np.sum(pb * np.log(pb))
    pij = cnt / n
    ia = pair // (int(b.max()) + 1)
    ib = pair % (int(b.max()) + 1)
    mi = float(np.sum(pij * (np.log(pij) - np.log(pa[ia]) - np.log(pb[ib]))))
    if ha <= 0.0 or hb <= 0.0:
        return 1.0 if ha == hb else 0.0
    return max(0.0, min(1.0, mi / np.sqrt(ha * hb)))


def read_edge_list(path: str, skip_line: int = 0) -> CSRGraph:
    """Parse an unweighted ``a b`` edge list the way the reference's GraphHost does
    (graph.cu:17-87): skip header lines, dedup undirected pairs, emit both directions with
    weight 1, subtract the smallest ID. IDs must then be contiguous (the reference needs
    that too, graph.cuh:66-91); this raises instead of silently mis-indexing."""
    with open(path, "r") as f:
        for _ in range(skip_line):
            f.readline()
        data = np.array(f.read().split(), dtype=np.int64)
    if data.size == 0:
        raise ValueError("Error during parsing: no node found")
    data = data[: data.size // 2 * 2].reshape(-1, 2)
    ids = np.unique(data)
    if ids[-1] - ids[0] + 1 != ids.size:
        raise ValueError("vertex IDs are not contiguous")
    g = canonical_from_pairs(data[:, 0] - ids[0], data[:, 1] - ids[0], name=path)
    if g.n != ids.size:
        raise ValueError("input has vertices whose only edges are self-loops")
    return g


def to_device_canonical(u, v, device="cuda", name: str = "") -> CSRGraph:
    """torch version of ``canonical_from_pairs`` (unit weights) for the scale-22 graph; the
    output is identical because every step is a sort or a unique."""
    import torch

    u = torch.as_tensor(u, device=device, dtype=torch.int64)
    v = torch.as_tensor(v, device=device, dtype=torch.int64)
    keep = u != v
    u, v = u[keep], v[keep]
    lo = torch.minimum(u, v)
    hi = torch.maximum(u, v)
    del u, v
    key = torch.unique((lo << 32) | hi)
    lo = key >> 32
    hi = key & 0xFFFFFFFF
    ids = torch.unique(torch.cat([lo, hi]))
    lo = torch.searchsorted(ids, lo)
    hi = torch.searchsorted(ids, hi)
    n = int(ids.numel())
    k2 = torch.sort(torch.cat([(lo << 32) | hi, (hi << 32) | lo])).values
    src = k2 >> 32
    col = (k2 & 0xFFFFFFFF).to(torch.int32)
    counts = torch.bincount(src, minlength=n)
    row_ptr = torch.zeros(n + 1, dtype=torch.int64, device=device)
    row_ptr[1:] = torch.cumsum(counts, 0)
    return CSRGraph(n=n, row_ptr=row_ptr.cpu().numpy(), col=col.cpu().numpy(), w=None, name=name)


@dataclasses.dataclass
class PackedBatch:
    """Many graphs packed into one CSR on a device: vertex ranges vtx_offsets[g]..[g+1],
    global column IDs, unit weights. Tensors are torch (int64 offsets/row_ptr, int32 col)."""
    vtx_offsets: object
    row_ptr: object
    col: object
    n: np.ndarray   # vertices per graph (host)
    m: np.ndarray   # undirected edges per graph (host)
    name: str = ""

    @property
    def G(self) -> int:
        return int(self.n.size)

    def graph(self, g: int):
        """Graph g as (n, row_ptr, col) device tensors with local IDs (for single-graph runs)."""
        import torch
        vb = int(self.vtx_offsets[g]); ve = int(self.vtx_offsets[g + 1])
        rp = self.row_ptr[vb: ve + 1]
        e0 = int(rp[0])
        return ve - vb, (rp - e0).contiguous(), (self.col[e0: int(rp[-1])] - vb).to(torch.int32).contiguous()


def _device_csr_from_keys(lo, hi, n_total: int, vtx_offsets_old, device):
    """Deduplicated undirected pairs (global IDs) -> packed CSR with isolated vertices dropped
    and IDs compacted in ascending order; vertex offsets move with the compaction."""
    import torch
    key = torch.unique((lo << 32) | hi)
    lo = key >> 32
    hi = key & 0xFFFFFFFF
    del key
    ids = torch.unique(torch.cat([lo, hi]))
    lo = torch.searchsorted(ids, lo)
    hi = torch.searchsorted(ids, hi)
    offs = torch.searchsorted(ids, vtx_offsets_old)
    n = int(ids.numel())
    del ids
    k2 = torch.sort(torch.cat([(lo << 32) | hi, (hi << 32) | lo])).values
    del lo, hi
    src = k2 >> 32
    col = (k2 & 0xFFFFFFFF).to(torch.int32)
    del k2
    counts = torch.bincount(src, minlength=n)
    del src
    row_ptr = torch.zeros(n + 1, dtype=torch.int64, device=device)
    row_ptr[1:] = torch.cumsum(counts, 0)
    return offs, row_ptr, col


def chung_lu_batch_device(G: int = 4096, n_min: int = 200, n_max: int = 200_000,
                          exponent: float = 2.1, mean_degree: float = 8.0, seed: int = 1,
                          device="cuda") -> PackedBatch:
    """The batched workload, generated on a CUDA device with torch: G independent Chung-Lu
    graphs (the ``chung_lu_mean`` weight sequence w_i ~ (i+1)^(-1/(exponent-1)), mean degree
    fixed, weights capped at sqrt(sum)), vertex counts log-uniform in [n_min, n_max], each
    graph's IDs randomly permuted, canonicalised per graph and packed. Vertex counts come from
    numpy's PCG64 with ``seed``; the endpoints from torch's device generator with ``seed``."""
    import torch
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(math.log(n_min), math.log(n_max), G)).astype(np.int64)
    ms = np.rint(mean_degree * ns / 2.0).astype(np.int64)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    ns_t = torch.from_numpy(ns).to(device)
    voff = torch.zeros(G + 1, dtype=torch.int64, device=device)
    voff[1:] = torch.cumsum(ns_t, 0)
    N = int(ns.sum())
    gid = torch.repeat_interleave(torch.arange(G, device=device), ns_t)
    local = torch.arange(N, device=device, dtype=torch.int64) - voff[gid]
    wts = (local.to(torch.float64) + 1.0) ** (-1.0 / (exponent - 1.0))
    del local
    wsum = torch.zeros(G, dtype=torch.float64, device=device).index_add_(0, gid, wts)
    wts *= (mean_degree * ns_t.to(torch.float64) / wsum)[gid]
    wts = torch.minimum(wts, torch.sqrt(mean_degree * ns_t.to(torch.float64))[gid])
    # per-graph CDF shifted by the graph index: segment g covers (g, g + 1]
    c = torch.cumsum(wts, 0)
    del wts
    start = torch.zeros(G, dtype=torch.float64, device=device)
    start[1:] = c[voff[1:-1] - 1]
    total = c[voff[1:] - 1] - start
    cdf = (c - start[gid]) / total[gid] + gid.to(torch.float64)
    del c
    ms_t = torch.from_numpy(ms).to(device)
    eg = torch.repeat_interleave(torch.arange(G, device=device), ms_t)
    last = voff[1:] - 1

    def endpoints():
        r = torch.rand(eg.numel(), generator=gen, device=device, dtype=torch.float64) + eg.to(torch.float64)
        return torch.minimum(torch.searchsorted(cdf, r, right=True), last[eg])

    u = endpoints()
    v = endpoints()
    del cdf
    # random relabelling inside each graph so hubs are not all at low IDs
    keys = torch.rand(N, generator=gen, device=device, dtype=torch.float64) + gid.to(torch.float64)
    order = torch.argsort(keys)
    del keys
    newid = torch.empty_like(order)
    newid[order] = torch.arange(N, device=device, dtype=torch.int64)
    del order
    u = newid[u]
    v = newid[v]
    del newid, eg, gid
    keep = u != v
    u, v = u[keep], v[keep]
    lo = torch.minimum(u, v)
    hi = torch.maximum(u, v)
    del u, v, keep
    offs, row_ptr, col = _device_csr_from_keys(lo, hi, N, voff, device)
    offs_h = offs.cpu().numpy()
    rp_h = row_ptr[offs].cpu().numpy()
    n_out = np.diff(offs_h)
    m_out = np.diff(rp_h) // 2
    return PackedBatch(offs, row_ptr, col, n_out, m_out,
                       name=f"chung_lu_batch_G{G}_n{n_min}-{n_max}_g{exponent}_k{mean_degree}_s{seed}")


def rmat_device(n_target: int, edge_factor: int = 8, a: float = 0.57, b: float = 0.19,
                c: float = 0.19, seed: int = 1, device="cuda") -> CSRGraph:
    """R-MAT graph with about n_target vertices, generated on a CUDA device: edge_factor *
    n_target edges drawn at scale ceil(log2 n_target), IDs scaled down onto [0, n_target)
    (u * n_target >> scale keeps the skew), then canonicalised (host CSR returned)."""
    import torch
    scale = max(1, int(math.ceil(math.log2(max(2, n_target)))))
    n_edges = edge_factor * n_target
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    u = torch.zeros(n_edges, dtype=torch.int64, device=device)
    v = torch.zeros(n_edges, dtype=torch.int64, device=device)
    ab, abc = a + b, a + b + c
    for _ in range(scale):
        r = torch.rand(n_edges, generator=gen, device=device, dtype=torch.float32)
        ubit = r >= ab
        vbit = ((r >= a) & (r < ab)) | (r >= abc)
        u = (u << 1) | ubit
        v = (v << 1) | vbit
    u = (u * n_target) >> scale
    v = (v * n_target) >> scale
    return to_device_canonical(u, v, device=device, name=f"rmat_n{n_target}_ef{edge_factor}_s{seed}")


def edge_list_bytes(u: np.ndarray, v: np.ndarray) -> bytes:
    """``"u v\\n"`` lines for non-negative integer arrays, formatted with vectorised digit
    extraction (no per-line Python work)."""
    u = np.asarray(u, dtype=np.int64)
    v = np.asarray(v, dtype=np.int64)
    if u.size and min(int(u.min()), int(v.min())) < 0:
        raise ValueError("non-negative ids only")

    def ndig(x):
        d = np.ones(x.shape, dtype=np.int64)
        p = 10
        for _ in range(18):
            d += x >= p
            p *= 10
        return d

    du, dv = ndig(u), ndig(v)
    line = du + dv + 2
    end = np.cumsum(line)
    start = end - line
    buf = np.empty(int(end[-1]) if end.size else 0, dtype=np.uint8)

    def put(x, nd, first):
        y = x.copy()
        for k in range(int(nd.max()) if nd.size else 0):
            m = k < nd
            buf[(first + nd - 1 - k)[m]] = (y[m] % 10 + 48).astype(np.uint8)
            y //= 10

    put(u, du, start)
    buf[start + du] = ord(" ")
    put(v, dv, start + du + 1)
    buf[end - 1] = ord("\n")
    return buf.tobytes()
