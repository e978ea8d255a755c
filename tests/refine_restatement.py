"""A second, independent restatement of the refinement step, in plain Python (test
infrastructure: it checks the C oracle's refine_partition on small graphs).

Leiden's RefinePartition / MergeNodesSubset (Traag, Waltman, van Eck 2019, Algorithm A.2) in
the greedy, pass-synchronous form the engine defines:

* refined partition starts as singletons; totals aref[v] = k_v;
* v is eligible iff, at the start, 2m * w(v, S - v) >= k_v * (K_S - k_v) (exact integers);
* each pass: every eligible v that is still a singleton looks at the refined communities of its
  neighbours inside S, evaluates the regular pass's gain (the reference's float formula with
  self = 0, a_own = k_v) under the mode's tie rule, and proposes the best if its gain is > 0;
* resolution from the pre-pass state: v -> t is kept unless t is a singleton that proposes,
  except that of two singletons proposing each other the higher id joins the lower;
* passes repeat while the refined partition's modularity rises by more than the threshold (and
  at most `max_passes` when that is > 0).
"""
from __future__ import annotations

import numpy as np


def _gain(w_vc: float, k: float, a_own: float, a_c: float, m: float) -> np.float32:
    # operatorsDelta.h:29-45: float subtraction w_vc - self (self = 0 here), the rest in double
    diff = np.float32(np.float32(w_vc) - np.float32(0.0))
    t1 = float(diff) / m
    t2 = (k * ((a_own - k) - a_c)) / ((2.0 * m) * m)
    return np.float32(t1 + t2)


def _modularity(row, col, w, part, tot, m) -> float:
    internal = 0
    for v in range(len(row) - 1):
        for e in range(row[v], row[v + 1]):
            if part[col[e]] == part[v]:
                internal += int(w[e])
    sq = sum(int(t) * int(t) for t in tot)
    return internal / (2.0 * m) - float(sq) / ((4.0 * m) * m)


def refine(row, col, w, k, comm, a, m, mode=1, threshold=1e-3, max_passes=0, max_iterations=10**9):
    """Refined labels (vertex ids) of the coarse partition `comm` with totals `a`; integer
    weights. mode: 0 HASH, 1 SORT, 2 ADAPTIVE_SPEED, 3 ADAPTIVE_MEMORY (their tie rules)."""
    n = len(row) - 1
    two_m = int(round(2.0 * m))
    kk = [int(round(x)) for x in k]
    K = [int(round(x)) for x in a]
    wi = [int(x) for x in w]
    elig = []
    for v in range(n):
        s = comm[v]
        wv = sum(wi[e] for e in range(row[v], row[v + 1]) if col[e] != v and comm[col[e]] == s)
        elig.append(two_m * wv >= kk[v] * (K[s] - kk[v]))
    ref = list(range(n))
    aref = [float(x) for x in k]
    size = [1] * n
    q = _modularity(row, col, wi, ref, aref, m)
    p = 0
    while True:
        hash_rule = mode in (0, 3) or (mode == 2 and p > 4)
        prop = list(ref)
        for v in range(n):
            if not (ref[v] == v and size[v] == 1 and elig[v]):
                continue
            acc = {}
            for e in range(row[v], row[v + 1]):
                u = col[e]
                if u == v or comm[u] != comm[v]:
                    continue
                acc[ref[u]] = acc.get(ref[u], 0.0) + wi[e]
            best_c, best_g, have = -1, np.float32(0.0), False
            for c in sorted(acc):
                if hash_rule and c == ref[v]:
                    continue
                g = _gain(acc[c], float(kk[v]), aref[ref[v]], aref[c], m)
                if hash_rule:
                    if g > 0 and (not have or g >= best_g):
                        best_c, best_g, have = c, g, True
                elif not have or g > best_g:
                    best_c, best_g, have = c, g, True
            if best_c >= 0 and best_c != ref[v] and best_g > 0:
                prop[v] = best_c
        keep = []
        for v in range(n):
            if prop[v] == ref[v]:
                continue
            t = prop[v]
            t_proposes = ref[t] == t and size[t] == 1 and prop[t] != t
            if not t_proposes or (prop[t] == v and t < v):
                keep.append(v)
        for v in keep:
            t, o = prop[v], ref[v]
            aref[t] += kk[v]
            aref[o] -= kk[v]
            ref[v] = t
            size[t] += 1
            size[o] -= 1
        qn = _modularity(row, col, wi, ref, aref, m)
        dq, q = qn - q, qn
        p += 1
        if not (dq > threshold) or p > max_iterations or (max_passes > 0 and p >= max_passes):
            return np.array(ref, dtype=np.int64)


def renumber(labels: np.ndarray) -> np.ndarray:
    """New ids in ascending label order (phaseAggregation.cuh:27-43 on the refined labels)."""
    used = np.unique(labels)
    return np.searchsorted(used, labels)
