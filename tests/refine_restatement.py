"""A second, independent restatement of the refined pipeline, in plain Python (test
infrastructure: it checks the C oracle's refine_partition and its refined level loop on small
graphs). `refine` is the refinement step; `louvain_refined` the whole run: the reference's
passes (fast pass with the v <= c gate, SORT / HASH tie rules, synchronous moves, the active
set), the refinement, aggregation by the refined partition, the continuation rule (a smaller
aggregate and either a gain above the threshold since the previous level's end or fewer than
tolerance x n refined communities) and the return to the previous level's partition when the
last level ends below it.

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


# ---- the whole refined run (small graphs; no edge chunking) ---------------------------------------
def _gain_self(w_vc: float, self_v: float, k: float, a_own: float, a_c: float, m: float) -> np.float32:
    diff = np.float32(np.float32(w_vc) - np.float32(self_v))
    t1 = float(diff) / m
    t2 = (k * ((a_own - k) - a_c)) / ((2.0 * m) * m)
    return np.float32(t1 + t2)


def _pass(row, col, w, k, comm, a, active, m, mode, it_in_level, fast):
    """One synchronous pass with the reference's rules; returns the moved flags."""
    n = len(row) - 1
    hash_rule = (not fast) and (mode in (0, 3) or (mode == 2 and it_in_level > 4))
    dec = [-1] * n
    dg = [np.float32(0.0)] * n
    for v in range(n):
        if not active[v] or not any(col[e] != v for e in range(row[v], row[v + 1])):
            continue
        cv, kv, a_own = comm[v], k[v], a[comm[v]]
        bc, bg, have = -1, np.float32(0.0), False
        if fast:
            for e in range(row[v], row[v + 1]):
                u = col[e]
                if u == v:
                    continue
                g = _gain_self(w[e], 0.0, kv, a_own, a[comm[u]], m)
                if not have or g > bg:
                    bc, bg, have = comm[u], g, True
        else:
            acc = {}
            for e in range(row[v], row[v + 1]):
                u = col[e]
                if u != v:
                    acc[comm[u]] = acc.get(comm[u], 0.0) + w[e]
            self_v = float(np.float32(acc[cv])) if cv in acc else 0.0
            for c in sorted(acc):
                if hash_rule and c == cv:
                    continue
                g = _gain_self(acc[c], self_v, kv, a_own, a[c], m)
                if hash_rule:
                    if g > 0 and (not have or g >= bg):
                        bc, bg, have = c, g, True
                elif not have or g > bg:
                    bc, bg, have = c, g, True
        dec[v], dg[v] = bc, bg
    moved = [False] * n
    for v in range(n):
        c = dec[v]
        if c < 0 or comm[v] == c or not (dg[v] > 0) or (fast and v > c):
            continue
        a[c] += k[v]
        a[comm[v]] -= k[v]
        comm[v] = c
        moved[v] = True
    for v in range(n):
        active[v] = any(moved[col[e]] and comm[col[e]] != comm[v] for e in range(row[v], row[v + 1]))
    return moved


def _aggregate(row, col, w, part):
    """Renumber `part` by ascending label, contract: sorted rows, summed integer weights."""
    n = len(row) - 1
    new = renumber(np.array(part))
    n2 = int(new.max()) + 1
    rows = [dict() for _ in range(n2)]
    for v in range(n):
        r = rows[new[v]]
        for e in range(row[v], row[v + 1]):
            d = int(new[col[e]])
            r[d] = r.get(d, 0) + int(w[e])
    row2, col2, w2 = [0], [], []
    for r in rows:
        for d in sorted(r):
            col2.append(d)
            w2.append(r[d])
        row2.append(len(col2))
    k2 = [float(sum(w2[row2[s]:row2[s + 1]])) for s in range(n2)]
    return new, row2, col2, w2, k2


def louvain_refined(row, col, w, mode=1, threshold=1e-3, tolerance=0.95, fast_first=True,
                    max_passes=0, info=None):
    """Final (best partition per input vertex, modularity) of a refined run; `info` (a dict),
    if given, receives the number of levels and whether the run returned to the previous
    level's partition."""
    row, col, w = list(row), list(col), [int(x) for x in w]
    n0 = len(row) - 1
    k = [float(sum(w[row[v]:row[v + 1]])) for v in range(n0)]
    m = sum(k) / 2.0
    best = np.arange(n0)
    prev = None      # per vertex: its members' community at the previous level's end
    prev_end = 0.0
    level = 0
    while True:
        n = len(row) - 1
        comm, a, active = list(range(n)), list(k), [True] * n
        q = _modularity(row, col, w, comm, a, m)
        start = q
        it = 0
        while True:
            _pass(row, col, w, k, comm, a, active, m, mode, it, fast_first and it == 0)
            it += 1
            qn = _modularity(row, col, w, comm, a, m)
            delta, q = qn - q, qn
            if not (delta > threshold):
                break
        old = prev_end if level > 0 else start
        cont = (q - old) > threshold
        prev_end = q
        labels = refine(row, col, w, k, comm, a, m, mode=mode, threshold=threshold, max_passes=max_passes)
        n_ref = int(sum(1 for v in range(n) if labels[v] == v))
        cont = n_ref < n and (cont or n_ref < tolerance * n)
        if not cont:
            final = comm
            reverted = level > 0 and q < old
            if reverted:
                final, q = prev, old
            if info is not None:
                info["levels"] = level + 1
                info["reverted"] = reverted
            ids = renumber(np.array(final))
            return ids[best], q
        new, row2, col2, w2, k2 = _aggregate(row, col, w, labels)
        # each new vertex keeps its members' community, labelled by its smallest new vertex
        lab = {}
        for v in range(n):
            lab[comm[v]] = min(lab.get(comm[v], 1 << 62), int(new[v]))
        prev = [0] * (int(new.max()) + 1)
        for v in range(n):
            prev[int(new[v])] = lab[comm[v]]
        best = new[best]
        row, col, w, k = row2, col2, w2, k2
        level += 1


def louvain_plain(row, col, w, mode=1, threshold=1e-3, fast_first=True):
    """Final (best partition per input vertex, modularity) of an unrefined run: the level loop
    of modularityAlgorithms.h:31-67 over the same passes (small graphs, no edge chunking)."""
    row, col, w = list(row), list(col), [int(x) for x in w]
    n0 = len(row) - 1
    k = [float(sum(w[row[v]:row[v + 1]])) for v in range(n0)]
    m = sum(k) / 2.0
    best = np.arange(n0)
    while True:
        n = len(row) - 1
        comm, a, active = list(range(n)), list(k), [True] * n
        q = _modularity(row, col, w, comm, a, m)
        start = q
        it = 0
        while True:
            _pass(row, col, w, k, comm, a, active, m, mode, it, fast_first and it == 0)
            it += 1
            qn = _modularity(row, col, w, comm, a, m)
            delta, q = qn - q, qn
            if not (delta > threshold):
                break
        new, row2, col2, w2, k2 = _aggregate(row, col, w, comm)
        best = new[best]
        if not (q - start) > threshold:
            return best, q
        row, col, w, k = row2, col2, w2, k2
