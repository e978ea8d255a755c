// lv_refine.cuh -- the refinement phase: a Leiden-style refinement of each level's partition
// before it is aggregated. The reference has only an empty hook for it (RefinePhase,
// phaseRefine.cuh:1-3); the step follows Leiden's RefinePartition / MergeNodesSubset (Traag,
// Waltman, van Eck 2019, Algorithm A.2) in a greedy, pass-synchronous form:
//
//   * the refined partition starts as singletons: ref[v] = v, aref[v] = k_v, rsz[v] = 1;
//   * v may move iff it is still a singleton and was well connected to its community S when
//     the refinement began: 2m w(v, S - v) >= k_v (K_S - k_v), K_S = a[S];
//   * a pass evaluates, for each such v, the refined communities of its neighbours inside S
//     with the gain and tie rule of a regular pass and proposes the best one if its gain is > 0;
//   * proposals are resolved from the pre-pass state: v -> t is kept unless t is a singleton
//     that proposes a move itself, except that of two singletons proposing each other the
//     higher id joins the lower (so a vertex that is joined never leaves in the same pass, and
//     every refined community stays connected);
//   * passes repeat while the refined partition's modularity rises by more than the threshold.
//
// The passes reuse the optimisation kernels unchanged. They run through a second Dev (the
// "refine view") in which the graph is the level restricted to entries inside a community
// (rows in rowB/colB/wB, built by k_ref_count[_long] + scan + k_ref_fill[_long]), the partition is ref /
// ref_new, the totals aref and the graph states gsR. So a singleton's candidates are exactly
// the refined communities inside its own community, with self = 0 and a_own = k_v. Only the
// active set (k_ref_select) and the resolution (k_ref_resolve, k_ref_reject) are specific.
//
// After the passes the level is aggregated by the refined partition when it continues: a
// refined level continues iff its aggregate graph is smaller (n_ref < n) and either Q rose by
// more than the threshold since the previous level's end or n_ref < refine_tolerance * n
// (k_ref_decide); the next level starts from singletons as usual. Each new vertex remembers
// its members' community (prev, labelled by the community's smallest new vertex), so a run
// whose last level ends below the previous level's end returns the previous level's partition
// instead (k_ref_revert_*): a refined run never ends below an earlier level's end.
#pragma once

#include "lv_kernels.cuh"

namespace lv {

constexpr uint32_t kRefEligible = 1u;  // rflag: well connected to its community at the start
constexpr uint32_t kRefReject = 2u;    // rflag: this pass's proposal was not kept
// Rows longer than kRefLong entries are restricted in pieces of kHubPiece entries, one block
// per piece (queued in long_items, counted by long_count, both free until the aggregation):
// a warp per row would leave the GPU waiting on a few hub rows.
constexpr uint32_t kRefLong = 1024;

// Set-up of a refinement (main view). Graphs that aggregate now and are below the level cap
// refine (gsR[g].agg = 1, phase kIterating); the others sit it out (kFinished). The chunk
// early-return emulation is off for refinement passes (the next level start recomputes it).
__global__ void k_ref_init(int dslot, uint32_t max_levels) {
  const Dev& D = c_dev[dslot];
  Ctrl* C = D.ctrl;
  const uint32_t n = C->n;
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  for (uint32_t g = tid; g < C->G; g += nth) {
    GraphState r = D.gs[g];
    const bool on = r.agg && !(max_levels > 0 && r.level + 1 >= max_levels);
    r.phase = on ? kIterating : kFinished;
    r.agg = on ? 1u : 0u;
    r.I = 0ull;
    r.S = 0ull;
    r.iters = 0;
    r.total_iters = 0;
    r.n_next = 0;  // counts the refined communities at the end
    r.moved = 0;
    D.gsR[g] = r;
  }
  for (uint32_t v = tid; v < n; v += nth) {
    D.ref[v] = v;
    D.ref_new[v] = v;
    D.aref[v] = D.k[v];
    D.rsz[v] = 1u;
    D.rflag[v] = 0u;
  }
  if (tid == 0) {
    C->chunk_on = 0;
    C->n_next = n;  // length of the row-offset scan (kScanDeg scans n_next + 1 entries)
    C->long_count = 0;
  }
}

// The eligibility test 2m w(v, S - v) >= k_v (K_S - k_v), K_S = a[S]: exact in 128-bit integers
// (2m, k_v, K_S and w(v, S - v) are integers below 2^33), in double for fp32 weights.
template <bool WINT>
__device__ __forceinline__ bool ref_well_connected(const Dev& D, uint32_t v, uint32_t g, uint32_t cv,
                                                   unsigned long long wi, double wf) {
  const double m = D.gsR[g].m, kv = D.k[v], K = D.a[cv];
  if (WINT) {
    const unsigned long long two_m = (unsigned long long)__dmul_rn(2.0, m);
    const unsigned long long ki = (unsigned long long)kv, Ki = (unsigned long long)K;
    return (unsigned __int128)two_m * wi >= (unsigned __int128)ki * (Ki - ki);
  }
  return __dmul_rn(__dmul_rn(2.0, m), wf) >= __dmul_rn(kv, __dsub_rn(K, kv));
}

// Per vertex of a refining graph, a team of kRefT lanes per vertex (main view): its entries
// inside its community (the restricted row length, in newdeg for the offsets scan), the
// eligibility test and its self-loop weight (the singleton partition's internal weight).
// Rows longer than kRefLong are queued in pieces for k_ref_count_long.
constexpr int kRefT = 8;
template <bool WINT>
__global__ void __launch_bounds__(256) k_ref_count(int dslot) {
  const Dev& D = c_dev[dslot];
  using Tr = WTraits<WINT>;
  using Wt = typename Tr::W;
  using Acc = typename Tr::Acc;  // a row's weight sum is at most k_v
  const Wt* __restrict__ w = reinterpret_cast<const Wt*>(D.w);
  Ctrl* C = D.ctrl;
  const uint32_t n = C->n;
  const int lane = threadIdx.x & 31, tl = lane & (kRefT - 1);
  constexpr uint32_t kPerWarp = 32 / kRefT;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  // warp-uniform trip count: every lane reaches the team sums
  for (uint32_t vb = warp * kPerWarp; vb < n; vb += nwarps * kPerWarp) {
    const uint32_t v = vb + (uint32_t)(lane / kRefT);
    bool live = v < n;
    uint32_t g = 0, cv = 0, rs = 0, re = 0;
    if (live) {
      g = D.gid ? D.gid[v] : 0u;
      if (D.gsR[g].phase != kIterating) {
        if (tl == 0) D.newdeg[v] = 0;
        live = false;
      } else {
        cv = D.comm[v];
        rs = D.row[v];
        re = D.row[v + 1];
        if (re - rs > kRefLong) {
          // pieces for k_ref_count_long, which adds into newdeg[v] and hubself[v]
          if (tl == 0) {
            const uint32_t np = (re - rs + kHubPiece - 1) / kHubPiece;
            const uint32_t p0 = atomicAdd(&C->long_count, np);
            for (uint32_t k = 0; k < np; ++k) D.long_items[p0 + k] = ((unsigned long long)v << 32) | k;
            D.newdeg[v] = 0;
            D.hubself[v] = 0ull;
          }
          live = false;
        }
      }
    }
    uint32_t cnt = 0;
    Acc wi = Acc(0), si = Acc(0);
    if (live) {
      for (uint32_t e = rs + tl; e < re; e += kRefT) {
        const uint32_t u = D.col[e];
        if (D.comm[u] != cv) continue;
        ++cnt;
        if (u == v) si += (Acc)w[e]; else wi += (Acc)w[e];
      }
    }
    cnt = team_sum<kRefT>(cnt);
    wi = team_sum<kRefT>(wi);
    si = team_sum<kRefT>(si);
    if (live && tl == 0) {
      D.newdeg[v] = cnt;
      if (si != Acc(0)) {
        if (WINT) atomicAdd(&D.gsR[g].I, (unsigned long long)si);
        else atomicAdd(reinterpret_cast<double*>(&D.gsR[g].I), (double)si);
      }
      D.rflag[v] = ref_well_connected<WINT>(D, v, g, cv, (unsigned long long)wi, (double)wi)
                       ? kRefEligible : 0u;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) D.newdeg[n] = 0;
}

// A piece of a long row (main view), one block each: its kept entries, intra-community weight
// (into hubself[v]) and self-loop weight.
template <bool WINT>
__global__ void __launch_bounds__(256) k_ref_count_long(int dslot) {
  const Dev& D = c_dev[dslot];
  using Tr = WTraits<WINT>;
  using Wt = typename Tr::W;
  const Wt* __restrict__ w = reinterpret_cast<const Wt*>(D.w);
  __shared__ unsigned long long shu[33];
  __shared__ double shd[33];
  __shared__ uint32_t shc[33];
  Ctrl* C = D.ctrl;
  const uint32_t count = C->long_count, n = C->n;
  for (uint32_t idx = blockIdx.x; idx < count; idx += gridDim.x) {
    const unsigned long long it = D.long_items[idx];
    const uint32_t v = (uint32_t)(it >> 32), piece = (uint32_t)it;
    if (v >= n) continue;  // never: k_ref_count queued it
    const uint32_t g = D.gid ? D.gid[v] : 0u;
    const uint32_t cv = D.comm[v];
    const uint32_t rs = D.row[v] + piece * kHubPiece, re = min(D.row[v + 1], rs + kHubPiece);
    uint32_t cnt = 0;
    unsigned long long wi = 0, si = 0;
    double wf = 0.0, sf = 0.0;
    for (uint32_t e = rs + threadIdx.x; e < re; e += blockDim.x) {
      const uint32_t u = D.col[e];
      if (D.comm[u] != cv) continue;
      ++cnt;
      if (WINT) {
        if (u == v) si += (unsigned long long)w[e]; else wi += (unsigned long long)w[e];
      } else {
        if (u == v) sf += Tr::w_double(w[e]); else wf += Tr::w_double(w[e]);
      }
    }
    cnt = block_sum<256>(cnt, shc);
    if (WINT) { wi = block_sum<256>(wi, shu); si = block_sum<256>(si, shu); }
    else { wf = block_sum<256>(wf, shd); sf = block_sum<256>(sf, shd); }
    if (threadIdx.x == 0) {
      if (cnt) atomicAdd(&D.newdeg[v], cnt);
      if (WINT) {
        if (wi) atomicAdd(&D.hubself[v], wi);
        if (si) atomicAdd(&D.gsR[g].I, si);
      } else {
        if (wf != 0.0) atomicAdd(reinterpret_cast<double*>(&D.hubself[v]), wf);
        if (sf != 0.0) atomicAdd(reinterpret_cast<double*>(&D.gsR[g].I), sf);
      }
    }
  }
}

// Eligibility of the long rows, once their pieces are summed (main view): one thread per row
// (its first piece).
template <bool WINT>
__global__ void k_ref_elig_long(int dslot) {
  const Dev& D = c_dev[dslot];
  Ctrl* C = D.ctrl;
  const uint32_t count = C->long_count, n = C->n;
  for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < count; idx += gridDim.x * blockDim.x) {
    const unsigned long long it = D.long_items[idx];
    const uint32_t v = (uint32_t)(it >> 32), piece = (uint32_t)it;
    if (piece != 0 || v >= n) continue;
    const uint32_t g = D.gid ? D.gid[v] : 0u;
    const unsigned long long acc = D.hubself[v];
    D.rflag[v] = ref_well_connected<WINT>(D, v, g, D.comm[v], acc, __longlong_as_double((long long)acc))
                     ? kRefEligible : 0u;
    D.rank[v] = D.rowB[v];  // k_ref_fill_long's output cursor (rank is free until the aggregation)
  }
}

// The restricted rows (main view): entries inside the vertex's community, in row order, to
// rowB/colB/wB (offsets from the scan of k_ref_count's counts). One warp per row, a ballot per
// 32 entries places the kept ones (teams of kRefT lanes, as in k_ref_count, were slower here:
// 3.7 against 2.3 ms at R-MAT scale 22). Long rows are left to k_ref_fill_long.
template <bool WINT>
__global__ void __launch_bounds__(256) k_ref_fill(int dslot) {
  const Dev& D = c_dev[dslot];
  using Wt = typename WTraits<WINT>::W;
  const Wt* __restrict__ w = reinterpret_cast<const Wt*>(D.w);
  Wt* __restrict__ wo = reinterpret_cast<Wt*>(D.wB);
  const uint32_t n = D.ctrl->n;
  const int lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t v = warp; v < n; v += nwarps) {
    const uint32_t g = D.gid ? D.gid[v] : 0u;
    if (D.gsR[g].phase != kIterating) continue;
    const uint32_t cv = D.comm[v], rs = D.row[v], re = D.row[v + 1];
    if (re - rs > kRefLong) continue;  // k_ref_fill_long
    uint32_t out = D.rowB[v];
    for (uint32_t b = rs; b < re; b += 32) {
      const uint32_t e = b + lane;
      uint32_t u = 0;
      bool keep = false;
      if (e < re) {
        u = D.col[e];
        keep = D.comm[u] == cv;
      }
      const unsigned m = __ballot_sync(kFull, keep);
      if (keep) {
        const uint32_t p = out + __popc(m & lanemask_lt());
        D.colB[p] = u;
        wo[p] = w[e];
      }
      out += __popc(m);
    }
  }
}

// The long rows' pieces (main view), one block each: kept entries are placed through the row's
// cursor (rank[v]), one atomic per warp and 32 entries. Their order inside the row is not the
// level's; nothing depends on it (the refinement passes are table passes, their sums exact
// with integer weights).
template <bool WINT>
__global__ void __launch_bounds__(256) k_ref_fill_long(int dslot) {
  const Dev& D = c_dev[dslot];
  using Wt = typename WTraits<WINT>::W;
  const Wt* __restrict__ w = reinterpret_cast<const Wt*>(D.w);
  Wt* __restrict__ wo = reinterpret_cast<Wt*>(D.wB);
  Ctrl* C = D.ctrl;
  const uint32_t count = C->long_count, n = C->n;
  const int lane = threadIdx.x & 31;
  for (uint32_t idx = blockIdx.x; idx < count; idx += gridDim.x) {
    const unsigned long long it = D.long_items[idx];
    const uint32_t v = (uint32_t)(it >> 32), piece = (uint32_t)it;
    if (v >= n) continue;
    const uint32_t cv = D.comm[v];
    const uint32_t rs = D.row[v] + piece * kHubPiece, re = min(D.row[v + 1], rs + kHubPiece);
    const uint32_t lim = D.rowB[v + 1];
    // warp-uniform trip count: every lane takes part in each ballot
    for (uint32_t b = rs + (threadIdx.x & ~31u); b < re; b += blockDim.x) {
      const uint32_t e = b + lane;
      uint32_t u = 0;
      bool keep = false;
      if (e < re) {
        u = D.col[e];
        keep = D.comm[u] == cv;
      }
      const unsigned m = __ballot_sync(kFull, keep);
      if (!m) continue;
      uint32_t base = 0;
      if (lane == 0) base = atomicAdd(&D.rank[v], (uint32_t)__popc(m));
      base = __shfl_sync(kFull, base, 0);
      if (keep) {
        const uint32_t p = base + __popc(m & lanemask_lt());
        if (p < lim) {
          D.colB[p] = u;
          wo[p] = w[e];
        }
      }
    }
  }
}

// Active set of a refinement pass (refine view: comm = ref, gs = gsR): eligible singletons.
__global__ void k_ref_select(int dslot) {
  const Dev& D = c_dev[dslot];
  Ctrl* C = D.ctrl;
  const uint32_t n = C->n, it = C->it;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const uint32_t g = D.gid ? D.gid[v] : 0u;
    const bool on = D.gs[g].phase == kIterating && D.comm[v] == v && D.rsz[v] == 1u &&
                    (D.rflag[v] & kRefEligible);
    D.active_it[v] = on ? it : kNever;
  }
}

// The pass's movers (both lists of the optimisation kernels).
__device__ __forceinline__ uint32_t mover_at(const Dev& D, const Ctrl* C, uint32_t i, uint32_t count) {
  return D.movers[i < count ? i : C->n - 1u - (i - count)];
}

// Resolution (refine view), reading only the pre-pass state and the proposals: a proposal
// v -> t is rejected when t is a singleton that proposes too, unless t proposes v and t < v.
__global__ void k_ref_resolve(int dslot) {
  const Dev& D = c_dev[dslot];
  Ctrl* C = D.ctrl;
  const uint32_t count = C->mover_count, total = count + C->hub_mover_count, n = C->n;
  uint32_t err = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const uint32_t v = mover_at(D, C, i, count);
    const uint32_t t = D.new_comm[v];
    if (v >= n || t >= n) { err |= kErrIndex; continue; }
    const uint32_t pt = D.new_comm[t];
    const bool t_proposes = D.comm[t] == t && D.rsz[t] == 1u && pt != t;
    const bool keep = !t_proposes || (pt == v && t < v);
    if (!keep) D.rflag[v] |= kRefReject;
  }
  if (err) atomicOr(&C->err, err);
}

// Rejected proposals become "no move" (new_comm = comm; the apply kernels skip such movers);
// kept ones update the member counts.
__global__ void k_ref_reject(int dslot) {
  const Dev& D = c_dev[dslot];
  Ctrl* C = D.ctrl;
  const uint32_t count = C->mover_count, total = count + C->hub_mover_count, n = C->n;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const uint32_t v = mover_at(D, C, i, count);
    if (v >= n) continue;
    if (D.rflag[v] & kRefReject) {
      D.rflag[v] &= ~kRefReject;
      D.new_comm[v] = D.comm[v];
    } else {
      const uint32_t t = D.new_comm[v];
      if (t >= n) continue;
      atomicAdd(&D.rsz[t], 1u);
      atomicSub(&D.rsz[D.comm[v]], 1u);
    }
  }
}

// Refined communities per graph (main view): a label is in use iff its own vertex still holds
// it (only singletons move, and a joined vertex never leaves).
__global__ void k_ref_labels(int dslot) {
  const Dev& D = c_dev[dslot];
  const uint32_t n = D.ctrl->n;
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const uint32_t v = base + threadIdx.x;
    bool own = false;
    uint32_t g = 0;
    if (v < n) {
      g = D.gid ? D.gid[v] : 0u;
      own = D.gsR[g].agg && D.ref[v] == v;
    }
    if (!D.gid) {
      const unsigned m = __ballot_sync(kFull, own);
      if ((threadIdx.x & 31) == 0 && m) atomicAdd(&D.gsR[0].n_next, (uint32_t)__popc(m));
    } else if (own) {
      atomicAdd(&D.gsR[g].n_next, 1u);
    }
  }
}

// Whether each refined graph continues (main view). force >= 0 overrides (phase-level API).
// A continuing graph's end-of-level modularity becomes the baseline its next level's gain is
// measured from (kept by the level start), and its internal weight is rebuilt by the
// contraction from zero.
__global__ void k_ref_decide(int dslot, int force, double tolerance) {
  const Dev& D = c_dev[dslot];
  Ctrl* C = D.ctrl;
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < C->G; g += gridDim.x * blockDim.x) {
    GraphState* st = &D.gs[g];
    const GraphState& r = D.gsR[g];
    if (!st->agg || !r.agg) continue;
    const uint32_t ng = st->ve - st->vb, nref = r.n_next;
    uint32_t cont;
    if (force >= 0) cont = (uint32_t)force;
    else cont = (nref < ng && (st->cont || (double)nref < tolerance * (double)ng)) ? 1u : 0u;
    st->cont = cont;
    if (cont) {
      st->I = 0ull;
      st->Q_level = st->Q;
    }
  }
}

// Continuing refined graphs are aggregated by their refined partition (main view); their
// partition is kept in `coarse` for the prev labels.
__global__ void k_ref_swap(int dslot) {
  const Dev& D = c_dev[dslot];
  const uint32_t n = D.ctrl->n;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const uint32_t g = D.gid ? D.gid[v] : 0u;
    D.lab[v] = kEmpty;
    if (D.gs[g].agg && D.gs[g].cont && D.gsR[g].agg) {
      D.coarse[v] = D.comm[v];
      D.comm[v] = D.ref[v];
    }
  }
}

// After k_agg_count has given each vertex its next-level vertex (new_comm): every community of
// a continuing refined graph is labelled by its smallest next-level vertex ...
__global__ void k_ref_prev_label(int dslot) {
  const Dev& D = c_dev[dslot];
  const uint32_t n = D.ctrl->n;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const uint32_t g = D.gid ? D.gid[v] : 0u;
    if (D.gs[g].agg && D.gs[g].cont && D.gsR[g].agg) atomicMin(&D.lab[D.coarse[v]], D.new_comm[v]);
  }
}
// ... and each next-level vertex records that label (all its members share it).
__global__ void k_ref_prev(int dslot) {
  const Dev& D = c_dev[dslot];
  const uint32_t n = D.ctrl->n;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const uint32_t g = D.gid ? D.gid[v] : 0u;
    if (D.gs[g].agg && D.gs[g].cont && D.gsR[g].agg) D.prev[D.new_comm[v]] = D.lab[D.coarse[v]];
  }
}

// A graph that ends at a level above 0 with Q below the previous level's end (Q_level) ends
// with the previous level's partition: its vertices take their prev labels ...
__device__ __forceinline__ bool ref_reverts(const GraphState& st) {
  return st.agg && !st.cont && st.level > 0 && st.Q < st.Q_level;
}
__global__ void k_ref_revert_comm(int dslot) {
  const Dev& D = c_dev[dslot];
  const uint32_t n = D.ctrl->n;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const uint32_t g = D.gid ? D.gid[v] : 0u;
    if (ref_reverts(D.gs[g])) D.comm[v] = D.prev[v];
  }
}
// ... and its modularity is that level's.
__global__ void k_ref_revert_q(int dslot) {
  const Dev& D = c_dev[dslot];
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < D.ctrl->G; g += gridDim.x * blockDim.x) {
    GraphState* st = &D.gs[g];
    if (ref_reverts(*st)) st->Q = st->Q_level;
  }
}

}  // namespace lv
