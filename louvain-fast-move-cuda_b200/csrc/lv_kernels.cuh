// lv_kernels.cuh -- the engine's sm_100a kernels.
//
// One pass of the optimisation phase (the reference's optimize() + fast_move_update() +
// compute_modularity(), phaseOptimization.cuh:116-181) is, here:
//   k_chunk_flags -> k_bin_vertices -> k_opt_team<T> x6 / k_opt_block x2 -> k_apply ->
//   k_commit_sq -> k_finalize
// and aggregation (phaseAggregation.cuh:19-190) is:
//   k_agg_flags -> scan -> k_agg_meta -> k_agg_best -> k_agg_count -> scan -> k_agg_scatter
//   -> k_agg_bin -> k_contract_team<T> x6 / k_contract_block x2 -> scan -> k_agg_compact
// All loops are grid-stride over sizes read from the device control block, so the grids do
// not depend on the level and the sequence can be captured once and replayed.
#pragma once

#include "lv_device.cuh"

namespace lv {

// Everything a kernel needs about the current level. Pointers never change during a run
// (aggregation copies the next level into the same buffers), so a captured launch stays
// valid from level to level.
struct Dev {
  uint32_t* row;        // [n+1] edge offsets
  uint32_t* col;        // [E] destination vertex
  void* w;              // [E] u32 (integer mode) or f32 weights
  double* k;            // [n] tot_weight_per_nodes
  uint32_t* gid;        // [n] graph of each vertex (nullptr: one graph)
  uint32_t* comm;       // [n] communities
  double* a;            // [n] communities_weight
  uint32_t* new_comm;   // [n] target of this pass's move
  uint32_t* active_it;  // [n] pass stamp for which the vertex is active
  uint32_t* bins[kListBins];  // vertex lists per degree bin (+ kHalfBin)
  uint32_t* hub_off;    // [n] arena offset per entry of the global-table bin
  uint32_t* hubtab;     // [n] aggregation: arena offset of each bin-7 new community, else kEmpty
  unsigned long long* hubself;  // [n] aggregation: self-loop weight of each bin-7 community
  unsigned long long* long_items;  // [n + E/kHubPiece + 16] (vertex << 32 | piece) of long rows
  unsigned long long* apply_items; // [n + E/kHubPiece + 16] (mover << 32 | piece) of hub movers
  uint32_t* movers;     // [n]
  uint32_t* arena_keys;
  void* arena_vals;     // 8 bytes per slot
  uint32_t* hub_owner;  // [arena slots / kHubChunk] new community owning each table chunk
  GraphState* gs;
  Ctrl* ctrl;
  double* partials;     // [kMaxPartials] per-block partial sums (single graph)
  // aggregation scratch
  unsigned long long* map;   // [n] packed (nonempty, nonempty&&continue) inclusive counts
  unsigned long long* cd;    // [n+1] packed (member count, degree sum) per new community
  uint32_t* rank;            // [n] rank of a vertex inside its new community
  uint32_t* members;         // [n]
  uint32_t* newdeg;          // [n+1]
  uint32_t* rowB;            // [n+1]
  uint32_t* colB;            // [E]
  void* wB;                  // [E]
  double* kB;                // [n]
  uint32_t* gidB;            // [n]
  uint32_t* best;            // [n0] current-level vertex of each input vertex
  uint32_t* gid0;            // [n0] graph of each input vertex (nullptr: one graph)
  int32_t* out;              // [n0] final community ids
  unsigned long long* scan_tmp;  // [(n + 1) / kScanTile + 2] tile sums of the scans
  unsigned long long* cn;    // [n] apply phase: (new_comm << 32) | comm, one gather per entry
  // [n] table passes with integer weights: (total of comm[v] << 32) | comm[v], written by
  // k_bin_vertices, so that an entry's community and that community's total (a u32: integer
  // totals stay below 2m < 2^32) arrive with one gather
  unsigned long long* ca;
  // refinement (allocated only when it is on; lv_refine.cuh)
  uint32_t* ref;             // [n] refined partition
  uint32_t* ref_new;         // [n] its pass targets
  double* aref;              // [n] refined totals
  uint32_t* rsz;             // [n] members per refined label
  uint32_t* rflag;           // [n] kRefEligible / kRefReject
  GraphState* gsR;           // [G] graph states of the refinement passes
  uint32_t* coarse;          // [n] the level's partition, kept when aggregating by ref
  uint32_t* lab;             // [n] per community of the level: its smallest next-level vertex
  uint32_t* prev;            // [n] per vertex: its members' community at the previous level's end
};

// The Dev of every live slot (a context's, each serving slot's), in constant memory: kernels
// take the slot index and read their pointers through the constant cache, as fast as kernel
// parameters, while a captured graph's arguments stay fixed from run to run.
constexpr int kMaxDevSlots = 96;
__constant__ Dev c_dev[kMaxDevSlots];

struct BinCfg {
  uint32_t maxdeg[kNumBins];  // bin b: maxdeg[b-1] < d <= maxdeg[b]; the last bin is open
  uint32_t block_cap;         // shared-memory table slots of the block kernels (bin 6)
};

// Table granule of the multi-block global tables: every global table is a multiple of it.
constexpr uint32_t kHubChunk = 4096;
// In the contraction's global tables, rows longer than kHubLongRow entries are inserted in
// pieces of kHubInsPiece by separate blocks (k_hub_insert_long); shorter ones by warps taking
// 32 member rows at a time (k_hub_insert). At R-MAT scale 22 a 256-entry split costs 5.2 ms
// for both kernels against 6.0 ms with 2048 (one warp per 2048-entry piece: 6.1 ms).
constexpr uint32_t kHubLongRow = 256;
constexpr uint32_t kHubInsPiece = 8192;
constexpr uint32_t kHubPiece = 8192;

constexpr int kMaxPartials = 2048;

// Capacity of a bin-7 vertex's global optimisation table: table_cap rounded up to a whole
// kHubChunk, so every chunk of the arena belongs to one vertex.
__device__ __forceinline__ uint32_t hub_table_cap(uint32_t d, uint32_t ng) {
  const uint32_t c = table_cap(d, ng);
  return c < kHubChunk ? kHubChunk : c;
}

// Error bits found by a kernel, and which kernel found them (Ctrl::err_site, bit `site`), so
// that a failed device check names the kernel.
__device__ __forceinline__ void report_err(Ctrl* C, uint32_t err, int site) {
  atomicOr(&C->err, err);
  atomicOr(&C->err_site, 1u << site);
}

__device__ __forceinline__ int bin_of(const BinCfg& B, uint32_t d) {
#pragma unroll
  for (int b = 0; b < kNumBins - 1; ++b)
    if (d <= B.maxdeg[b]) return b;
  return kNumBins - 1;
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Append `item` to list `b` with one atomic per warp and bin. Every lane of the warp must
// call it (bin == -1 for lanes with nothing to append). Returns the slot or kEmpty.
__device__ __forceinline__ uint32_t warp_append(int bin, int b, uint32_t* counter) {
  const unsigned mask = __ballot_sync(kFull, bin == b);
  if (!mask) return kEmpty;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(mask) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
  base = __shfl_sync(kFull, base, leader);
  return bin == b ? base + __popc(mask & lanemask_lt()) : kEmpty;
}

// Does vertex v take part in this pass at all: the reference's copy_if keeps edges with
// changed[src] && src != dst (operatorsCommunity.h:7-19), so a vertex whose only entries are
// self-loops selects nothing.
__device__ __forceinline__ bool has_nonloop(const Dev& D, uint32_t v, uint32_t d) {
  return d >= 2 || (d == 1 && D.col[D.row[v]] != v);
}

// ---- pass: chunk early-return emulation ---------------------------------------------------------
// phaseOptimizationSort.cu:46-86 / 186-240 walk the edges in chunks of STEP_ROUND and
// `return` from the whole pass at the first chunk whose copy_if selects nothing; vertices
// of that chunk and of every later chunk are not considered in that pass.
__global__ void k_chunk_flags(int dslot) {
  const Dev& D = c_dev[dslot];
  Ctrl* C = D.ctrl;
  if (blockIdx.x == 0 && threadIdx.x == 0) C->t_pass0 = global_ns();  // first kernel of a pass
  if (!C->chunk_on || !(C->fast || C->rule_sort)) return;
  const uint32_t n = C->n, it = C->it, nch = C->n_chunks;
  // chunks seen by this thread (the first 32 as bits; later ones, rare, flagged at once),
  // merged over the warp, so that a flag takes one atomic per warp instead of a read per vertex
  uint32_t seen = 0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    if (D.active_it[v] != it) continue;
    const uint32_t d = D.row[v + 1] - D.row[v];
    if (!has_nonloop(D, v, d)) continue;
    uint32_t ch = 0;
    while (ch + 1 < nch && C->chunk_lo[ch + 1] <= v) ++ch;
    if (ch < 32) seen |= 1u << ch;
    else if (!((volatile uint32_t*)C->chunk_any)[ch]) atomicOr(&C->chunk_any[ch], 1u);
  }
  seen = __reduce_or_sync(kFull, seen);
  if ((threadIdx.x & 31) == 0)
    while (seen) {
      const uint32_t ch = __ffs(seen) - 1;
      seen &= seen - 1u;
      if (!((volatile uint32_t*)C->chunk_any)[ch]) atomicOr(&C->chunk_any[ch], 1u);
    }
}

// ---- pass: degree binning of the active vertices ----------------------------------------------
// Blocks take tiles of kBinTile consecutive vertices (kBinPer per thread). A tile's bin sizes
// are summed over the block first, so that each bin's list space is claimed with one atomic
// per tile and bin (one per warp and bin contended on the eight counters and made the kernel
// atomic-bound), and the pass accounting is added once per block.
constexpr int kBinNT = 256, kBinPer = 4, kBinTile = kBinNT * kBinPer;

__global__ void __launch_bounds__(kBinNT) k_bin_vertices(int dslot, BinCfg B, int pack_ca) {
  const Dev& D = c_dev[dslot];
  Ctrl* C = D.ctrl;
  const uint32_t n = C->n, it = C->it;
  // table passes with integer weights: every vertex's (total, community) word for the gathers
  // of the gain kernels (the totals do not change before this pass's apply kernels)
  if (pack_ca && !C->fast)
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
      const uint32_t c = D.comm[v];
      D.ca[v] = ((unsigned long long)(uint32_t)D.a[c] << 32) | c;
    }
  uint32_t v_end = n;
  if (C->chunk_on && (C->fast || C->rule_sort)) {
    for (uint32_t ch = 0; ch < C->n_chunks; ++ch)
      if (!C->chunk_any[ch]) { v_end = C->chunk_lo[ch]; break; }
  }
  const bool want_off = !C->fast;
  constexpr int NW = kBinNT / 32;
  __shared__ uint32_t s_cnt[NW][kListBins];  // per warp and bin: members in this tile, then list base
  __shared__ unsigned long long s_acc[NW];
  __shared__ uint32_t s_accv[NW];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const uint32_t lt = lanemask_lt();
  unsigned long long act_e = 0;  // pass accounting for the roofline: entries and vertices binned
  uint32_t act_v = 0;
  for (uint32_t t0 = blockIdx.x * kBinTile; t0 < n; t0 += gridDim.x * kBinTile) {
    int bin[kBinPer];
    uint32_t dd[kBinPer], cap[kBinPer];
#pragma unroll
    for (int j = 0; j < kBinPer; ++j) {
      const uint32_t v = t0 + j * kBinNT + threadIdx.x;
      bin[j] = -1;
      dd[j] = 0;
      cap[j] = 0;
      if (v < v_end && D.active_it[v] == it) {
        const uint32_t g = D.gid ? D.gid[v] : 0u;
        if (D.gs[g].phase == kIterating) {
          const uint32_t d = D.row[v + 1] - D.row[v];
          if (d > 0) {
            int b = bin_of(B, d);
            // a long row whose distinct communities fit the shared table stays in bin 6
            if (b >= kNumBins - 2) {
              cap[j] = table_cap(d, D.gid ? D.gs[g].ve - D.gs[g].vb : n);
              if (b == kNumBins - 1 && cap[j] <= B.block_cap) b = kNumBins - 2;
              // a bin-6 row whose table fits half the block table: the half-block list
              if (b == kNumBins - 2 && 2u * cap[j] <= B.block_cap) b = kHalfBin;
            }
            bin[j] = b;
            dd[j] = d;
            act_e += d;
            ++act_v;
          }
        }
      }
    }
    // members per bin in this warp (lane b keeps bin b's count)
    uint32_t mine = 0;
#pragma unroll
    for (int b = 0; b < kListBins; ++b) {
      uint32_t c = 0;
#pragma unroll
      for (int j = 0; j < kBinPer; ++j) c += __popc(__ballot_sync(kFull, bin[j] == b));
      if (lane == b) mine = c;
    }
    if (lane < kListBins) s_cnt[wid][lane] = mine;
    __syncthreads();
    if (threadIdx.x < kListBins) {
      // one claim per bin for the whole tile; warps get consecutive ranges in warp order
      const int b = threadIdx.x;
      uint32_t tot = 0;
#pragma unroll
      for (int w = 0; w < NW; ++w) tot += s_cnt[w][b];
      uint32_t base = tot ? atomicAdd(&C->bin_count[b], tot) : 0u;
#pragma unroll
      for (int w = 0; w < NW; ++w) {
        const uint32_t c = s_cnt[w][b];
        s_cnt[w][b] = base;
        base += c;
      }
    }
    __syncthreads();
    uint32_t run = lane < kListBins ? s_cnt[wid][lane] : 0u;  // lane b: next position in bin b
#pragma unroll
    for (int j = 0; j < kBinPer; ++j) {
      const uint32_t v = t0 + j * kBinNT + threadIdx.x;
#pragma unroll
      for (int b = 0; b < kListBins; ++b) {
        const unsigned mask = __ballot_sync(kFull, bin[j] == b);
        if (!mask) continue;
        const uint32_t base = __shfl_sync(kFull, run, b);
        if (lane == b) run += __popc(mask);
        if (bin[j] != b) continue;
        const uint32_t pos = base + __popc(mask & lt);
        D.bins[b][pos] = v;
        if (b == kNumBins - 1) {
          // the row is cut into pieces for separate blocks; the table (table passes only) is a
          // whole number of kHubChunk-slot chunks, each chunk recording its owner
          if (want_off) {
            const uint32_t hc = cap[j] < kHubChunk ? kHubChunk : cap[j];
            const uint32_t off = atomicAdd(&C->hub_cursor, hc);
            D.hub_off[pos] = off;
            if ((unsigned long long)off + hc <= C->arena_slots)
              for (uint32_t q = 0; q < hc / kHubChunk; ++q) D.hub_owner[off / kHubChunk + q] = pos;
          }
          const uint32_t np = (dd[j] + kHubPiece - 1) / kHubPiece;
          const uint32_t p0 = atomicAdd(&C->hub_items, np);
          for (uint32_t q = 0; q < np; ++q) D.long_items[p0 + q] = ((unsigned long long)pos << 32) | q;
        }
      }
    }
    __syncthreads();  // s_cnt is rewritten by the next tile
  }
  act_e = warp_sum(act_e);
  act_v = warp_sum(act_v);
  if (lane == 0) { s_acc[wid] = act_e; s_accv[wid] = act_v; }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long e = 0;
    uint32_t nv = 0;
    for (int w = 0; w < NW; ++w) { e += s_acc[w]; nv += s_accv[w]; }
    if (nv) {
      atomicAdd(&C->act_entries, e);
      atomicAdd(&C->act_vertices, nv);
    }
  }
}

// Warp-aggregated append of movers; every lane of the warp must call it.
__device__ __forceinline__ void emit_move(const Dev& D, bool move, uint32_t v, uint32_t c,
                                          uint32_t it) {
  const unsigned mask = __ballot_sync(kFull, move);
  if (!mask) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(mask) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(&D.ctrl->mover_count, (uint32_t)__popc(mask));
  base = __shfl_sync(kFull, base, leader);
  if (move) {
    D.new_comm[v] = c;
    D.movers[base + __popc(mask & lanemask_lt())] = v;
  }
}

// A mover found by a block kernel: recorded in the hub part of the mover list, its row cut into
// pieces of kHubPiece entries for k_apply_hub.
__device__ __forceinline__ void emit_hub_move(const Dev& D, uint32_t v, uint32_t c, uint32_t it,
                                              uint32_t d) {
  Ctrl* C = D.ctrl;
  D.new_comm[v] = c;
  D.movers[C->n - 1u - atomicAdd(&C->hub_mover_count, 1u)] = v;
  const uint32_t np = (d + kHubPiece - 1) / kHubPiece;
  const uint32_t p0 = atomicAdd(&C->apply_items, np);
  for (uint32_t k = 0; k < np; ++k) D.apply_items[p0 + k] = ((unsigned long long)v << 32) | k;
}

struct VtxCtx {
  uint32_t rs, re, cv, ng;  // ng: vertices of v's graph at this level
  double kv, a_own, m, two_m2;
  double own_minus_k, inv_m, inv_2m2;  // a_own - k (the reference's first subtraction); bounds
  bool unit;                // every weight of the level is 1 (Ctrl::unit_w): w is not loaded
};

// Ctrl::unit_w as a kernel reads it once: only integer-mode kernels may take the shortcut.
template <bool WINT>
__device__ __forceinline__ bool unit_weights(const Ctrl* C) {
  return WINT && C->unit_w != 0;
}

__device__ __forceinline__ VtxCtx load_vtx(const Dev& D, uint32_t v, bool unit = false) {
  VtxCtx x;
  x.unit = unit;
  x.rs = D.row[v];
  x.re = D.row[v + 1];
  x.cv = D.comm[v];
  x.kv = D.k[v];
  x.a_own = D.a[x.cv];
  const uint32_t g = D.gid ? D.gid[v] : 0u;
  const GraphState& st = D.gs[g];
  x.m = st.m;
  x.two_m2 = st.two_m2;
  x.own_minus_k = __dsub_rn(x.a_own, x.kv);
  x.inv_m = st.inv_m;
  x.inv_2m2 = st.inv_2m2;
  x.ng = D.gid ? st.ve - st.vb : D.ctrl->n;
  return x;
}

// ---- entry loops shared by the optimisation kernels -----------------------------------------------
// Each lane walks entries e0, e0+step, ... of the vertex in groups of kBatch: it issues the
// group's independent loads (destinations, then their communities / totals) before using any,
// so a lane keeps kBatch gathers in flight instead of one dependent chain per entry.
constexpr int kBatch = 4;
// The apply kernels' gathers per lane in flight: their chains are short and register-light,
// so they take twice the optimisation kernels' depth (8 vs 4: 6 % less apply time at scale 22).
constexpr int kApplyBatch = 8;

// Fast pass: best key over positive per-entry gains (self = 0, destination's own total).
template <bool WINT>
__device__ __forceinline__ unsigned long long fast_scan(const Dev& D, const VtxCtx& x, uint32_t v,
                                                        uint32_t e0, uint32_t step) {
  using Tr = WTraits<WINT>;
  using Wt = typename Tr::W;
  const Wt* __restrict__ w = reinterpret_cast<const Wt*>(D.w);
  unsigned long long best = 0;
  for (uint32_t e = e0; e < x.re; e += kBatch * step) {
    uint32_t uu[kBatch];
    float wf[kBatch];
    double au[kBatch];
#pragma unroll
    for (int k = 0; k < kBatch; ++k) {
      const uint32_t ek = e + k * step;
      const bool in = ek < x.re;
      uu[k] = in ? D.col[ek] : v;
      wf[k] = in ? (x.unit ? 1.0f : Tr::w_float(w[ek])) : 0.0f;
    }
#pragma unroll
    for (int k = 0; k < kBatch; ++k) au[k] = uu[k] != v ? D.a[uu[k]] : 0.0;
#pragma unroll
    for (int k = 0; k < kBatch; ++k) {
      if (uu[k] == v) continue;
      // self = 0: diff = w - 0 = w exactly
      const double p = gain_p(x.kv, x.own_minus_k, au[k]);
      const float g = gain_fast(wf[k], p, x.inv_m, x.inv_2m2, x.m, x.two_m2);
      if (g > 0.0f) {
        const unsigned long long key = argmax_key(g, uu[k], true);
        if (key > best) best = key;
      }
    }
  }
  return best;
}

// Table pass, insert half: non-loop entries into the table by destination community, the
// vertex's own community summed into self_acc.
template <bool WINT, class Tbl>
__device__ __forceinline__ void insert_scan(const Dev& D, const VtxCtx& x, uint32_t v, uint32_t e0,
                                            uint32_t step, const Tbl& tbl,
                                            typename WTraits<WINT>::Acc& self_acc, uint32_t& err) {
  using Tr = WTraits<WINT>;
  using Acc = typename Tr::Acc;
  using Wt = typename Tr::W;
  const Wt* __restrict__ w = reinterpret_cast<const Wt*>(D.w);
  for (uint32_t e = e0; e < x.re; e += kBatch * step) {
    uint32_t uu[kBatch], cc[kBatch];
    Acc ww[kBatch];
#pragma unroll
    for (int k = 0; k < kBatch; ++k) {
      const uint32_t ek = e + k * step;
      const bool in = ek < x.re;
      uu[k] = in ? D.col[ek] : v;
      ww[k] = in ? (x.unit ? Acc(1) : (Acc)w[ek]) : Acc(0);
    }
#pragma unroll
    for (int k = 0; k < kBatch; ++k) cc[k] = uu[k] != v ? D.comm[uu[k]] : kEmpty;
#pragma unroll
    for (int k = 0; k < kBatch; ++k) {
      if (cc[k] == kEmpty) continue;
      if (cc[k] == x.cv) { self_acc += ww[k]; continue; }
      if (!tbl.add(cc[k], ww[k])) err |= kErrTableFull;
    }
  }
}

// Table pass, evaluation half: best key over the table's communities (slots s0, s0+step, ...).
template <bool WINT, class Tbl>
__device__ __forceinline__ unsigned long long cand_scan(const Dev& D, const VtxCtx& x, const Tbl& tbl,
                                                        uint32_t s0, uint32_t cap, uint32_t step,
                                                        float self_v, bool lowest) {
  using Tr = WTraits<WINT>;
  using Acc = typename Tr::Acc;
  unsigned long long best = 0;
  for (uint32_t s = s0; s < cap; s += kBatch * step) {
    uint32_t cc[kBatch];
    Acc vv[kBatch];
    double ac[kBatch];
#pragma unroll
    for (int k = 0; k < kBatch; ++k) {
      const uint32_t sk = s + k * step;
      cc[k] = kEmpty;
      vv[k] = Acc(0);
      if (sk < cap) tbl.load(sk, cc[k], vv[k]);
      if (cc[k] == x.cv) cc[k] = kEmpty;
    }
#pragma unroll
    for (int k = 0; k < kBatch; ++k) ac[k] = cc[k] != kEmpty ? D.a[cc[k]] : 0.0;
#pragma unroll
    for (int k = 0; k < kBatch; ++k) {
      if (cc[k] == kEmpty) continue;
      const float diff = __fsub_rn(Tr::to_float(vv[k]), self_v);
      const double p = gain_p(x.kv, x.own_minus_k, ac[k]);
      const float g = gain_fast(diff, p, x.inv_m, x.inv_2m2, x.m, x.two_m2);
      if (g > 0.0f) {
        const unsigned long long key = argmax_key(g, cc[k], lowest);
        if (key > best) best = key;
      }
    }
  }
  return best;
}

// Table pass with a key list: the insert half also records, for every community it creates in
// the table, the slot it sits in, so that the evaluation half reads only those slots (the
// distinct neighbouring communities) instead of scanning the whole table, and empties only
// them again -- a table is cleared once when a kernel starts and stays empty between vertices.
// The list has room for min(d, ng) slots, half the table's capacity, as u16 indices.
//
// Insert half. The entries of the row are walked in team-uniform steps (every lane of the team
// takes the same number of steps, lanes past the row's end carry nothing), so the lanes that
// created a key can agree on their list positions with one ballot per entry batch. `tmask` is
// the team's lanes within the warp. BLOCK: the team is the whole block; warps take list space
// from the shared counter *bcount (one atomic per warp and batch), which the caller reads after
// a barrier. Otherwise the team is part of one warp and the count is returned.
// With integer weights (WINT) each entry gathers its neighbour's (total, community) word
// (Dev::ca) instead of the community alone, and the lane that creates a key also lists the
// community's total (`lista`, beside the slot index), so that the evaluation half reads no
// global memory at all.
template <bool WINT, bool BLOCK, int NB, class Tbl>
__device__ __forceinline__ uint32_t insert_list(const Dev& D, const VtxCtx& x, uint32_t v, uint32_t lane,
                                                uint32_t step, unsigned tmask, const Tbl& tbl,
                                                uint16_t* list, uint32_t* lista, uint32_t* bcount,
                                                typename WTraits<WINT>::Acc& self_acc, uint32_t& err) {
  using Tr = WTraits<WINT>;
  using Acc = typename Tr::Acc;
  using Wt = typename Tr::W;
  const Wt* __restrict__ w = reinterpret_cast<const Wt*>(D.w);
  const uint32_t lt = lanemask_lt();
  uint32_t nl = 0;
  for (uint32_t b = x.rs; b < x.re; b += NB * step) {
    uint32_t uu[NB], cc[NB], at[NB];
    Acc ww[NB];
#pragma unroll
    for (int k = 0; k < NB; ++k) {
      const uint32_t ek = b + lane + k * step;
      const bool in = ek < x.re;
      uu[k] = in ? D.col[ek] : v;
      ww[k] = in ? (x.unit ? Acc(1) : (Acc)w[ek]) : Acc(0);
    }
#pragma unroll
    for (int k = 0; k < NB; ++k) {
      if constexpr (WINT) {
        const unsigned long long y = uu[k] != v ? D.ca[uu[k]] : 0xFFFFFFFFFFFFFFFFull;
        cc[k] = (uint32_t)y;
        at[k] = (uint32_t)(y >> 32);
      } else {
        cc[k] = uu[k] != v ? D.comm[uu[k]] : kEmpty;
        at[k] = 0;
      }
    }
#pragma unroll
    for (int k = 0; k < NB; ++k) {
      bool made = false;
      uint32_t slot = 0;
      if (cc[k] != kEmpty) {
        if (cc[k] == x.cv) {
          self_acc += ww[k];
        } else {
          const int r = tbl.template add_at<true>(cc[k], ww[k], slot);
          if (!r) err |= kErrTableFull;
          made = r == 2;
        }
      }
      const unsigned m = __ballot_sync(tmask, made) & tmask;
      if (BLOCK) {
        if (m) {
          const int leader = __ffs(m) - 1;
          uint32_t base = 0;
          if ((int)(threadIdx.x & 31) == leader) base = atomicAdd(bcount, (uint32_t)__popc(m));
          base = __shfl_sync(kFull, base, leader);
          if (made) {
            list[base + __popc(m & lt)] = (uint16_t)slot;
            if constexpr (WINT) lista[base + __popc(m & lt)] = at[k];
          }
        }
      } else {
        if (made) {
          list[nl + __popc(m & lt)] = (uint16_t)slot;
          if constexpr (WINT) lista[nl + __popc(m & lt)] = at[k];
        }
        nl += __popc(m);
      }
    }
  }
  return nl;
}

// Evaluation half over the listed slots [i0, nl) with stride `step`: best key over the
// distinct neighbouring communities (as cand_scan), emptying each slot after reading it.
template <bool WINT, int NB, class Tbl>
__device__ __forceinline__ unsigned long long list_scan(const Dev& D, const VtxCtx& x, const Tbl& tbl,
                                                        const uint16_t* list, const uint32_t* lista,
                                                        uint32_t i0, uint32_t nl,
                                                        uint32_t step, float self_v, bool lowest) {
  using Tr = WTraits<WINT>;
  using Acc = typename Tr::Acc;
  unsigned long long best = 0;
  for (uint32_t i = i0; i < nl; i += NB * step) {
    uint32_t cc[NB];
    Acc vv[NB];
    double ac[NB];
#pragma unroll
    for (int k = 0; k < NB; ++k) {
      const uint32_t ik = i + k * step;
      cc[k] = kEmpty;
      vv[k] = Acc(0);
      ac[k] = 0.0;
      if (ik < nl) {
        const uint32_t sl = list[ik];
        tbl.load(sl, cc[k], vv[k]);
        tbl.clear(sl);
        if constexpr (WINT) ac[k] = (double)lista[ik];
      }
      if (cc[k] == x.cv) cc[k] = kEmpty;
    }
    if constexpr (!WINT) {
#pragma unroll
      for (int k = 0; k < NB; ++k) ac[k] = cc[k] != kEmpty ? D.a[cc[k]] : 0.0;
    }
#pragma unroll
    for (int k = 0; k < NB; ++k) {
      if (cc[k] == kEmpty) continue;
      const float diff = __fsub_rn(Tr::to_float(vv[k]), self_v);
      const double p = gain_p(x.kv, x.own_minus_k, ac[k]);
      const float g = gain_fast(diff, p, x.inv_m, x.inv_2m2, x.m, x.two_m2);
      if (g > 0.0f) {
        const unsigned long long key = argmax_key(g, cc[k], lowest);
        if (key > best) best = key;
      }
    }
  }
  return best;
}

// Entries per thread and step for a row of d entries over `lanes` lanes: as many as the row
// needs, up to kBatch (unused batch slots still cost their instructions).
__device__ __forceinline__ int batch_for(uint32_t d, uint32_t lanes) {
  return d <= lanes ? 1 : (d <= 2u * lanes ? 2 : kBatch);
}

// ---- pass: optimisation, one team of T lanes per vertex -----------------------------------------
// Fast pass (iteration 0 of a level, phaseOptimizationSort.cu:28-158): per-entry gains with
// self = 0 and the destination's own (singleton) community, argmax over positive gains with
// the lowest community winning ties, then the v <= c gate (phaseOptimizationUpdate.cu:99).
// Other passes (phaseOptimizationSort.cu:161-379 / phaseOptimizationHash.cu:38-162): exact
// per-community sums of non-loop weights in a shared-memory hash table sized 2x the degree,
// self_v = sum into the vertex's own community, gains for every other neighbouring
// community, argmax with the mode's tie rule. Only positive gains can move a vertex, so only
// they enter the argmax (the reference's own-community and negative candidates can never
// win a move).
template <int T, bool WINT>
__global__ void __launch_bounds__(256, 4) k_opt_team(int dslot, int bin, uint32_t cap) {
  const Dev& D = c_dev[dslot];
  using Tr = WTraits<WINT>;
  using Acc = typename Tr::Acc;
  constexpr int TEAMS = 256 / T;
  extern __shared__ __align__(16) unsigned char smem[];
  const int team = threadIdx.x / T, lane = threadIdx.x % T;
  // per team: a table of `cap` slots (packed u64, or u32 keys + sums), a list of cap / 2 u16
  // slot indices (table capacities stay below 2^16: they must fit shared memory) and, with
  // integer weights, the cap / 2 listed communities' totals (u32)
  constexpr size_t kSlotBytes = WINT ? 8 : 4 + sizeof(Acc);
  uint32_t* keys = reinterpret_cast<uint32_t*>(smem) + (size_t)team * cap;
  Acc* vals = reinterpret_cast<Acc*>(smem + (size_t)TEAMS * cap * sizeof(uint32_t)) + (size_t)team * cap;
  unsigned long long* slots = reinterpret_cast<unsigned long long*>(smem) + (size_t)team * cap;
  uint16_t* list = reinterpret_cast<uint16_t*>(smem + (size_t)TEAMS * cap * kSlotBytes) + (size_t)team * (cap / 2);
  // integer weights: the listed communities' totals, cap / 2 u32 per team after the lists
  uint32_t* lista = reinterpret_cast<uint32_t*>(smem + (size_t)TEAMS * cap * (kSlotBytes + 1)) + (size_t)team * (cap / 2);

  Ctrl* C = D.ctrl;
  const uint32_t count = C->bin_count[bin];
  if (blockIdx.x * TEAMS >= count) return;  // (block-uniform)
  const uint32_t* vlist = D.bins[bin];
  const uint32_t it = C->it;
  const bool fast = C->fast != 0;
  const bool lowest = fast || C->rule_sort != 0;
  const bool unit = unit_weights<WINT>(C);
  const unsigned tmask = T == 32 ? kFull : (((1u << T) - 1u) << ((threadIdx.x & 31) & ~(uint32_t)(T - 1)));
  uint32_t err = 0;
  ScratchTable<WINT> tbl{keys, vals, slots, cap - 1u, 0u};
  if (!fast) {
    for (uint32_t s = lane; s < cap; s += T) tbl.clear(s);
    __syncwarp();
  }

  for (uint32_t base = blockIdx.x * TEAMS; base < count; base += gridDim.x * TEAMS) {
    const uint32_t idx = base + team;
    const bool live = idx < count;
    const uint32_t v = live ? vlist[idx] : 0u;
    VtxCtx x{};
    if (live) x = load_vtx(D, v, unit);
    unsigned long long best = 0;
    if (fast) {
      if (live) best = fast_scan<WINT>(D, x, v, x.rs + lane, T);
      best = team_max<T>(best, kFull);
    } else {
      const uint32_t cap_v = live ? table_cap(x.re - x.rs, x.ng) : 2u;
      tbl.mask = cap_v - 1u;
      tbl.shift = 32u - log2_pow2(cap_v);
      // weight into the vertex's own community stays in registers (it is the hottest key)
      Acc self_acc = Acc(0);
      uint32_t nl = 0;
      // entries per lane and step as the row needs (team-uniform choice): unused batch slots
      // still cost their instructions
      const int nb = batch_for(x.re - x.rs, T);
      if (live) {
        if (nb == 1) nl = insert_list<WINT, false, 1>(D, x, v, lane, T, tmask, tbl, list, lista, nullptr, self_acc, err);
        else if (nb == 2) nl = insert_list<WINT, false, 2>(D, x, v, lane, T, tmask, tbl, list, lista, nullptr, self_acc, err);
        else nl = insert_list<WINT, false, kBatch>(D, x, v, lane, T, tmask, tbl, list, lista, nullptr, self_acc, err);
      }
      self_acc = team_sum<T>(self_acc);
      __syncwarp();
      if (live) {
        const float self_v = Tr::to_float(self_acc);
        if (nb == 1) best = list_scan<WINT, 1>(D, x, tbl, list, lista, lane, nl, T, self_v, lowest);
        else if (nb == 2) best = list_scan<WINT, 2>(D, x, tbl, list, lista, lane, nl, T, self_v, lowest);
        else best = list_scan<WINT, kBatch>(D, x, tbl, list, lista, lane, nl, T, self_v, lowest);
      }
      best = team_max<T>(best, kFull);
      __syncwarp();  // the listed slots are empty again before the next vertex inserts
    }
    bool move = false;
    uint32_t c = 0;
    if (live && lane == 0 && best) {
      c = key_comm(best, lowest);
      move = c != x.cv && (!fast || v <= c);
    }
    emit_move(D, move, v, c, it);
  }
  if (err) report_err(C, err, 0);  // k_opt_team
}

// Block-wide sum (all threads call; result valid in every thread; `sh` holds >= 33 values).
// The reduction tree is fixed, so a double sum is the same on every run.
template <int NT, class V>
__device__ __forceinline__ V block_sum(V x, V* sh) {
  x = warp_sum(x);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = x;
  __syncthreads();
  if (wid == 0) {
    V y = lane < NT / 32 ? sh[lane] : V(0);
    y = warp_sum(y);
    if (lane == 0) sh[32] = y;
  }
  __syncthreads();
  const V r = sh[32];
  __syncthreads();
  return r;
}

// Block-wide max of a u64 (all threads call; result valid in every thread).
template <int NT>
__device__ __forceinline__ unsigned long long block_max(unsigned long long x, unsigned long long* sh) {
  x = team_max<32>(x, kFull);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = x;
  __syncthreads();
  if (wid == 0) {
    unsigned long long y = lane < NT / 32 ? sh[lane] : 0ull;
    y = team_max<32>(y, kFull);
    if (lane == 0) sh[32] = y;
  }
  __syncthreads();
  const unsigned long long r = sh[32];
  __syncthreads();
  return r;
}

// ---- pass: optimisation, one block per high-degree vertex ----------------------------------------
// The vertex's table lives in shared memory (capacity `cap` slots; vertices whose table would
// not fit are in bin 7, handled by the k_opt_hub_* kernels).
// NT threads per block: 512 for bin 6, 256 for the half-block list (tables of half the size, so
// twice as many blocks fit an SM's shared memory and registers).
template <bool WINT, int NT = 512>
__global__ void __launch_bounds__(NT, 1024 / NT) k_opt_block(int dslot, int bin, uint32_t cap) {
  const Dev& D = c_dev[dslot];
  using Tr = WTraits<WINT>;
  using Acc = typename Tr::Acc;
  constexpr int NW = NT / 32;
  extern __shared__ __align__(16) unsigned char smem[];
  // per-warp partials and the list count, double-buffered by vertex parity so that a vertex
  // needs two barriers (table pass) or one (fast pass): one before the keys are evaluated,
  // one before warp 0 reads the per-warp best keys
  __shared__ unsigned long long red_best[2][NW];
  __shared__ Acc red_self[2][NW];
  __shared__ uint32_t nlist[2];
  // a table of `cap` slots (packed u64, or u32 keys + sums), a list of cap / 2 u16 slot indices
  // and, with integer weights, the listed communities' totals (cap / 2 u32)
  constexpr size_t kSlotBytes = WINT ? 8 : 4 + sizeof(Acc);
  uint32_t* keys = reinterpret_cast<uint32_t*>(smem);
  Acc* vals = reinterpret_cast<Acc*>(smem + (size_t)cap * sizeof(uint32_t));
  unsigned long long* slots = reinterpret_cast<unsigned long long*>(smem);
  uint16_t* list = reinterpret_cast<uint16_t*>(smem + (size_t)cap * kSlotBytes);
  uint32_t* lista = reinterpret_cast<uint32_t*>(smem + (size_t)cap * (kSlotBytes + 1));  // integer weights
  Ctrl* C = D.ctrl;
  const uint32_t count = C->bin_count[bin];
  if (blockIdx.x >= count) return;  // (block-uniform)
  const uint32_t* vlist = D.bins[bin];
  const uint32_t it = C->it;
  const bool fast = C->fast != 0;
  const bool lowest = fast || C->rule_sort != 0;
  const bool unit = unit_weights<WINT>(C);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t err = 0;
  ScratchTable<WINT> tbl{keys, vals, slots, cap - 1u, 0u};
  if (!fast)
    for (uint32_t s = threadIdx.x; s < cap; s += NT) tbl.clear(s);
  if (threadIdx.x < 2) nlist[threadIdx.x] = 0;
  __syncthreads();

  int par = 0;
  for (uint32_t idx = blockIdx.x; idx < count; idx += gridDim.x, par ^= 1) {
    const uint32_t v = vlist[idx];
    const VtxCtx x = load_vtx(D, v, unit);
    const uint32_t d = x.re - x.rs;
    const int nb = batch_for(d, NT);
    unsigned long long best = 0;
    if (fast) {
      best = fast_scan<WINT>(D, x, v, x.rs + threadIdx.x, NT);
    } else {
      const uint32_t cap_v = table_cap(d, x.ng);
      const bool ok = cap_v <= cap;
      if (!ok) err |= kErrArena;
      tbl.mask = cap_v - 1u;
      tbl.shift = 32u - log2_pow2(cap_v);
      Acc self_acc = Acc(0);  // the own community's weight, kept out of the table
      if (ok) {
        if (nb == 1) insert_list<WINT, true, 1>(D, x, v, threadIdx.x, NT, kFull, tbl, list, lista, &nlist[par], self_acc, err);
        else if (nb == 2) insert_list<WINT, true, 2>(D, x, v, threadIdx.x, NT, kFull, tbl, list, lista, &nlist[par], self_acc, err);
        else insert_list<WINT, true, kBatch>(D, x, v, threadIdx.x, NT, kFull, tbl, list, lista, &nlist[par], self_acc, err);
      }
      self_acc = warp_sum(self_acc);
      if (lane == 0) red_self[par][wid] = self_acc;
      __syncthreads();  // the table and the list are complete
      Acc self_all = Acc(0);
#pragma unroll
      for (int i = 0; i < NW; ++i) self_all += red_self[par][i];  // fixed order
      const uint32_t nl = nlist[par];
      const float self_v = Tr::to_float(self_all);
      if (ok) {
        if (nb == 1) best = list_scan<WINT, 1>(D, x, tbl, list, lista, threadIdx.x, nl, NT, self_v, lowest);
        else if (nb == 2) best = list_scan<WINT, 2>(D, x, tbl, list, lista, threadIdx.x, nl, NT, self_v, lowest);
        else best = list_scan<WINT, kBatch>(D, x, tbl, list, lista, threadIdx.x, nl, NT, self_v, lowest);
      }
      if (threadIdx.x == 0) nlist[par ^ 1] = 0;  // the next vertex's count (read by no one now)
    }
    best = team_max<32>(best, kFull);
    if (lane == 0) red_best[par][wid] = best;
    __syncthreads();  // every key is evaluated and every listed slot empty again
    if (wid == 0) {
      unsigned long long y = lane < NW ? red_best[par][lane] : 0ull;
      y = team_max<32>(y, kFull);
      if (lane == 0 && y) {
        const uint32_t c = key_comm(y, lowest);
        if (c != x.cv && (!fast || v <= c)) emit_hub_move(D, v, c, it, d);
      }
    }
  }
  if (err) report_err(C, err, 1);  // k_opt_block
}

// ---- pass: optimisation of the longest rows (bin 7), many blocks per vertex ------------------------
// Each bin-7 row is cut into pieces of kHubPiece entries (k_bin_vertices listed them in
// long_items); pieces are scanned by separate blocks into the vertex's global table, the table is
// evaluated chunk by chunk by separate blocks, and the per-vertex argmax key is merged with
// atomicMax (map[] holds it during a pass; the own-community weight goes to hubself[]).
// Global tables are packed (key << 32 | sum) with integer weights, split arrays with fp32 ones.
template <bool WINT>
__device__ __forceinline__ void arena_clear_slot(const Dev& D, uint32_t s) {
  unsigned long long* vals = reinterpret_cast<unsigned long long*>(D.arena_vals);
  if (WINT) {
    vals[s] = kEmptySlot;
  } else {
    D.arena_keys[s] = kEmpty;
    vals[s] = 0ull;
  }
}

template <bool WINT>
__global__ void k_opt_hub_prep(int dslot) {
  const Dev& D = c_dev[dslot];
  Ctrl* C = D.ctrl;
  const uint32_t count = C->bin_count[kNumBins - 1];
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  for (uint32_t i = tid; i < count; i += nth) {
    D.map[i] = 0ull;
    D.hubself[i] = 0ull;
  }
  if (!C->fast) {
    const uint32_t slots = min(C->hub_cursor, C->arena_slots);
    for (uint32_t s = tid; s < slots; s += nth) arena_clear_slot<WINT>(D, s);
  }
}

template <bool WINT>
__global__ void __launch_bounds__(256) k_opt_hub_scan(int dslot) {
  const Dev& D = c_dev[dslot];
  using Tr = WTraits<WINT>;
  using Acc = typename Tr::Acc;
  __shared__ unsigned long long red[33];
  Ctrl* C = D.ctrl;
  const uint32_t count = C->hub_items;
  const bool fast = C->fast != 0;
  const bool unit = unit_weights<WINT>(C);
  uint32_t err = 0;
  for (uint32_t i = blockIdx.x; i < count; i += gridDim.x) {
    const unsigned long long item = D.long_items[i];
    const uint32_t pos = (uint32_t)(item >> 32), piece = (uint32_t)item;
    const uint32_t v = D.bins[kNumBins - 1][pos];
    VtxCtx x = load_vtx(D, v, unit);
    const uint32_t d = x.re - x.rs;
    const uint32_t pstart = x.rs + piece * kHubPiece;
    x.re = min(x.re, pstart + kHubPiece);
    if (fast) {
      unsigned long long best = fast_scan<WINT>(D, x, v, pstart + threadIdx.x, blockDim.x);
      best = block_max<256>(best, red);
      if (threadIdx.x == 0 && best) atomicMax(&D.map[pos], best);
    } else {
      const uint32_t cap = hub_table_cap(d, x.ng);
      const uint32_t off = D.hub_off[pos];
      const bool ok = (unsigned long long)off + cap <= C->arena_slots;
      if (!ok) err |= kErrArena;
      Acc self_acc = Acc(0);
      if (ok) {
        if constexpr (WINT) {
          const PackedTable tbl{reinterpret_cast<unsigned long long*>(D.arena_vals) + off, cap - 1u,
                                32u - log2_pow2(cap)};
          insert_scan<WINT>(D, x, v, pstart + threadIdx.x, blockDim.x, tbl, self_acc, err);
        } else {
          const SplitTable<Acc> tbl{D.arena_keys + off, reinterpret_cast<Acc*>(D.arena_vals) + off,
                                    cap - 1u, 32u - log2_pow2(cap)};
          insert_scan<WINT>(D, x, v, pstart + threadIdx.x, blockDim.x, tbl, self_acc, err);
        }
      }
      self_acc = block_sum<256>(self_acc, reinterpret_cast<Acc*>(red));
      if (threadIdx.x == 0 && self_acc != Acc(0)) {
        if (WINT) atomicAdd(&D.hubself[pos], (unsigned long long)self_acc);
        else atomicAdd(reinterpret_cast<double*>(&D.hubself[pos]), (double)self_acc);
      }
    }
  }
  if (err) report_err(C, err, 2);  // k_opt_hub_scan
}

template <bool WINT>
__global__ void __launch_bounds__(256) k_opt_hub_eval(int dslot) {
  const Dev& D = c_dev[dslot];
  using Tr = WTraits<WINT>;
  using Acc = typename Tr::Acc;
  __shared__ unsigned long long red[33];
  Ctrl* C = D.ctrl;
  if (C->fast) return;
  const bool lowest = C->rule_sort != 0;
  const uint32_t nchunks = min(C->hub_cursor, C->arena_slots) / kHubChunk;
  const Acc* vals = reinterpret_cast<const Acc*>(D.arena_vals);
  for (uint32_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
    const uint32_t pos = D.hub_owner[c];
    const uint32_t v = D.bins[kNumBins - 1][pos];
    const VtxCtx x = load_vtx(D, v);
    const unsigned long long hs = D.hubself[pos];
    float self_v;
    if (WINT) self_v = Tr::to_float((Acc)hs);
    else self_v = Tr::to_float((Acc)__longlong_as_double((long long)hs));
    unsigned long long best;
    if constexpr (WINT) {
      const PackedTable tbl{reinterpret_cast<unsigned long long*>(D.arena_vals), 0u, 0u};
      best = cand_scan<WINT>(D, x, tbl, c * kHubChunk + threadIdx.x, (c + 1) * kHubChunk, blockDim.x,
                             self_v, lowest);
    } else {
      const SplitTable<Acc> tbl{D.arena_keys, const_cast<Acc*>(vals), 0u, 0u};
      best = cand_scan<WINT>(D, x, tbl, c * kHubChunk + threadIdx.x, (c + 1) * kHubChunk, blockDim.x,
                             self_v, lowest);
    }
    best = block_max<256>(best, red);
    if (threadIdx.x == 0 && best) atomicMax(&D.map[pos], best);
  }
}

__global__ void k_opt_hub_decide(int dslot) {
  const Dev& D = c_dev[dslot];
  Ctrl* C = D.ctrl;
  const uint32_t count = C->bin_count[kNumBins - 1], it = C->it;
  const bool fast = C->fast != 0;
  const bool lowest = fast || C->rule_sort != 0;
  for (uint32_t pos = blockIdx.x * blockDim.x + threadIdx.x; pos < count; pos += gridDim.x * blockDim.x) {
    const unsigned long long best = D.map[pos];
    if (!best) continue;
    const uint32_t v = D.bins[kNumBins - 1][pos];
    const uint32_t c = key_comm(best, lowest);
    if (c != D.comm[v] && (!fast || v <= c)) emit_hub_move(D, v, c, it, D.row[v + 1] - D.row[v]);
  }
}

// ---- pass: apply the moves, propagate activity, update the internal weight ---------------------
// update_value_kernel_* (phaseOptimizationUpdate.cu:14-115): totals of the old and new
// community change by -/+ k_v with double atomics (integer-valued, so exact and
// order-independent). update_changed_kernel (:117-132) -- "src is active next pass iff some
// neighbour dst moved and comm[dst] != comm[src]" -- is evaluated by pushing from each mover
// to its neighbours, which the symmetric CSR makes identical. The internal weight of
// community.h:87-100 is kept incrementally: each directed entry (v,u) touching a mover
// changes by w([post_v == post_u] - [pre_v == pre_u]); the mirror entry (u,v) is counted here
// too when u did not move (factor 2).
// Entries [e0, re) with stride `step` of mover v (old -> nw): activity push and the mover's
// share of the internal-weight change.
template <bool WINT>
__device__ __forceinline__ void apply_entries(const Dev& D, uint32_t v, uint32_t old, uint32_t nw,
                                              uint32_t it, uint32_t e0, uint32_t re, uint32_t step,
                                              bool unit, long long& di, double& df) {
  using Tr = WTraits<WINT>;
  using Wt = typename Tr::W;
  const Wt* __restrict__ w = reinterpret_cast<const Wt*>(D.w);
  // kApplyBatch entries per lane at a time: their gathers are issued before any is used
  for (uint32_t e = e0; e < re; e += kApplyBatch * step) {
    uint32_t uu[kApplyBatch], pre[kApplyBatch], nc[kApplyBatch];
#pragma unroll
    for (int k = 0; k < kApplyBatch; ++k) {
      const uint32_t ek = e + k * step;
      uu[k] = ek < re ? D.col[ek] : kEmpty;
    }
#pragma unroll
    for (int k = 0; k < kApplyBatch; ++k) {
      const unsigned long long x = uu[k] != kEmpty ? D.cn[uu[k]] : 0ull;
      pre[k] = (uint32_t)x;
      nc[k] = (uint32_t)(x >> 32);
    }
#pragma unroll
    for (int k = 0; k < kApplyBatch; ++k) {
      if (uu[k] == kEmpty) continue;
      const uint32_t u = uu[k];
      // new_comm equals comm for every vertex that did not move this pass
      const bool mu = nc[k] != pre[k];
      const uint32_t post = nc[k];
      if (post != nw) D.active_it[u] = it + 1;
      const int dd = (int)(nw == post) - (int)(old == pre[k]);
      if (dd) {
        const uint32_t ek = e + k * step;
        const int f = mu ? dd : 2 * dd;
        if (WINT) di += (long long)f * (unit ? 1ll : (long long)w[ek]);
        else df += (double)f * Tr::w_double(w[ek]);
      }
    }
  }
}

// Movers found by the team kernels, 32 per warp (one per lane): the warp walks the entries of
// all 32 rows together -- lane i takes entries i, i+32, ... of the concatenated rows, kApplyBatch at
// a time -- so every lane is busy and keeps kApplyBatch independent gathers in flight however short
// the rows are (most movers have a handful of entries). Rows longer than kApplyShort are left
// to k_apply_long (a warp each; movers sit in the list grouped by degree, so a warp taking 32
// long rows would hold up the whole kernel). An entry's change of the internal weight goes to
// its own graph, which is the mover's (edges never cross graphs).
// Before the apply kernels: each vertex's pre-pass community and this pass's target packed
// in one word, so that an entry costs one 8-byte gather instead of two 4-byte ones.
__global__ void k_pack_cn(int dslot) {
  const Dev& D = c_dev[dslot];
  const uint32_t n = D.ctrl->n;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    D.cn[v] = ((unsigned long long)D.new_comm[v] << 32) | D.comm[v];
}

constexpr uint32_t kApplyShort = 32;

template <bool WINT>
__global__ void __launch_bounds__(256) k_apply(int dslot) {
  const Dev& D = c_dev[dslot];
  using Tr = WTraits<WINT>;
  using Wt = typename Tr::W;
  const Wt* __restrict__ w = reinterpret_cast<const Wt*>(D.w);
  Ctrl* C = D.ctrl;
  // the optimisation kernels of this pass ended when the first apply block starts
  if (blockIdx.x == 0 && threadIdx.x == 0) C->t_optk_ns += global_ns() - C->t_pass0;
  const uint32_t count = C->mover_count, it = C->it;
  const bool unit = unit_weights<WINT>(C);
  const int lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  uint32_t gcur = 0;  // graph of the running internal-weight change
  long long di = 0;
  double df = 0.0;
  auto flush = [&]() {
    if (WINT) {
      if (di) atomicAdd(&D.gs[gcur].I, (unsigned long long)di);
    } else if (df != 0.0) {
      atomicAdd(reinterpret_cast<double*>(&D.gs[gcur].I), df);
    }
    di = 0;
    df = 0.0;
  };
  for (uint32_t base = warp * 32u; base < count; base += nwarps * 32u) {
    const uint32_t idx = base + lane;
    uint32_t rs = 0, len = 0, old = 0, nw = 0, v = 0;
    if (idx < count) {
      v = D.movers[idx];
      old = D.comm[v];
      nw = D.new_comm[v];
      // a refinement pass leaves rejected proposals in the list with new_comm == comm
      if (nw != old) {
        rs = D.row[v];
        len = D.row[v + 1] - rs;
        const double kv = D.k[v];
        atomicAdd(&D.a[nw], kv);
        atomicAdd(&D.a[old], -kv);
      }
    }
    // long rows: queued for k_apply_long (the list lives in `members`, unused during passes)
    const bool defer = len > kApplyShort;
    const unsigned dm = __ballot_sync(kFull, defer);
    if (dm) {
      uint32_t b0 = 0;
      if (lane == __ffs(dm) - 1) b0 = atomicAdd(&C->long_movers, (uint32_t)__popc(dm));
      b0 = __shfl_sync(kFull, b0, __ffs(dm) - 1);
      if (defer) D.members[b0 + __popc(dm & lanemask_lt())] = v;
    }
    if (defer) len = 0;
    uint32_t incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += y;
    }
    const uint32_t total = __shfl_sync(kFull, incl, 31);
    const uint32_t excl = incl - len;
    for (uint32_t jb = 0; jb < total; jb += 32u * kApplyBatch) {
      uint32_t ee[kApplyBatch], oo[kApplyBatch], nn[kApplyBatch], uu[kApplyBatch], pre[kApplyBatch], nc[kApplyBatch];
#pragma unroll
      for (int q = 0; q < kApplyBatch; ++q) {
        const uint32_t j = jb + (uint32_t)q * 32u + lane;
        int k = 0;  // owner: the last lane whose row starts at or before j
#pragma unroll
        for (int step = 16; step >= 1; step >>= 1) {
          const uint32_t ex = __shfl_sync(kFull, excl, k + step);
          if (ex <= j) k += step;
        }
        ee[q] = __shfl_sync(kFull, rs, k) + (j - __shfl_sync(kFull, excl, k));
        oo[q] = __shfl_sync(kFull, old, k);
        nn[q] = __shfl_sync(kFull, nw, k);
        uu[q] = j < total ? D.col[ee[q]] : kEmpty;
      }
#pragma unroll
      for (int q = 0; q < kApplyBatch; ++q) {
        const unsigned long long x = uu[q] != kEmpty ? D.cn[uu[q]] : 0ull;
        pre[q] = (uint32_t)x;
        nc[q] = (uint32_t)(x >> 32);
      }
#pragma unroll
      for (int q = 0; q < kApplyBatch; ++q) {
        if (uu[q] == kEmpty) continue;
        const uint32_t u = uu[q];
        const bool mu = nc[q] != pre[q];  // new_comm equals comm unless u moved this pass
        const uint32_t post = nc[q];
        if (post != nn[q]) D.active_it[u] = it + 1;
        const int dd = (int)(nn[q] == post) - (int)(oo[q] == pre[q]);
        if (dd) {
          const int f = mu ? dd : 2 * dd;
          if (D.gid) {
            const uint32_t g = D.gid[u];
            if (g != gcur) {
              flush();
              gcur = g;
            }
          }
          if (WINT) di += (long long)f * (unit ? 1ll : (long long)w[ee[q]]);
          else df += (double)f * Tr::w_double(w[ee[q]]);
        }
      }
    }
  }
  if (!D.gid) {
    // one graph: a single sum per warp
    di = warp_sum(di);
    df = warp_sum(df);
    if (lane == 0) flush();
  } else {
    flush();
  }
}

// The team kernels' movers with rows longer than kApplyShort (queued by k_apply, which also
// moved their totals): one warp per mover, kApplyBatch gathers in flight per lane.
template <bool WINT>
__global__ void __launch_bounds__(256) k_apply_long(int dslot) {
  const Dev& D = c_dev[dslot];
  Ctrl* C = D.ctrl;
  const uint32_t count = C->long_movers, it = C->it;
  const bool unit = unit_weights<WINT>(C);
  const int lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t idx = warp; idx < count; idx += nwarps) {
    const uint32_t v = D.members[idx];
    const uint32_t old = D.comm[v], nw = D.new_comm[v];
    const uint32_t g = D.gid ? D.gid[v] : 0u;
    long long di = 0;
    double df = 0.0;
    apply_entries<WINT>(D, v, old, nw, it, D.row[v] + lane, D.row[v + 1], 32, unit, di, df);
    if (WINT) {
      di = warp_sum(di);
      if (lane == 0 && di) atomicAdd(&D.gs[g].I, (unsigned long long)di);
    } else {
      df = warp_sum(df);
      if (lane == 0 && df != 0.0) atomicAdd(reinterpret_cast<double*>(&D.gs[g].I), df);
    }
  }
}

// Movers found by the block kernels (vertices with long rows): one block per piece of
// kHubPiece entries of their rows; the first piece also moves the totals.
template <bool WINT>
__global__ void __launch_bounds__(512) k_apply_hub(int dslot) {
  const Dev& D = c_dev[dslot];
  Ctrl* C = D.ctrl;
  const uint32_t count = C->apply_items, it = C->it;
  const bool unit = unit_weights<WINT>(C);
  __shared__ long long shi[32];
  __shared__ double shf[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (uint32_t idx = blockIdx.x; idx < count; idx += gridDim.x) {
    const unsigned long long item = D.apply_items[idx];
    const uint32_t v = (uint32_t)(item >> 32), piece = (uint32_t)item;
    const uint32_t old = D.comm[v], nw = D.new_comm[v];
    if (nw == old) continue;  // a rejected refinement proposal (the whole block skips it)
    const uint32_t g = D.gid ? D.gid[v] : 0u;
    if (threadIdx.x == 0 && piece == 0) {
      const double kv = D.k[v];
      atomicAdd(&D.a[nw], kv);
      atomicAdd(&D.a[old], -kv);
    }
    long long di = 0;
    double df = 0.0;
    const uint32_t ps = D.row[v] + piece * kHubPiece;
    const uint32_t pe = min(D.row[v + 1], ps + kHubPiece);
    apply_entries<WINT>(D, v, old, nw, it, ps + threadIdx.x, pe, blockDim.x, unit, di, df);
    di = warp_sum(di);
    df = warp_sum(df);
    if (lane == 0) { shi[wid] = di; shf[wid] = df; }
    __syncthreads();
    if (threadIdx.x == 0) {
      long long ti = 0;
      double tf = 0.0;
      for (int i = 0; i < (int)(blockDim.x >> 5); ++i) { ti += shi[i]; tf += shf[i]; }
      if (WINT) { if (ti) atomicAdd(&D.gs[g].I, (unsigned long long)ti); }
      else if (tf != 0.0) atomicAdd(reinterpret_cast<double*>(&D.gs[g].I), tf);
    }
    __syncthreads();
  }
}

// ---- pass: commit moves and recompute sum_c a_c^2 -----------------------------------------------
// Integer mode squares exactly in u64 (a_c <= 2m < 2^32). One graph: per-block partials,
// summed in a fixed order by k_finalize. Several graphs: one block per graph.
template <bool WINT>
__global__ void __launch_bounds__(256) k_commit_sq(int dslot, int single) {
  const Dev& D = c_dev[dslot];
  Ctrl* C = D.ctrl;
  const uint32_t count = C->mover_count, hubs = C->hub_mover_count, nn = C->n;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count + hubs; i += gridDim.x * blockDim.x) {
    const uint32_t v = D.movers[i < count ? i : nn - 1u - (i - count)];
    D.comm[v] = D.new_comm[v];
  }
  __shared__ double shd[33];
  __shared__ unsigned long long shu[33];
  if (single) {
    const uint32_t n = C->n;
    unsigned long long su = 0;
    double sf = 0.0;
    if (D.gs[0].phase == kIterating) {
      for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const double x = D.a[c];
        if (WINT) { const unsigned long long xi = (unsigned long long)x; su += xi * xi; }
        else sf = __dadd_rn(sf, __dmul_rn(x, x));
      }
    }
    if (WINT) {
      unsigned long long tot;
      block_excl_scan<unsigned long long, 256>(su, shu, &tot);
      if (threadIdx.x == 0) reinterpret_cast<unsigned long long*>(D.partials)[blockIdx.x] = tot;
    } else {
      double tot;
      block_excl_scan<double, 256>(sf, shd, &tot);
      if (threadIdx.x == 0) D.partials[blockIdx.x] = tot;
    }
  } else {
    for (uint32_t g = blockIdx.x; g < C->G; g += gridDim.x) {
      GraphState* st = &D.gs[g];
      if (st->phase != kIterating) continue;
      unsigned long long su = 0;
      double sf = 0.0;
      for (uint32_t c = st->vb + threadIdx.x; c < st->ve; c += blockDim.x) {
        const double x = D.a[c];
        if (WINT) { const unsigned long long xi = (unsigned long long)x; su += xi * xi; }
        else sf = __dadd_rn(sf, __dmul_rn(x, x));
      }
      if (WINT) {
        unsigned long long tot;
        block_excl_scan<unsigned long long, 256>(su, shu, &tot);
        if (threadIdx.x == 0) st->S = tot;
      } else {
        double tot;
        block_excl_scan<double, 256>(sf, shd, &tot);
        if (threadIdx.x == 0) st->S = __double_as_longlong(tot);
      }
    }
  }
}

__device__ __forceinline__ double modularity_of(double I, double S, double m) {
  // community.h:104: in / (2m) - sum_a2 / (4 m m)
  return __dsub_rn(__ddiv_rn(I, __dmul_rn(2.0, m)), __ddiv_rn(S, __dmul_rn(__dmul_rn(4.0, m), m)));
}

// Sets ctrl->fast / rule_sort for pass index p of a level (execution_number in
// phaseOptimization.cuh:116-146): p == 0 is the fast pass; afterwards SORT uses the lowest-c
// rule, HASH / ADAPTIVE_MEMORY the highest-c rule, ADAPTIVE_SPEED the lowest-c rule for p <= 4.
__device__ __forceinline__ void set_pass_rule(Ctrl* C, uint32_t p, int mode, int fast_first) {
  C->fast = (fast_first && p == 0) ? 1u : 0u;
  uint32_t sort_rule;
  if (mode == 1) sort_rule = 1;
  else if (mode == 2) sort_rule = p <= 4 ? 1u : 0u;
  else sort_rule = 0;
  C->rule_sort = sort_rule;
}

__global__ void k_set_pass(Ctrl* C, uint32_t p, int mode, int fast_first) {
  if (threadIdx.x == 0 && blockIdx.x == 0) set_pass_rule(C, p, mode, fast_first);
}

// ---- pass end: modularity, stop rule, counters ----------------------------------------------------
// phaseOptimization.cuh:167-179: dQ = Q_after - Q_before; the level's passes stop when
// dQ <= threshold (or after EARLY_STOP_LIMIT passes). `level_start` = 1 evaluates the level's
// starting modularity instead (Community::update -> compute_modularity, community.h:57-65).
// level_start = 2 keeps Q_level (a refined run's next level measures its gain from the
// previous level's end). view = 1: a refinement pass (no trace record, no pass statistics).
template <bool WINT>
__global__ void __launch_bounds__(1024) k_finalize(int dslot, int single, int nparts, int level_start,
                                                   int mode, int fast_first, GraphCtl gc, int view) {
  const Dev& D = c_dev[dslot];
  Ctrl* C = D.ctrl;
  __shared__ double shd[33];
  __shared__ unsigned long long shu[33];
  __shared__ uint32_t shc[33];
  if (single) {
    unsigned long long su = 0;
    double sf = 0.0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
      if (WINT) su += reinterpret_cast<const unsigned long long*>(D.partials)[i];
      else sf = __dadd_rn(sf, D.partials[i]);
    }
    if (WINT) {
      unsigned long long tot;
      block_excl_scan<unsigned long long, 1024>(su, shu, &tot);
      if (threadIdx.x == 0 && D.gs[0].phase == kIterating) D.gs[0].S = tot;
    } else {
      double tot;
      block_excl_scan<double, 1024>(sf, shd, &tot);
      if (threadIdx.x == 0 && D.gs[0].phase == kIterating) D.gs[0].S = __double_as_longlong(tot);
    }
    __syncthreads();
  }
  uint32_t iterating = 0;
  for (uint32_t g = threadIdx.x; g < C->G; g += blockDim.x) {
    GraphState* st = &D.gs[g];
    if (st->phase != kIterating) continue;
    const double I = WINT ? (double)st->I : __longlong_as_double((long long)st->I);
    const double S = WINT ? (double)st->S : __longlong_as_double((long long)st->S);
    const double Q = modularity_of(I, S, st->m);
    if (level_start) {
      st->Q = Q;
      if (level_start == 1) st->Q_level = Q;
      st->iters = 0;
      ++iterating;
      continue;
    }
    const double dq = __dsub_rn(Q, st->Q);
    st->Q = Q;
    st->iters += 1;
    st->total_iters += 1;
    if (single && !view) {
      st->moved = C->mover_count + C->hub_mover_count;
      const uint32_t t = C->trace_len;
      if (t < kTraceCap) {
        TraceRec r;
        r.level = st->level; r.iteration = st->iters - 1; r.n_moved = st->moved; r.pad = 0;
        r.internal = I; r.sum_a2 = S; r.modularity = Q; r.delta = dq;
        C->trace[t] = r;
        C->trace_len = t + 1;
      }
    }
    if (!(dq > C->threshold) || st->iters > C->max_iterations) st->phase = kLevelDone;
    else ++iterating;
  }
  // count graphs still iterating
  uint32_t tot;
  block_excl_scan<uint32_t, 1024>(iterating, shc, &tot);
  if (threadIdx.x == 0) {
    C->n_iterating = tot;
    C->loop_continue = tot > 0;
    for (int b = 0; b < kListBins; ++b) C->bin_count[b] = 0;
    C->mover_count = 0;
    C->long_movers = 0;
    C->hub_mover_count = 0;
    C->hub_items = 0;
    C->apply_items = 0;
    C->hub_cursor = 0;
    for (uint32_t i = 0; i < C->n_chunks && i < kMaxChunks; ++i) C->chunk_any[i] = 0;
    if (!view) {
      C->act_entries_total += C->act_entries;
      C->act_vertices_total += C->act_vertices;
    }
    C->act_entries = 0;
    C->act_vertices = 0;
    if (level_start) {
      C->pass = 0;
    } else {
      C->it += 1;
      C->pass += 1;
      if (!view) {
        C->seg_passes += 1;
        C->t_opt_ns += global_ns() - C->t_pass0;
      }
      if (C->seg_passes > kGuardPasses) atomicOr(&C->err, kErrLoop);
      // the captured pass loop runs while a graph iterates (and no guard has tripped)
      set_cond(gc, gc.pass, tot > 0 && !(C->err & kErrLoop));
    }
    set_pass_rule(C, C->pass, mode, fast_first);
  }
}


// ---- level start ------------------------------------------------------------------------------------
// Community::update (community.h:57-65): identity partition, totals = k, every vertex active
// (phaseOptimization.cuh:52).
__global__ void k_level_init(int dslot) {
  const Dev& D = c_dev[dslot];
  Ctrl* C = D.ctrl;
  const uint32_t n = C->n, it = C->it;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const uint32_t g = D.gid ? D.gid[v] : 0u;
    if (D.gs[g].phase != kIterating) continue;
    // new_comm == comm marks "did not move" for the apply kernels (movers get new_comm != comm
    // and k_commit_sq copies it back), so it starts equal too
    D.comm[v] = v;
    D.new_comm[v] = v;
    D.a[v] = D.k[v];
    D.active_it[v] = it;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    C->mover_count = 0;
    C->long_movers = 0;
    C->hub_mover_count = 0;
    C->hub_items = 0;
    C->apply_items = 0;
    for (int b = 0; b < kListBins; ++b) C->bin_count[b] = 0;
    C->hub_cursor = 0;
    C->arena_need = 0;
    for (int i = 0; i < kMaxChunks; ++i) C->chunk_any[i] = 0;
  }
}

// Chunk bounds of the reference's edge loop for the current level (single graph):
// limit = round + STEP; limit = (limit >= E) ? E : neighboorhood_sum[edge_source[limit] - 1].
__global__ void k_chunk_bounds(int dslot, unsigned long long step) {
  const Dev& D = c_dev[dslot];
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  Ctrl* C = D.ctrl;
  const uint32_t n = C->n, E = C->E;
  C->chunk_on = 0;
  C->n_chunks = 1;
  C->chunk_lo[0] = 0;
  C->chunk_lo[1] = n;
  if (step == 0 || (unsigned long long)E <= step) return;
  unsigned long long round = 0;
  uint32_t nch = 0;
  while (round < E) {
    if (nch >= kMaxChunks) { atomicOr(&C->err, kErrChunks); return; }
    // first vertex of this chunk: the one whose row starts at `round`
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) { const uint32_t mid = (lo + hi) / 2; if (D.row[mid] <= round) lo = mid; else hi = mid; }
    C->chunk_lo[nch++] = lo;
    unsigned long long limit = round + step;
    if (limit >= E) break;
    lo = 0; hi = n;
    while (hi - lo > 1) { const uint32_t mid = (lo + hi) / 2; if (D.row[mid] <= limit) lo = mid; else hi = mid; }
    if (lo == 0) return;  // the reference would read neighboorhood_sum[-1]: no emulation
    limit = D.row[lo - 1];
    if (limit <= round) return;  // a row longer than STEP_ROUND: the reference loops forever; no emulation
    round = limit;
  }
  C->n_chunks = nch;
  C->chunk_lo[nch] = n;
  C->chunk_on = 1;
}

// ---- level 0: input validation, weights, k, self-loop weight, total weight --------------------------
// GraphDevice(GraphHost&) (graph.cuh:46-99) and the Community constructor (community.h:31-46):
// k = sum of incident weights, m = total weight / 2 (graph.cu:81). One warp per vertex.
constexpr uint32_t kPrepLongRow = 4096;
// k_prep's local marker (never stored in Ctrl::err): a weight other than 1 was seen.
constexpr uint32_t kErrNotUnit = 1u << 31;

// Validation and weight conversion of entries [e0, re) with stride `step` of row v (graph
// vertex range [lo, hi)); sums of the row's weights and of its self-loop weights.
template <bool WINT>
__device__ __forceinline__ void prep_entries(const Dev& D, uint32_t v, long long e0, long long re,
                                             uint32_t step, uint32_t lo, uint32_t hi, const float* wf_in,
                                             const uint32_t* wu_in, unsigned long long& ki,
                                             unsigned long long& si, double& kf, double& sf,
                                             uint32_t& err) {
  for (long long e = e0; e < re; e += step) {
    const uint32_t u = D.col[e];
    if (u < lo || u >= hi) { err |= kErrInput; continue; }
    const float x = wf_in ? wf_in[e] : 1.0f;
    if (WINT) {
      // integer weights come as floats (exact below 2^24) or, for a resumed level whose sums
      // may exceed that, as u32 (wu_in)
      if (!wu_in && (!(x >= 1.0f) || x != floorf(x) || x > 4294967040.0f)) { err |= kErrInput; continue; }
      const uint32_t xi = wu_in ? wu_in[e] : (uint32_t)x;
      if (xi == 0u) { err |= kErrInput; continue; }
      if (xi != 1u) err |= kErrNotUnit;
      reinterpret_cast<uint32_t*>(D.w)[e] = xi;
      ki += xi;
      if (u == v) si += xi;
    } else {
      if (!(x > 0.0f) || !(x < INFINITY)) { err |= kErrInput; continue; }
      reinterpret_cast<float*>(D.w)[e] = x;
      kf += (double)x;
      if (u == v) sf += (double)x;
    }
  }
}

template <bool WINT>
__global__ void __launch_bounds__(256) k_prep(int dslot, const long long* row64, const float* wf_in,
                                              const uint32_t* wu_in,
                                              uint32_t n, unsigned long long E) {
  const Dev& D = c_dev[dslot];
  Ctrl* C = D.ctrl;
  const int lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  uint32_t err = 0;
  // per-graph totals are kept in registers and flushed when the graph changes
  uint32_t cur_g = kEmpty;
  unsigned long long tk_i = 0, ts_i = 0;
  double tk_f = 0.0, ts_f = 0.0;
  auto flush = [&]() {
    if (cur_g == kEmpty || lane != 0) return;
    if (WINT) {
      if (ts_i) atomicAdd(&D.gs[cur_g].I, ts_i);
      if (tk_i) atomicAdd(&D.gs[cur_g].S, tk_i);  // S holds sum k (= 2m) until k_prep_total
    } else {
      if (ts_f != 0.0) atomicAdd(reinterpret_cast<double*>(&D.gs[cur_g].I), ts_f);
      if (tk_f != 0.0) atomicAdd(reinterpret_cast<double*>(&D.gs[cur_g].S), tk_f);
    }
  };
  for (uint32_t v = warp; v < n; v += nwarps) {
    const long long rs = row64[v], re = row64[v + 1];
    const uint32_t g = D.gid ? D.gid[v] : 0u;
    const uint32_t lo = D.gs[g].vb, hi = D.gs[g].ve;
    if (rs < 0 || re <= rs || (unsigned long long)re > E) {
      if (lane == 0) { err |= kErrInput; D.row[v] = 0; D.k[v] = 0.0; }
      continue;
    }
    if (lane == 0) {
      D.row[v] = (uint32_t)rs;
      if (v == n - 1) D.row[n] = (uint32_t)re;
    }
    if (re - rs > kPrepLongRow) {  // a block takes it (k_prep_long)
      if (lane == 0) D.bins[kNumBins - 1][atomicAdd(&C->bin_count[kNumBins - 1], 1u)] = v;
      continue;
    }
    if (g != cur_g) {
      flush();
      cur_g = g;
      tk_i = ts_i = 0;
      tk_f = ts_f = 0.0;
    }
    unsigned long long ki = 0, si = 0;
    double kf = 0.0, sf = 0.0;
    prep_entries<WINT>(D, v, rs + lane, re, 32, lo, hi, wf_in, wu_in, ki, si, kf, sf, err);
    if (WINT) {
      ki = warp_sum(ki);
      si = warp_sum(si);
      if (lane == 0) D.k[v] = (double)ki;
      tk_i += ki;
      ts_i += si;
    } else {
      kf = warp_sum(kf);
      sf = warp_sum(sf);
      if (lane == 0) D.k[v] = kf;
      tk_f += kf;
      ts_f += sf;
    }
  }
  flush();
  if (err & kErrNotUnit) C->unit_w = 0;
  err &= ~kErrNotUnit;
  if (err) report_err(C, err, 3);  // k_prep
}

// Rows longer than kPrepLongRow entries, one block each.
template <bool WINT>
__global__ void __launch_bounds__(512) k_prep_long(int dslot, const float* wf_in, const uint32_t* wu_in) {
  const Dev& D = c_dev[dslot];
  Ctrl* C = D.ctrl;
  __shared__ unsigned long long shu[33];
  __shared__ double shd[33];
  const uint32_t count = C->bin_count[kNumBins - 1];
  uint32_t err = 0;
  for (uint32_t idx = blockIdx.x; idx < count; idx += gridDim.x) {
    const uint32_t v = D.bins[kNumBins - 1][idx];
    const uint32_t rs = D.row[v], re = D.row[v + 1];
    const uint32_t g = D.gid ? D.gid[v] : 0u;
    unsigned long long ki = 0, si = 0;
    double kf = 0.0, sf = 0.0;
    prep_entries<WINT>(D, v, rs + threadIdx.x, re, blockDim.x, D.gs[g].vb, D.gs[g].ve, wf_in, wu_in, ki, si, kf, sf, err);
    if (WINT) {
      ki = block_sum<512>(ki, shu);
      si = block_sum<512>(si, shu);
      if (threadIdx.x == 0) {
        D.k[v] = (double)ki;
        if (si) atomicAdd(&D.gs[g].I, si);
        atomicAdd(&D.gs[g].S, ki);
      }
    } else {
      kf = block_sum<512>(kf, shd);
      sf = block_sum<512>(sf, shd);
      if (threadIdx.x == 0) {
        D.k[v] = kf;
        if (sf != 0.0) atomicAdd(reinterpret_cast<double*>(&D.gs[g].I), sf);
        atomicAdd(reinterpret_cast<double*>(&D.gs[g].S), kf);
      }
    }
  }
  if (err & kErrNotUnit) C->unit_w = 0;
  err &= ~kErrNotUnit;
  if (err) report_err(C, err, 4);  // k_prep_long
}

// m = (sum of k) / 2 per graph; integer mode requires 2m < 2^32 (the reference's u32 sums).
template <bool WINT>
__global__ void k_prep_total(int dslot) {
  const Dev& D = c_dev[dslot];
  Ctrl* C = D.ctrl;
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < C->G; g += gridDim.x * blockDim.x) {
    GraphState* st = &D.gs[g];
    double twice;
    if (WINT) {
      if (st->S >= 4294967296ull) atomicOr(&C->err, kErrRange);
      twice = (double)st->S;
    } else {
      twice = __longlong_as_double((long long)st->S);
    }
    st->m = twice / 2.0;
    st->two_m2 = __dmul_rn(__dmul_rn(2.0, st->m), st->m);
    st->inv_m = __drcp_rn(st->m);
    st->inv_2m2 = __drcp_rn(st->two_m2);
    st->S = 0;
  }
}

// Integer-weight detection for LV_WEIGHTS_AUTO: any weight that is not a non-negative integer
// representable in u32 selects float mode.
__global__ void k_weights_integral(const float* w, unsigned long long E, uint32_t* flag) {
  for (unsigned long long e = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; e < E;
       e += (unsigned long long)gridDim.x * blockDim.x) {
    const float x = w[e];
    if (!(x >= 0.0f) || x != floorf(x) || x > 4294967040.0f) { *flag = 1; return; }
  }
}

// Graph ids of each vertex from the packed offsets (batched input).
__global__ void k_fill_gid(uint32_t* gid, const long long* offs, uint32_t G) {
  for (uint32_t g = blockIdx.x; g < G; g += gridDim.x) {
    const long long b = offs[g], e = offs[g + 1];
    for (long long v = b + threadIdx.x; v < e; v += blockDim.x) gid[v] = g;
  }
}

// Graphs uploaded one by one into a packed batch keep their local numbering; this rebases
// them: row offsets of graph g gain its first entry eoffs[g], destinations its first vertex
// voffs[g]. An entry finds its graph by binary search over eoffs (G is small).
__global__ void k_rebase_pieces(long long* row64, uint32_t* col, const long long* voffs,
                                const long long* eoffs, uint32_t G, uint32_t n, uint32_t E) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  for (uint32_t e = tid; e < E; e += nth) {
    uint32_t lo = 0, hi = G;  // last g with eoffs[g] <= e
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if ((unsigned long long)eoffs[mid] <= e) lo = mid; else hi = mid;
    }
    col[e] += (uint32_t)voffs[lo];
  }
  for (uint32_t v = tid; v < n; v += nth) {
    uint32_t lo = 0, hi = G;  // last g with voffs[g] <= v
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if ((unsigned long long)voffs[mid] <= v) lo = mid; else hi = mid;
    }
    row64[v] += eoffs[lo];
  }
  if (tid == 0) row64[n] = E;
}

// Hash-table arena needed by the global-table bin at this level: sum over vertices with
// degree above the shared-memory bound of next_pow2(2 d).
__global__ void k_arena_need(int dslot, uint32_t min_deg, uint32_t block_cap) {
  const Dev& D = c_dev[dslot];
  unsigned long long* need = &D.ctrl->arena_need;
  const uint32_t n = D.ctrl->n;
  unsigned long long s = 0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const uint32_t d = D.row[v + 1] - D.row[v];
    if (d <= min_deg) continue;
    const uint32_t g = D.gid ? D.gid[v] : 0u;
    const uint32_t ng = D.gid ? D.gs[g].ve - D.gs[g].vb : n;
    if (table_cap(d, ng) > block_cap) s += hub_table_cap(d, ng);
  }
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0 && s) atomicAdd(need, s);
}

// ---- aggregation -------------------------------------------------------------------------------------
// phaseAggregation.cuh:27-43: new id = inclusive count of nonempty communities minus one. The
// reference tests a_c > 0 (CountNotZero); with every weight positive that is exactly "has a
// member", which is what is marked here, so no rounding residue in a_c can create an empty
// row. The low word counts only communities of graphs that continue to a new level.
__global__ void k_agg_mark(int dslot) {
  const Dev& D = c_dev[dslot];
  const uint32_t n = D.ctrl->n;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    D.map[D.comm[v]] = 1ull;
}

__global__ void k_agg_flags(int dslot) {
  const Dev& D = c_dev[dslot];
  const uint32_t n = D.ctrl->n;
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    const uint32_t g = D.gid ? D.gid[c] : 0u;
    const unsigned long long ne = D.map[c] != 0ull ? 1ull : 0ull;
    D.map[c] = (ne << 32) | (ne & (unsigned long long)D.gs[g].cont);
  }
}

// Per graph: n_of_best_communities, base of its final ids, next-level vertex range.
__global__ void k_agg_meta(int dslot) {
  const Dev& D = c_dev[dslot];
  Ctrl* C = D.ctrl;
  const uint32_t n = C->n;
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < C->G; g += gridDim.x * blockDim.x) {
    GraphState* st = &D.gs[g];
    if (!st->agg) continue;
    const unsigned long long before = st->vb > 0 ? D.map[st->vb - 1] : 0ull;
    const unsigned long long end = D.map[st->ve - 1];
    st->map_base = (uint32_t)(before >> 32);
    st->n_best = (uint32_t)(end >> 32) - st->map_base;
    st->n_next = (uint32_t)end - (uint32_t)before;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) C->n_next = n ? (uint32_t)D.map[n - 1] : 0u;
}

// community.h:48-55 update_best: best[v0] = new(comm[best[v0]]). Graphs that stop here get
// their final ids (0..K-1 within the graph) written to `out`.
__global__ void k_agg_best(int dslot) {
  const Dev& D = c_dev[dslot];
  Ctrl* C = D.ctrl;
  const uint32_t n0 = C->n0;
  for (uint32_t v0 = blockIdx.x * blockDim.x + threadIdx.x; v0 < n0; v0 += gridDim.x * blockDim.x) {
    const uint32_t g = D.gid0 ? D.gid0[v0] : 0u;
    const GraphState& st = D.gs[g];
    if (!st.agg) continue;
    const uint32_t b = D.best[v0];
    const unsigned long long mv = D.map[D.comm[b]];
    if (st.cont) {
      D.best[v0] = (uint32_t)mv - 1u;
    } else {
      const uint32_t id = (uint32_t)(mv >> 32) - 1u - st.map_base;
      D.best[v0] = id;
      D.out[v0] = (int32_t)id;
    }
  }
}

// Count members and degree sums of each new community (packed, one atomic per vertex); the
// returned old value is the vertex's rank inside its community.
__global__ void k_agg_count(int dslot) {
  const Dev& D = c_dev[dslot];
  const uint32_t n = D.ctrl->n;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const uint32_t g = D.gid ? D.gid[v] : 0u;
    if (!D.gs[g].cont) continue;
    const uint32_t s = (uint32_t)D.map[D.comm[v]] - 1u;
    const uint32_t d = D.row[v + 1] - D.row[v];
    const unsigned long long old = atomicAdd(&D.cd[s], (1ull << 32) | d);
    D.rank[v] = (uint32_t)(old >> 32);
    D.new_comm[v] = s;  // next-level id of v's community, read by the contraction
  }
}

__global__ void k_agg_scatter(int dslot) {
  const Dev& D = c_dev[dslot];
  const uint32_t n = D.ctrl->n;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const uint32_t g = D.gid ? D.gid[v] : 0u;
    if (!D.gs[g].cont) continue;
    const uint32_t s = D.new_comm[v];
    D.members[(uint32_t)(D.cd[s] >> 32) + D.rank[v]] = v;
  }
}

// Capacity of a new community's contraction table: distinct destinations are bounded by the
// member degree sum and by the graph's next-level vertex count. Global (bin 7) tables are
// whole multiples of kHubChunk so every chunk of the arena belongs to one table.
__device__ __forceinline__ uint32_t contract_cap(uint32_t dsum, uint32_t ng, bool global) {
  const uint32_t c = table_cap(dsum, ng);
  return global && c < kHubChunk ? kHubChunk : c;
}

// Bin the new communities by their summed member degree (the contraction's work). Bin 7
// communities (the largest) are contracted by many blocks at once into a global table whose
// arena offset is recorded per community in hubtab (kEmpty for every other community).
__global__ void k_agg_bin(int dslot, BinCfg B) {
  const Dev& D = c_dev[dslot];
  Ctrl* C = D.ctrl;
  const uint32_t n2 = C->n_next;
  for (uint32_t base = blockIdx.x * blockDim.x; base < n2; base += gridDim.x * blockDim.x) {
    const uint32_t s = base + threadIdx.x;
    int bin = -1;
    uint32_t dsum = 0, cap = 0;
    if (s < n2) {
      dsum = (uint32_t)D.cd[s + 1] - (uint32_t)D.cd[s];
      bin = bin_of(B, dsum);
      if (bin >= kNumBins - 2) {
        const uint32_t g = D.gid ? D.gid[D.members[(uint32_t)(D.cd[s] >> 32)]] : 0u;
        cap = contract_cap(dsum, D.gs[g].n_next, bin == kNumBins - 1);
        // a bin-6 community whose table fits half the block table: the half-block list
        if (bin == kNumBins - 2 && 2u * cap <= B.block_cap) bin = kHalfBin;
      }
    }
#pragma unroll
    for (int b = 0; b < kListBins; ++b) {
      const uint32_t pos = warp_append(bin, b, &C->bin_count[b]);
      if (pos != kEmpty) {
        D.bins[b][pos] = s;
        if (b == kNumBins - 1) {
          const uint32_t off = atomicAdd(&C->hub_cursor, cap);
          D.hub_off[pos] = off;
          D.hubtab[s] = off;
        }
      }
    }
  }
}

// Bin-7 set-up once the arena is large enough: owner of every table chunk, and zeroed
// accumulators (row length, k') of each such community.
__global__ void k_hub_owner(int dslot, int bin) {
  const Dev& D = c_dev[dslot];
  Ctrl* C = D.ctrl;
  const uint32_t count = C->bin_count[bin];
  for (uint32_t idx = blockIdx.x; idx < count; idx += gridDim.x) {
    const uint32_t s = D.bins[bin][idx];
    const uint32_t v0 = D.members[(uint32_t)(D.cd[s] >> 32)];
    const uint32_t g = D.gid ? D.gid[v0] : 0u;
    const uint32_t dsum = (uint32_t)D.cd[s + 1] - (uint32_t)D.cd[s];
    const uint32_t cap = contract_cap(dsum, D.gs[g].n_next, true);
    const uint32_t c0 = D.hub_off[idx] / kHubChunk;
    for (uint32_t j = threadIdx.x; j < cap / kHubChunk; j += blockDim.x) D.hub_owner[c0 + j] = s;
    if (threadIdx.x == 0) {
      D.newdeg[s] = 0;
      D.kB[s] = 0.0;
      D.hubself[s] = 0ull;
      if (D.gidB) D.gidB[s] = g;
    }
  }
}

// Insert into a community's global contraction table at arena offset `off` (capacity `cap`).
template <bool WINT>
__device__ __forceinline__ bool hub_table_add(const Dev& D, uint32_t off, uint32_t cap, uint32_t d,
                                              typename WTraits<WINT>::Acc w) {
  using Acc = typename WTraits<WINT>::Acc;
  const uint32_t mask = cap - 1u, shift = 32u - log2_pow2(cap);
  if constexpr (WINT) {
    return PackedTable{reinterpret_cast<unsigned long long*>(D.arena_vals) + off, mask, shift}.add(d, w);
  } else {
    return table_add(D.arena_keys + off, reinterpret_cast<Acc*>(D.arena_vals) + off, mask, shift, d, w);
  }
}
// Slot `i` of the arena: its community (kEmpty if unused) and sum.
template <bool WINT>
__device__ __forceinline__ void hub_table_load(const Dev& D, uint32_t i, uint32_t& key,
                                               typename WTraits<WINT>::Acc& sum) {
  using Acc = typename WTraits<WINT>::Acc;
  if constexpr (WINT) {
    const unsigned long long x = reinterpret_cast<const unsigned long long*>(D.arena_vals)[i];
    key = (uint32_t)(x >> 32);
    sum = (Acc)(uint32_t)x;
  } else {
    key = D.arena_keys[i];
    sum = key != kEmpty ? reinterpret_cast<const Acc*>(D.arena_vals)[i] : Acc(0);
  }
}

// Where the members of each bin-7 community start among all bin-7 members (exclusive prefix of
// their member counts, in `rank`, which is free after the scatter) and how many there are.
__global__ void __launch_bounds__(1024) k_hub_member_prefix(int dslot) {
  const Dev& D = c_dev[dslot];
  __shared__ uint32_t sh[33];
  Ctrl* C = D.ctrl;
  const uint32_t count = C->bin_count[kNumBins - 1];
  uint32_t run = 0;
  for (uint32_t base = 0; base < count; base += 1024) {
    const uint32_t idx = base + threadIdx.x;
    uint32_t m = 0;
    if (idx < count) {
      const uint32_t s = D.bins[kNumBins - 1][idx];
      m = (uint32_t)(D.cd[s + 1] >> 32) - (uint32_t)(D.cd[s] >> 32);
    }
    uint32_t tot;
    const uint32_t ex = block_excl_scan<uint32_t, 1024>(m, sh, &tot);
    if (idx < count) D.rank[idx] = run + ex;
    run += tot;
  }
  if (threadIdx.x == 0) C->hub_members = run;
}

// Bin-7 insert: the members of all large communities at once (and no other vertex), 32 per
// warp (groups taken from a shared counter), their rows spread over the lanes, into their
// communities' global tables (L2 atomics). Rows over kHubLongRow go to k_hub_insert_long in
// pieces.
template <bool WINT>
__global__ void __launch_bounds__(256) k_hub_insert(int dslot) {
  const Dev& D = c_dev[dslot];
  using Tr = WTraits<WINT>;
  using Acc = typename Tr::Acc;
  using Wt = typename Tr::W;
  Ctrl* C = D.ctrl;
  const uint32_t count = C->bin_count[kNumBins - 1], total = C->hub_members;
  const uint32_t* hubs = D.bins[kNumBins - 1];
  const Wt* __restrict__ w = reinterpret_cast<const Wt*>(D.w);
  const int lane = threadIdx.x & 31;
  uint32_t err = 0;
  // entries staying inside their community are summed in registers
  uint32_t self_s = kEmpty;  // per-lane running self-loop sum, flushed when the community changes
  Acc self_acc = Acc(0);
  auto flush_self = [&]() {
    if (self_s == kEmpty || self_acc == Acc(0)) return;
    if (WINT) atomicAdd(&D.hubself[self_s], (unsigned long long)self_acc);
    else atomicAdd(reinterpret_cast<double*>(&D.hubself[self_s]), (double)self_acc);
  };
  auto add = [&](uint32_t e, uint32_t s, uint32_t off, uint32_t cap) {
    const uint32_t d = D.new_comm[D.col[e]];
    if (d == s) {
      if (s != self_s) {
        flush_self();
        self_s = s;
        self_acc = Acc(0);
      }
      self_acc += (Acc)w[e];
      return;
    }
    if (!hub_table_add<WINT>(D, off, cap, d, (Acc)w[e])) err |= kErrTableFull;
  };
  // warps take groups of 32 members from a shared counter (row lengths are heavy-tailed)
  for (;;) {
    uint32_t pb = 0;
    if (lane == 0) pb = atomicAdd(&C->hub_work, 32u);
    pb = __shfl_sync(kFull, pb, 0);
    if (pb >= total) break;
    const uint32_t p = pb + lane;
    uint32_t rs = 0, len = 0, s = 0, off = 0, cap = 0;
    if (p < total) {
      uint32_t lo = 0, hi = count;  // last community whose members start at or before p
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (D.rank[mid] <= p) lo = mid; else hi = mid;
      }
      s = hubs[lo];
      const unsigned long long a = D.cd[s], b = D.cd[s + 1];
      const uint32_t v = D.members[(uint32_t)(a >> 32) + (p - D.rank[lo])];
      const uint32_t g = D.gid ? D.gid[v] : 0u;
      off = D.hub_off[lo];
      cap = contract_cap((uint32_t)b - (uint32_t)a, D.gs[g].n_next, true);
      if ((unsigned long long)off + cap > C->arena_slots) {
        err |= kErrArena;
      } else {
        rs = D.row[v];
        len = D.row[v + 1] - rs;
        if (len > kHubLongRow) {
          // long rows are cut into pieces that separate blocks insert (k_hub_insert_long)
          const uint32_t np = (len + kHubInsPiece - 1) / kHubInsPiece;
          const uint32_t p0 = atomicAdd(&C->long_count, np);
          for (uint32_t k = 0; k < np; ++k) D.long_items[p0 + k] = ((unsigned long long)v << 32) | k;
          len = 0;
        }
      }
    }
    warp_expand_rows3(rs, len, s, off, cap, add);
  }
  flush_self();
  if (err) report_err(C, err, 5);  // k_hub_insert
}

// Pieces of the long rows deferred by k_hub_insert, one block per piece.
template <bool WINT>
__global__ void __launch_bounds__(256) k_hub_insert_long(int dslot) {
  const Dev& D = c_dev[dslot];
  using Tr = WTraits<WINT>;
  using Acc = typename Tr::Acc;
  using Wt = typename Tr::W;
  __shared__ Acc sh[33];
  Ctrl* C = D.ctrl;
  const uint32_t count = C->long_count;
  const Wt* __restrict__ w = reinterpret_cast<const Wt*>(D.w);
  const bool unit = unit_weights<WINT>(C);
  uint32_t err = 0;
  const uint32_t n = C->n, n2 = C->n_next;
  for (uint32_t idx = blockIdx.x; idx < count; idx += gridDim.x) {
    const unsigned long long it = D.long_items[idx];
    const uint32_t v = (uint32_t)(it >> 32), piece = (uint32_t)it;
    // an item always names a vertex of this level in a bin-7 community whose table fits the
    // arena (k_hub_insert checked that when it queued the item); anything else is reported
    if (v >= n) { err |= kErrIndex; continue; }
    const uint32_t g = D.gid ? D.gid[v] : 0u;
    const uint32_t s = D.new_comm[v];
    if (s >= n2) { err |= kErrIndex; continue; }
    const uint32_t off = D.hubtab[s];
    const uint32_t dsum = (uint32_t)D.cd[s + 1] - (uint32_t)D.cd[s];
    const uint32_t cap = contract_cap(dsum, D.gs[g].n_next, true);
    if (off == kEmpty || (unsigned long long)off + cap > C->arena_slots) { err |= kErrIndex; continue; }
    const uint32_t rs = D.row[v] + piece * kHubInsPiece;
    const uint32_t re = min(D.row[v + 1], rs + kHubInsPiece);
    Acc self_acc = Acc(0);
    // one entry per thread and step: batching the loads and inserts of several entries (or
    // trying the CAS before reading the slot) measured slower here -- more atomics in flight on
    // the hot keys of a large community's table; so did summing each 2048-entry chunk in a
    // shared-memory table before adding its distinct keys to the global table
    for (uint32_t e = rs + threadIdx.x; e < re; e += blockDim.x) {
      const uint32_t d = D.new_comm[D.col[e]];
      const Acc wv = unit ? Acc(1) : (Acc)w[e];
      if (d == s) { self_acc += wv; continue; }
      if (!hub_table_add<WINT>(D, off, cap, d, wv)) err |= kErrTableFull;
    }
    self_acc = block_sum<256>(self_acc, sh);
    if (threadIdx.x == 0 && self_acc != Acc(0)) {
      if (WINT) atomicAdd(&D.hubself[s], (unsigned long long)self_acc);
      else atomicAdd(reinterpret_cast<double*>(&D.hubself[s]), (double)self_acc);
    }
  }
  if (err) report_err(C, err, 6);  // k_hub_insert_long
}

// Bin-7 emit: one block per table chunk; occupied slots are appended to the community's row
// (positions claimed with one atomic per block), k' and the self-loop weight accumulated.
template <bool WINT>
__global__ void __launch_bounds__(512) k_hub_emit(int dslot) {
  const Dev& D = c_dev[dslot];
  const uint32_t nchunks = min(D.ctrl->hub_cursor, D.ctrl->arena_slots) / kHubChunk;
  using Tr = WTraits<WINT>;
  using Acc = typename Tr::Acc;
  using Wt = typename Tr::W;
  __shared__ uint32_t shu[33];
  __shared__ double shd[33];
  __shared__ uint32_t base_sh;
  Wt* __restrict__ wout = reinterpret_cast<Wt*>(D.wB);
  constexpr int PER = kHubChunk / 512;
  for (uint32_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
    const uint32_t s = D.hub_owner[c];
    const uint32_t tb = (uint32_t)D.cd[s];
    const uint32_t v0 = D.members[(uint32_t)(D.cd[s] >> 32)];
    const uint32_t g = D.gid ? D.gid[v0] : 0u;
    const uint32_t slot0 = c * kHubChunk + threadIdx.x * PER;
    uint32_t cnt = 0;
    uint32_t kk[PER];
    Acc ss[PER];
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      hub_table_load<WINT>(D, slot0 + i, kk[i], ss[i]);
      cnt += kk[i] != kEmpty;
    }
    uint32_t total;
    uint32_t off = block_excl_scan<uint32_t, 512>(cnt, shu, &total);
    if (threadIdx.x == 0) base_sh = total ? atomicAdd(&D.newdeg[s], total) : 0u;
    __syncthreads();
    off += base_sh;
    double ksum = 0.0, self = 0.0;
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      const uint32_t d = kk[i];
      if (d == kEmpty) continue;
      const Acc sum = ss[i];
      Wt wv;
      if (WINT) wv = (Wt)sum;
      else wv = (Wt)__double2float_rn((double)sum);
      D.colB[tb + off] = d;
      wout[tb + off] = wv;
      ++off;
      ksum += Tr::w_double(wv);
      if (d == s) self += Tr::w_double(wv);
    }
    double ktot, stot;
    block_excl_scan<double, 512>(ksum, shd, &ktot);
    block_excl_scan<double, 512>(self, shd, &stot);
    if (threadIdx.x == 0) {
      // the community's first chunk also emits its self-loop, summed outside the table
      if (c == D.hubtab[s] / kHubChunk && D.hubself[s] != 0ull) {
        const unsigned long long hs = D.hubself[s];
        Wt wv;
        if (WINT) wv = (Wt)hs;
        else wv = (Wt)__double2float_rn(__longlong_as_double((long long)hs));
        const uint32_t pos = atomicAdd(&D.newdeg[s], 1u);
        D.colB[tb + pos] = s;
        wout[tb + pos] = wv;
        ktot += Tr::w_double(wv);
        stot += Tr::w_double(wv);
      }
      if (ktot != 0.0) atomicAdd(&D.kB[s], ktot);
      if (stot != 0.0) {
        if (WINT) atomicAdd(&D.gs[g].I, (unsigned long long)stot);
        else atomicAdd(reinterpret_cast<double*>(&D.gs[g].I), stot);
      }
    }
    __syncthreads();
  }
}

struct CommCtx {
  uint32_t mb, me, tb, dsum, g;
};

__device__ __forceinline__ CommCtx load_comm(const Dev& D, uint32_t s) {
  CommCtx x;
  const unsigned long long a = D.cd[s], b = D.cd[s + 1];
  x.mb = (uint32_t)(a >> 32);
  x.me = (uint32_t)(b >> 32);
  x.tb = (uint32_t)a;
  x.dsum = (uint32_t)b - (uint32_t)a;
  const uint32_t v0 = D.members[x.mb];
  x.g = D.gid ? D.gid[v0] : 0u;
  return x;
}

// Contraction of one new community s (phaseAggregation.cuh:51-106 for SORT,
// :107-141 for HASH): every entry (v,u,w) of every member v goes to (s, new(comm u)), weights
// summed exactly (u32 in integer mode, double then one fp32 rounding in float mode). The
// unique destinations are written to colB/wB at the community's degree-sum offset, the row
// length to newdeg, k' = row sum to kB, the self-loop weight to the graph's next-level I.
template <int T, bool WINT>
__global__ void __launch_bounds__(256) k_contract_team(int dslot, int bin, uint32_t cap) {
  const Dev& D = c_dev[dslot];
  using Tr = WTraits<WINT>;
  using Acc = typename Tr::Acc;
  using Wt = typename Tr::W;
  constexpr int TEAMS = 256 / T;
  extern __shared__ __align__(16) unsigned char smem[];
  const int team = threadIdx.x / T, lane = threadIdx.x % T;
  // per team: a table of `cap` slots and a list of cap / 2 u16 slot indices (as k_opt_team)
  constexpr size_t kSlotBytes = WINT ? 8 : 4 + sizeof(Acc);
  uint32_t* keys = reinterpret_cast<uint32_t*>(smem) + (size_t)team * cap;
  Acc* vals = reinterpret_cast<Acc*>(smem + (size_t)TEAMS * cap * sizeof(uint32_t)) + (size_t)team * cap;
  unsigned long long* slots = reinterpret_cast<unsigned long long*>(smem) + (size_t)team * cap;
  uint16_t* klist = reinterpret_cast<uint16_t*>(smem + (size_t)TEAMS * cap * kSlotBytes) + (size_t)team * (cap / 2);
  Ctrl* C = D.ctrl;
  const uint32_t count = C->bin_count[bin];
  if (blockIdx.x * TEAMS >= count) return;  // (block-uniform)
  const uint32_t* list = D.bins[bin];
  const Wt* __restrict__ w = reinterpret_cast<const Wt*>(D.w);
  Wt* __restrict__ wout = reinterpret_cast<Wt*>(D.wB);
  const bool unit = unit_weights<WINT>(C);
  const unsigned tmask = T == 32 ? kFull : (((1u << T) - 1u) << ((threadIdx.x & 31) & ~(uint32_t)(T - 1)));
  const uint32_t lt = lanemask_lt();
  uint32_t err = 0;
  ScratchTable<WINT> tbl{keys, vals, slots, cap - 1u, 0u};
  for (uint32_t i = lane; i < cap; i += T) tbl.clear(i);
  __syncwarp();
  for (uint32_t base = blockIdx.x * TEAMS; base < count; base += gridDim.x * TEAMS) {
    const uint32_t idx = base + team;
    const bool live = idx < count;
    const uint32_t s = live ? list[idx] : 0u;
    CommCtx x{};
    if (live) x = load_comm(D, s);
    const uint32_t cap_v = live ? contract_cap(x.dsum, D.gs[x.g].n_next, false) : 2u;
    tbl.mask = cap_v - 1u;
    tbl.shift = 32u - log2_pow2(cap_v);
    // entries staying inside the community (the new self-loop, the hottest key) are summed in
    // registers; only entries to other communities go through the table, and each community
    // the table gains is listed
    Acc self_acc = Acc(0);
    uint32_t nl = 0;
    auto add = [&](uint32_t e, bool valid) {
      bool made = false;
      uint32_t slot = 0;
      if (valid) {
        const uint32_t d = D.new_comm[D.col[e]];
        const Acc wv = unit ? Acc(1) : (Acc)w[e];
        if (d == s) {
          self_acc += wv;
        } else {
          const int r = tbl.add_at(d, wv, slot);
          if (!r) err |= kErrTableFull;
          made = r == 2;
        }
      }
      const unsigned m = __ballot_sync(tmask, made) & tmask;
      if (made) klist[nl + __popc(m & lt)] = (uint16_t)slot;
      nl += __popc(m);
    };
    if (T == 32) {
      // a warp per community: members taken 32 at a time, their entries spread over all lanes
      if (live) {
        for (uint32_t gb = x.mb; gb < x.me; gb += 32) {
          uint32_t rs = 0, len = 0;
          if (gb + lane < x.me) {
            const uint32_t v = D.members[gb + lane];
            rs = D.row[v];
            len = D.row[v + 1] - rs;
          }
          warp_expand_rows_all(rs, len, add);
        }
      }
    } else if (live) {
      for (uint32_t i = x.mb; i < x.me; ++i) {
        const uint32_t v = D.members[i];
        const uint32_t re = D.row[v + 1];
        for (uint32_t eb = D.row[v]; eb < re; eb += T) add(eb + lane, eb + lane < re);
      }
    }
    self_acc = team_sum<T>(self_acc);
    __syncwarp();
    // the listed communities become the output row, in list order; their slots are emptied
    double ksum = 0.0;
    if (live) {
      for (uint32_t i = lane; i < nl; i += T) {
        const uint32_t sl = klist[i];
        uint32_t d;
        Acc sum;
        tbl.load(sl, d, sum);
        tbl.clear(sl);
        Wt wv;
        if (WINT) wv = (Wt)sum;
        else wv = (Wt)__double2float_rn((double)sum);
        D.colB[x.tb + i] = d;
        wout[x.tb + i] = wv;
        ksum += Tr::w_double(wv);
      }
    }
#pragma unroll
    for (int o = T / 2; o > 0; o >>= 1) ksum += __shfl_xor_sync(kFull, ksum, o, T);
    if (live && lane == 0) {
      const bool has_self = self_acc != Acc(0);  // weights are positive
      if (has_self) {
        Wt wv;
        if (WINT) wv = (Wt)self_acc;
        else wv = (Wt)__double2float_rn((double)self_acc);
        D.colB[x.tb + nl] = s;
        wout[x.tb + nl] = wv;
        ksum += Tr::w_double(wv);
        if (WINT) atomicAdd(&D.gs[x.g].I, (unsigned long long)wv);
        else atomicAdd(reinterpret_cast<double*>(&D.gs[x.g].I), Tr::w_double(wv));
      }
      D.newdeg[s] = nl + (has_self ? 1u : 0u);
      D.kB[s] = ksum;
      if (D.gidB) D.gidB[s] = x.g;
    }
    __syncwarp();
  }
  if (err) report_err(C, err, 7);  // k_contract_team
}

// One block per new community of bin 6 (shared-memory table, listed keys as above).
// NT threads per block: 512 for bin 6, 256 for the half-table list (as k_opt_block).
template <bool WINT, int NT = 512>
__global__ void __launch_bounds__(NT) k_contract_block(int dslot, int bin, uint32_t cap) {
  const Dev& D = c_dev[dslot];
  using Tr = WTraits<WINT>;
  using Acc = typename Tr::Acc;
  using Wt = typename Tr::W;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ uint32_t shu[33];
  __shared__ double shd[33];
  __shared__ uint32_t mrs[NT], mex[NT];  // row start / entry offset of the members in flight
  __shared__ uint32_t nlist;
  constexpr size_t kSlotBytes = WINT ? 8 : 4 + sizeof(Acc);
  uint16_t* klist = reinterpret_cast<uint16_t*>(smem + (size_t)cap * kSlotBytes);
  Ctrl* C = D.ctrl;
  const uint32_t count = C->bin_count[bin];
  if (blockIdx.x >= count) return;  // (block-uniform)
  const uint32_t* list = D.bins[bin];
  const Wt* __restrict__ w = reinterpret_cast<const Wt*>(D.w);
  Wt* __restrict__ wout = reinterpret_cast<Wt*>(D.wB);
  const bool unit = unit_weights<WINT>(C);
  const int lane = threadIdx.x & 31;
  const uint32_t lt = lanemask_lt();
  uint32_t err = 0;
  ScratchTable<WINT> tbl{reinterpret_cast<uint32_t*>(smem),
                         reinterpret_cast<Acc*>(smem + (size_t)cap * sizeof(uint32_t)),
                         reinterpret_cast<unsigned long long*>(smem), cap - 1u, 0u};
  for (uint32_t i = threadIdx.x; i < cap; i += NT) tbl.clear(i);
  for (uint32_t idx = blockIdx.x; idx < count; idx += gridDim.x) {
    const uint32_t s = list[idx];
    const CommCtx x = load_comm(D, s);
    const uint32_t cap_v = contract_cap(x.dsum, D.gs[x.g].n_next, false);
    const bool ok = cap_v <= cap;
    tbl.mask = cap_v - 1u;
    tbl.shift = 32u - log2_pow2(cap_v);
    if (!ok) {
      err |= kErrArena;
      if (threadIdx.x == 0 &&
          atomicCAS(&C->err_info[0], 0ull, ((unsigned long long)s << 32) | x.dsum) == 0ull)
        C->err_info[1] = ((unsigned long long)cap_v << 32) | cap;
    }
    if (threadIdx.x == 0) nlist = 0;
    __syncthreads();  // the table is empty and the list count zero
    Acc self_acc = Acc(0);  // entries staying inside the community, kept out of the table
    if (ok) {
      // members taken NT at a time; their entries spread evenly over the whole block, each
      // thread finding its entry's member by binary search in shared memory
      for (uint32_t base = x.mb; base < x.me; base += NT) {
        const uint32_t i = base + threadIdx.x;
        uint32_t rs = 0, len = 0;
        if (i < x.me) {
          const uint32_t v = D.members[i];
          rs = D.row[v];
          len = D.row[v + 1] - rs;
        }
        uint32_t total;
        const uint32_t ex = block_excl_scan<uint32_t, NT>(len, shu, &total);
        mrs[threadIdx.x] = rs;
        mex[threadIdx.x] = ex;
        __syncthreads();
        const uint32_t cnt = min((uint32_t)NT, x.me - base);
        for (uint32_t jb = 0; jb < total; jb += NT) {
          const uint32_t j = jb + threadIdx.x;
          bool made = false;
          uint32_t slot = 0;
          if (j < total) {
            uint32_t lo = 0, hi = cnt;
            while (hi - lo > 1) {
              const uint32_t mid = (lo + hi) >> 1;
              if (mex[mid] <= j) lo = mid; else hi = mid;
            }
            const uint32_t e = mrs[lo] + (j - mex[lo]);
            const uint32_t d = D.new_comm[D.col[e]];
            const Acc wv = unit ? Acc(1) : (Acc)w[e];
            if (d == s) {
              self_acc += wv;
            } else {
              const int r = tbl.add_at(d, wv, slot);
              if (!r) err |= kErrTableFull;
              made = r == 2;
            }
          }
          const unsigned m = __ballot_sync(kFull, made);
          if (m) {
            const int leader = __ffs(m) - 1;
            uint32_t b0 = 0;
            if (lane == leader) b0 = atomicAdd(&nlist, (uint32_t)__popc(m));
            b0 = __shfl_sync(kFull, b0, leader);
            if (made) klist[b0 + __popc(m & lt)] = (uint16_t)slot;
          }
        }
        __syncthreads();
      }
    }
    self_acc = block_sum<NT>(self_acc, reinterpret_cast<Acc*>(shd));  // (its barriers order the list)
    const uint32_t nl = nlist;
    double ksum = 0.0;
    if (ok) {
      for (uint32_t i = threadIdx.x; i < nl; i += NT) {
        const uint32_t sl = klist[i];
        uint32_t d;
        Acc sum;
        tbl.load(sl, d, sum);
        tbl.clear(sl);
        Wt wv;
        if (WINT) wv = (Wt)sum;
        else wv = (Wt)__double2float_rn((double)sum);
        D.colB[x.tb + i] = d;
        wout[x.tb + i] = wv;
        ksum += Tr::w_double(wv);
      }
    }
    double ktot;
    block_excl_scan<double, NT>(ksum, shd, &ktot);
    if (threadIdx.x == 0) {
      const bool has_self = ok && self_acc != Acc(0);  // weights are positive
      if (has_self) {
        Wt wv;
        if (WINT) wv = (Wt)self_acc;
        else wv = (Wt)__double2float_rn((double)self_acc);
        D.colB[x.tb + nl] = s;
        wout[x.tb + nl] = wv;
        ktot += Tr::w_double(wv);
        if (WINT) atomicAdd(&D.gs[x.g].I, (unsigned long long)wv);
        else atomicAdd(reinterpret_cast<double*>(&D.gs[x.g].I), Tr::w_double(wv));
      }
      D.newdeg[s] = ok ? nl + (has_self ? 1u : 0u) : 0u;
      D.kB[s] = ktot;
      if (D.gidB) D.gidB[s] = x.g;
    }
    __syncthreads();
  }
  if (err) report_err(C, err, 8);  // k_contract_block
}

// Copy the gapped contracted rows into the dense next-level CSR (col/w), move k' and gid'.
// The output is cut into chunks of kCompactChunk entries, one block per chunk, so a row of any
// length is copied by as many blocks as it spans; each block stages the offsets (dense and
// gapped) of the rows that overlap its chunk in shared memory and finds every entry's row by
// binary search there. (Warps taking whole rows instead measured 2.8x slower: most contracted
// rows are short.)
constexpr uint32_t kCompactChunk = 2048;

template <bool WINT>
__global__ void __launch_bounds__(256) k_agg_compact(int dslot) {
  const Dev& D = c_dev[dslot];
  using Wt = typename WTraits<WINT>::W;
  __shared__ uint32_t rs[kCompactChunk + 2], src0[kCompactChunk + 1];
  __shared__ uint32_t r0_sh, nr_sh;
  Ctrl* C = D.ctrl;
  const uint32_t n2 = C->n_next;
  const uint32_t E2 = D.rowB[n2];
  const Wt* __restrict__ win = reinterpret_cast<const Wt*>(D.wB);
  Wt* __restrict__ wout = reinterpret_cast<Wt*>(D.w);
  const uint32_t nchunks = (E2 + kCompactChunk - 1) / kCompactChunk;
  for (uint32_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const uint32_t start = ch * kCompactChunk;
    const uint32_t end = min(start + kCompactChunk, E2);
    if (threadIdx.x == 0) {
      uint32_t lo = 0, hi = n2;  // last row with rowB[r] <= start
      while (hi - lo > 1) { const uint32_t mid = (lo + hi) >> 1; if (D.rowB[mid] <= start) lo = mid; else hi = mid; }
      uint32_t r1 = lo;           // first row with rowB[r] >= end
      hi = n2;
      uint32_t lo2 = lo;
      while (hi - lo2 > 1) { const uint32_t mid = (lo2 + hi) >> 1; if (D.rowB[mid] < end) lo2 = mid; else hi = mid; }
      r1 = lo2 + 1;
      r0_sh = lo;
      nr_sh = r1 - lo;  // rows lo..r1-1 overlap the chunk (every row has an entry: <= kCompactChunk)
    }
    __syncthreads();
    const uint32_t r0 = r0_sh, nr = nr_sh;
    for (uint32_t i = threadIdx.x; i <= nr; i += blockDim.x) {
      rs[i] = D.rowB[r0 + i];
      if (i < nr) src0[i] = (uint32_t)D.cd[r0 + i];  // the row's start in the gapped rows
    }
    __syncthreads();
    for (uint32_t p = start + threadIdx.x; p < end; p += blockDim.x) {
      uint32_t lo = 0, hi = nr;  // rs[lo] <= p < rs[lo + 1]
      while (hi - lo > 1) { const uint32_t mid = (lo + hi) >> 1; if (rs[mid] <= p) lo = mid; else hi = mid; }
      const uint32_t src = src0[lo] + (p - rs[lo]);
      D.col[p] = D.colB[src];
      wout[p] = win[src];
    }
    __syncthreads();
  }
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n2; s += gridDim.x * blockDim.x) {
    D.k[s] = D.kB[s];
    if (D.gid) D.gid[s] = D.gidB[s];
  }
}

__global__ void k_agg_finish(int dslot) {
  const Dev& D = c_dev[dslot];
  Ctrl* C = D.ctrl;
  const uint32_t n2 = C->n_next;
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s <= n2; s += gridDim.x * blockDim.x)
    D.row[s] = D.rowB[s];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    C->E_next = D.rowB[n2];
    // per-graph next-level ranges (graphs keep their order; finished graphs drop out)
    for (uint32_t g = 0; g < C->G; ++g) {
      GraphState* st = &D.gs[g];
      if (!st->agg) continue;
      if (st->cont) {
        const uint32_t before = st->vb > 0 ? (uint32_t)D.map[st->vb - 1] : 0u;
        const uint32_t end = (uint32_t)D.map[st->ve - 1];
        st->vb = before;
        st->ve = end;
        st->level += 1;
        st->phase = kIterating;
      } else {
        st->phase = kFinished;
        st->vb = st->ve = 0;
      }
      st->agg = 0;
    }
    C->n = n2;
    C->E = C->E_next;
    C->unit_w = 0;  // contracted weights are sums
    C->seg_levels += 1;
    C->t_agg_ns += global_ns() - C->t_agg0;
  }
}

// Which graphs aggregate now and whether they continue: modularityAlgorithms.h:52
// cont = Q_end - Q_level_start > threshold. force >= 0 overrides (phase-level API).
// defer_i: a refined run resets I in k_ref_decide, once refinement has decided.
__global__ void k_agg_decide(int dslot, int force, uint32_t max_levels, int defer_i) {
  const Dev& D = c_dev[dslot];
  Ctrl* C = D.ctrl;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    C->t_agg0 = global_ns();
    C->seg_aggs += 1;
  }
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < C->G; g += gridDim.x * blockDim.x) {
    GraphState* st = &D.gs[g];
    if (st->phase == kFinished) { st->agg = 0; continue; }
    st->agg = 1;
    uint32_t cont;
    if (force >= 0) cont = (uint32_t)force;
    else cont = __dsub_rn(st->Q, st->Q_level) > C->threshold ? 1u : 0u;
    if (max_levels > 0 && st->level + 1 >= max_levels) cont = 0;
    st->cont = cont;
    if (cont && !defer_i) st->I = 0;  // the contraction adds the next level's self-loop weight
  }
}

// ---- device-sized clears and the gates of a captured run ----------------------------------------
// Aggregation scratch cleared to the level's own sizes (read on the device).
__global__ void k_agg_clear_map(int dslot) {
  const Dev& D = c_dev[dslot];
  const uint32_t n = D.ctrl->n;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) D.map[i] = 0ull;
}
// Before the contraction: per-new-community counters and hub offsets, and the counters the
// binning appends with (so that an aggregation can be run again from its start).
__global__ void k_agg_clear_next(int dslot) {
  const Dev& D = c_dev[dslot];
  Ctrl* C = D.ctrl;
  const uint32_t n2 = C->n_next;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= n2; i += gridDim.x * blockDim.x) {
    D.cd[i] = 0ull;
    if (i < n2) D.hubtab[i] = kEmpty;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    D.newdeg[n2] = 0;
    for (int b = 0; b < kListBins; ++b) C->bin_count[b] = 0;
    C->hub_cursor = 0;
    C->long_count = 0;  // k_hub_insert queues this aggregation's long rows from zero
    C->hub_work = 0;    // and takes its member groups from zero
  }
}
// The global contraction tables of this aggregation: empty keys, zero values.
template <bool WINT>
__global__ void k_arena_clear(int dslot) {
  const Dev& D = c_dev[dslot];
  Ctrl* C = D.ctrl;
  const uint32_t used = min(C->hub_cursor, C->arena_slots);
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < used; s += gridDim.x * blockDim.x)
    arena_clear_slot<WINT>(D, s);
}
// Level body entry: the pass loop runs while some graph iterates.
__global__ void k_gate_pass(int dslot, GraphCtl gc) {
  const Dev& D = c_dev[dslot];
  Ctrl* C = D.ctrl;
  if (C->seg_aggs > kGuardLevels) atomicOr(&C->err, kErrLoop);
  const bool stop = (C->err & kErrLoop) != 0;
  set_cond(gc, gc.pass, C->n_iterating > 0 && !stop);
  if (stop) set_cond(gc, gc.level, false);
}
// After the renumbering: contract (then-branch) when some graph continues, else the run ends.
__global__ void k_gate_contract(int dslot, GraphCtl gc) {
  const Dev& D = c_dev[dslot];
  Ctrl* C = D.ctrl;
  const bool more = C->n_next > 0;
  if (more) C->seg_contract += 1; else C->seg_final += 1;
  const bool stop = (C->err & kErrLoop) != 0;
  set_cond(gc, gc.contract, more && !stop);
  if (!more || stop) set_cond(gc, gc.level, false);
}
// After the contraction binning: its global tables must fit the arena; if not, the run stops
// here (nothing of this aggregation is final yet) and the host grows the arena and redoes it.
__global__ void k_gate_arena_agg(int dslot, GraphCtl gc) {
  const Dev& D = c_dev[dslot];
  Ctrl* C = D.ctrl;
  const bool ok = C->hub_cursor <= C->arena_slots;
  if (ok) {
    C->seg_contract_ok += 1;
  } else {
    C->abort = kAbortAggArena;
    C->abort_need = C->hub_cursor;
    set_cond(gc, gc.level, false);
  }
  set_cond(gc, gc.ok, ok);
}
// End of a level start: the next level's optimisation tables must fit the arena; if not, the
// run stops with the level started and the host grows the arena and resumes.
__global__ void k_gate_level(int dslot, GraphCtl gc) {
  const Dev& D = c_dev[dslot];
  Ctrl* C = D.ctrl;
  const bool ok = C->arena_need <= C->arena_slots;
  if (!ok) {
    C->abort = kAbortOptArena;
    C->abort_need = C->arena_need;
  }
  set_cond(gc, gc.level, ok && !(C->err & kErrLoop));
}

// ---- scans (3-phase: tile sums, scan of tile sums, tile scan + offset) ---------------------------
// The three scans of an aggregation, each named by what it scans so that its arrays and length
// come from the device state (a captured run replays them at every level with every size):
//   kScanMap: map -> map, inclusive, n entries (community renumbering)
//   kScanCd:  cd -> cd, exclusive, n_next + 1 entries (members and degree sums per community)
//   kScanDeg: newdeg -> rowB, exclusive, n_next + 1 entries (next-level row offsets)
// The blocks stride over tiles, so the grid does not depend on the size either.
constexpr int kScanNT = 256;
constexpr int kScanIPT = 8;
constexpr int kScanTile = kScanNT * kScanIPT;
enum : int { kScanMap = 0, kScanCd = 1, kScanDeg = 2 };

template <int SRC>
__device__ __forceinline__ uint32_t scan_len(const Dev& D) {
  return SRC == kScanMap ? D.ctrl->n : D.ctrl->n_next + 1u;
}
template <class T, int SRC>
__device__ __forceinline__ const T* scan_in(const Dev& D) {
  if constexpr (SRC == kScanMap) return reinterpret_cast<const T*>(D.map);
  else if constexpr (SRC == kScanCd) return reinterpret_cast<const T*>(D.cd);
  else return reinterpret_cast<const T*>(D.newdeg);
}
template <class T, int SRC>
__device__ __forceinline__ T* scan_out(const Dev& D) {
  if constexpr (SRC == kScanMap) return reinterpret_cast<T*>(D.map);
  else if constexpr (SRC == kScanCd) return reinterpret_cast<T*>(D.cd);
  else return reinterpret_cast<T*>(D.rowB);
}

template <class T, int SRC>
__global__ void __launch_bounds__(kScanNT) k_scan_tiles(int dslot) {
  const Dev& D = c_dev[dslot];
  __shared__ T sh[33];
  const uint32_t n = scan_len<SRC>(D);
  const uint32_t ntiles = (n + kScanTile - 1) / kScanTile;
  const T* in = scan_in<T, SRC>(D);
  T* tile_sums = reinterpret_cast<T*>(D.scan_tmp);
  for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const uint64_t base = (uint64_t)t * kScanTile;
    T s = T(0);
#pragma unroll
    for (int i = 0; i < kScanIPT; ++i) {
      const uint64_t j = base + (uint64_t)i * kScanNT + threadIdx.x;
      if (j < n) s += in[j];
    }
    T tot;
    block_excl_scan<T, kScanNT>(s, sh, &tot);
    if (threadIdx.x == 0) tile_sums[t] = tot;
  }
}

template <class T, int SRC>
__global__ void __launch_bounds__(1024) k_scan_sums(int dslot) {
  const Dev& D = c_dev[dslot];
  __shared__ T sh[33];
  const uint32_t ntiles = (scan_len<SRC>(D) + kScanTile - 1) / kScanTile;
  T* tile_sums = reinterpret_cast<T*>(D.scan_tmp);
  // each thread scans a contiguous run, then the block scans the run totals
  const uint32_t per = (ntiles + 1023) / 1024;
  const uint32_t b = threadIdx.x * per, e = min(b + per, ntiles);
  T s = T(0);
  for (uint32_t i = b; i < e; ++i) s += tile_sums[i];
  T tot;
  T off = block_excl_scan<T, 1024>(s, sh, &tot);
  for (uint32_t i = b; i < e; ++i) {
    const T x = tile_sums[i];
    tile_sums[i] = off;
    off += x;
  }
}

// inclusive: out[i] = sum in[0..i]; exclusive: out[i] = sum in[0..i-1]. In place is fine: a
// thread reads its own elements before it writes them.
template <class T, int SRC, bool INCLUSIVE>
__global__ void __launch_bounds__(kScanNT) k_scan_apply(int dslot) {
  const Dev& D = c_dev[dslot];
  __shared__ T sh[33];
  const uint32_t n = scan_len<SRC>(D);
  const uint32_t ntiles = (n + kScanTile - 1) / kScanTile;
  const T* in = scan_in<T, SRC>(D);
  T* out = scan_out<T, SRC>(D);
  const T* tile_offs = reinterpret_cast<const T*>(D.scan_tmp);
  for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const uint64_t base = (uint64_t)t * kScanTile + (uint64_t)threadIdx.x * kScanIPT;
    T vals[kScanIPT];
    T s = T(0);
#pragma unroll
    for (int i = 0; i < kScanIPT; ++i) {
      const uint64_t j = base + i;
      vals[i] = j < n ? in[j] : T(0);
      s += vals[i];
    }
    T tot;
    T run = block_excl_scan<T, kScanNT>(s, sh, &tot) + tile_offs[t];
#pragma unroll
    for (int i = 0; i < kScanIPT; ++i) {
      const uint64_t j = base + i;
      if (INCLUSIVE) run += vals[i];
      if (j < n) out[j] = run;
      if (!INCLUSIVE) run += vals[i];
    }
  }
}

}  // namespace lv
