// lv_device.cuh -- device-side building blocks of the B200 Louvain engine: state layout,
// the reference's gain arithmetic, shared-memory hash tables, argmax keys, warp/block
// reductions and scans.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace lv {

constexpr uint32_t kEmpty = 0xFFFFFFFFu;  // empty hash slot / no community
constexpr uint32_t kNever = 0xFFFFFFFFu;  // iteration stamp that never matches
constexpr unsigned kFull = 0xFFFFFFFFu;

// Per-graph phase inside a batch.
enum : uint32_t { kIterating = 0, kLevelDone = 1, kFinished = 2 };

// Device error bits (lv_status LV_ERR_DEVICE_CHECK carries them).
enum : uint32_t {
  kErrTableFull = 1u << 0,    // a hash insert ran out of probes
  kErrArena = 1u << 1,        // a global table slice beyond the arena
  kErrIndex = 1u << 2,        // checked build: an index out of range
  kErrInput = 1u << 3,        // input validation: col out of range / empty row / bad weight
  kErrChunks = 1u << 4,       // more edge chunks than the emulation supports
  kErrRange = 1u << 5,        // integer mode: total weight >= 2^32
  kErrLoop = 1u << 6,         // captured run: pass or level count beyond its guard
};

// Guards of the captured run's device-side loops (far beyond any real run: Louvain's passes
// and levels each raise the modularity by more than the threshold, so both counts are small).
constexpr uint32_t kGuardPasses = 1u << 24;
constexpr uint32_t kGuardLevels = 1u << 16;

constexpr int kMaxChunks = 1024;
constexpr int kNumBins = 8;
// Vertex lists of a pass: the kNumBins degree bins, plus list kHalfBin holding the bin-6 rows
// whose table fits half of the block table (processed by 256-thread blocks, twice as many per SM).
constexpr int kHalfBin = kNumBins;
constexpr int kListBins = kNumBins + 1;
constexpr int kTraceCap = 4096;

// Per-graph state (one entry per graph of a batch; a single run has one).
struct GraphState {
  double m;           // total_weight, fixed at level 0 (graph.cu:81)
  double two_m2;      // (2*m)*m, the denominator as operatorsDelta.h:40 evaluates it
  double Q;           // Community::modularity
  double Q_level;     // modularity at the start of the current level
  unsigned long long I;  // internal weight: u64 (integer mode) or double bits (float mode)
  unsigned long long S;  // sum of squared totals: u64 or double bits
  uint32_t phase;
  uint32_t iters;     // passes in the current level
  uint32_t level;
  uint32_t n_best;    // n_of_best_communities
  uint32_t vb, ve;    // vertex range in the current level
  uint32_t cont;      // aggregation: contract (1) or finish (0)
  uint32_t agg;       // taking part in the running aggregation
  uint32_t map_base;  // aggregation: nonempty communities before this graph
  uint32_t total_iters;
  uint32_t moved;     // moves of the last pass
  uint32_t n_next;    // aggregation: vertices of this graph at the next level
  double inv_m;       // rn(1/m) and rn(1/two_m2), for the gain upper bound only
  double inv_2m2;
};

// Hash-table capacity for a row of d entries in a graph of ng vertices: twice the number of
// distinct keys it can hold (at most min(d, ng)), rounded up to a power of two.
// (2 x the smallest power of two >= k: 2 << ceil(log2 k), from the leading zeros of k - 1;
// k <= 2^30 since rows hold at most 2^30 entries)
__host__ __device__ __forceinline__ uint32_t table_cap(uint32_t d, uint32_t ng) {
  uint32_t k = d < ng ? d : ng;
  if (k < 1) k = 1;
#ifdef __CUDA_ARCH__
  const int lz = __clz((int)(k - 1u));  // 32 when k == 1
#else
  const int lz = k == 1 ? 32 : __builtin_clz(k - 1u);
#endif
  return 2u << (32 - lz);
}

struct TraceRec {
  uint32_t level, iteration, n_moved, pad;
  double internal, sum_a2, modularity, delta;
};

// Device control block: counters, loop state and the active-pass description. Kernels read
// sizes and the iteration stamp from here so that a captured graph can be replayed.
struct Ctrl {
  uint32_t it;                 // global pass stamp
  uint32_t n, E;               // current level sizes
  uint32_t n0;                 // original vertices
  uint32_t G;                  // graphs
  uint32_t n_iterating;        // graphs still in kIterating after the last pass
  uint32_t err;
  uint32_t err_site;           // kernels that reported an error bit (one bit per reporting site)
  unsigned long long err_info[2];  // the first failing check's own details (kernel-specific)
  uint32_t fast;               // 1 = this pass is the per-edge "fast" pass
  uint32_t rule_sort;          // 1 = lowest community wins ties, 0 = highest
  uint32_t unit_w;             // integer mode, level 0: every weight is 1, so no kernel loads w
  uint32_t bin_count[kListBins];
  uint32_t mover_count;        // movers found by team kernels: movers[0, mover_count)
  uint32_t hub_mover_count;    // movers found by block kernels: movers[n - hub_mover_count, n)
  uint32_t long_count;         // aggregation: pieces of long rows for k_hub_insert_long
  uint32_t long_movers;        // pass: team-kernel movers with long rows, for k_apply_long
  uint32_t hub_members;        // aggregation: members of the bin-7 communities, for k_hub_insert
  uint32_t hub_work;           // aggregation: next group of bin-7 members a k_hub_insert warp takes
  uint32_t hub_items;          // pass: pieces of the bin-7 (global-table) vertices' rows
  uint32_t apply_items;        // pass: pieces of the rows of movers found by block kernels
  uint32_t hub_cursor;         // global hash-table arena cursor (slots)
  uint32_t arena_slots;        // arena capacity (slots)
  uint32_t n_next, E_next;     // aggregation outputs
  uint32_t n_chunks;           // chunk early-return emulation (single graph)
  uint32_t chunk_lo[kMaxChunks + 1];
  uint32_t chunk_any[kMaxChunks];
  uint32_t chunk_on;           // emulation active for this level
  uint32_t loop_continue;      // device-side loop control for captured graphs
  uint32_t trace_len;
  uint32_t pass;               // pass index inside the current level
  uint32_t max_iterations;
  uint32_t act_vertices;       // this pass: vertices binned (active and considered)
  unsigned long long act_entries;         // this pass: their entries
  unsigned long long act_vertices_total;  // summed over the run's passes
  unsigned long long act_entries_total;
  double threshold;
  // device-driven runs (a captured graph with conditional nodes): why the graph stopped early
  // (0 none, kAbortAggArena / kAbortOptArena), the arena slots that were needed, per-run counts
  // of the captured segments that ran, and device-clock phase times in ns (%globaltimer)
  uint32_t abort;
  uint32_t pad_abort;
  unsigned long long arena_need;  // slots wanted by the global-table bin at this level start
  unsigned long long abort_need;
  uint32_t seg_levels, seg_passes, seg_aggs, seg_contract, seg_contract_ok, seg_final;
  unsigned long long t_pass0, t_agg0, t_opt_ns, t_optk_ns, t_agg_ns;
  TraceRec trace[kTraceCap];
};

constexpr uint32_t kAbortAggArena = 1;  // aggregation: contraction tables beyond the arena
constexpr uint32_t kAbortOptArena = 2;  // level start: optimisation tables beyond the arena

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Conditional-node handles of a captured run (on = 0: plain stream launches, no handles).
struct GraphCtl {
  unsigned long long level, pass, contract, ok;  // cudaGraphConditionalHandle values
  int on;
};
__device__ __forceinline__ void set_cond(const GraphCtl& gc, unsigned long long h, bool v) {
  if (gc.on) cudaGraphSetConditional((cudaGraphConditionalHandle)h, v ? 1u : 0u);
}

// ---- reference arithmetic -----------------------------------------------------------------
// operatorsDelta.h:29-45 (DeltaModularitySort / DeltaModularityHash): the float difference
// w_vc - self_v, then double: diff/m + k*(a_own - k - a_c)/((2m)m), rounded to float. The
// explicit _rn intrinsics keep every step a single IEEE rounding (no FMA contraction), so the
// result is bit-identical to the reference and to the oracle.
// The two operands of the gain: diff = w_vc - self_v (float) and p = k*((a_own - k) - a_c).
__device__ __forceinline__ double gain_p(double k, double own_minus_k, double a_c) {
  return __dmul_rn(k, __dsub_rn(own_minus_k, a_c));
}
__device__ __forceinline__ float gain_exact(float diff, double p, double m, double two_m2) {
  return __double2float_rn(__dadd_rn(__ddiv_rn((double)diff, m), __ddiv_rn(p, two_m2)));
}
__device__ __forceinline__ float gain_ref(float w_vc, float self_v, double k, double a_own,
                                          double a_c, double m, double two_m2) {
  return gain_exact(__fsub_rn(w_vc, self_v), gain_p(k, __dsub_rn(a_own, k), a_c), m, two_m2);
}

// The reference's gain (gain_exact's float result, bit for bit) without dividing, in almost
// every case. With r1 = rn(1/m) and r2 = rn(1/two_m2) (precomputed per graph), t1 = rn(diff*r1)
// and t2 = rn(p*r2) are each within 3 units of 2^-53 (relative) of the exact quotients
// rn(diff/m) and rn(p/two_m2) (one rounding in the reciprocal, one in the product, one in the
// quotient), so s = rn(t1 + t2) is within 5 * 2^-53 * (|t1| + |t2|) of the reference's double
// sum X. err = 2^-49 * (|t1| + |t2|) + 2^-1000 covers that with room to spare (the absolute
// term covers subnormal results), so X lies in [rd(s - err), ru(s + err)]. Rounding to float is
// monotone: when both ends of that interval round to the same float (compared bit for bit, so
// that -0 and +0 differ), that float is rn_f32(X) -- the test of Ziv's strategy for correctly
// rounded evaluation. Only when X may sit at a float rounding boundary (a relative window of
// about 2^-45 around one of them, so almost never) is the division-based gain_exact evaluated.
__device__ __forceinline__ float gain_fast(float diff, double p, double inv_m, double inv_2m2,
                                           double m, double two_m2) {
  const double t1 = __dmul_rn((double)diff, inv_m);
  const double t2 = __dmul_rn(p, inv_2m2);
  const double err = __fma_rn(__dadd_rn(fabs(t1), fabs(t2)), 0x1p-49, 0x1p-1000);
  const double s = __dadd_rn(t1, t2);
  const float lo = __double2float_rn(__dsub_rd(s, err));
  const float hi = __double2float_rn(__dadd_ru(s, err));
  if (__float_as_uint(lo) == __float_as_uint(hi)) return lo;
  return gain_exact(diff, p, m, two_m2);
}

// Argmax key for a positive gain: the float bits order positive floats, the low word breaks
// ties -- ~c makes the lowest community win (SORT: GetMaxValue keeps the first of equal
// values in ascending community order, operators.h:30-40), c makes the highest win (HASH:
// atomicMax of (gain bits << 32 | c), phaseOptimizationHash.cu:23-35). 0 = no candidate.
__device__ __forceinline__ unsigned long long argmax_key(float g, uint32_t c, bool lowest) {
  return ((unsigned long long)__float_as_uint(g) << 32) | (lowest ? (uint32_t)~c : c);
}
__device__ __forceinline__ uint32_t key_comm(unsigned long long key, bool lowest) {
  const uint32_t lo = (uint32_t)key;
  return lowest ? ~lo : lo;
}
__device__ __forceinline__ float key_gain(unsigned long long key) {
  return __uint_as_float((uint32_t)(key >> 32));
}

// ---- weight types ----------------------------------------------------------------------------
// Integer mode keeps u32 weights and exact u32/u64 sums (the reference's `unsigned` weights);
// float mode keeps fp32 weights and double sums.
template <bool WINT> struct WTraits;
template <> struct WTraits<true> {
  using W = uint32_t;
  using Acc = uint32_t;  // a row's weight sum is at most k_v <= 2m < 2^32
  __device__ static __forceinline__ float to_float(Acc x) { return __uint2float_rn(x); }
  __device__ static __forceinline__ float w_float(W x) { return __uint2float_rn(x); }
  __device__ static __forceinline__ double w_double(W x) { return (double)x; }
};
template <> struct WTraits<false> {
  using W = float;
  using Acc = double;
  __device__ static __forceinline__ float to_float(Acc x) { return __double2float_rn(x); }
  __device__ static __forceinline__ float w_float(W x) { return x; }
  __device__ static __forceinline__ double w_double(W x) { return (double)x; }
};

// ---- hashing -------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t hash_slot(uint32_t c, uint32_t shift) {
  return (c * 2654435761u) >> shift;
}
__device__ __forceinline__ uint32_t log2_pow2(uint32_t x) { return 31u - __clz(x); }
__host__ __device__ __forceinline__ uint32_t next_pow2(uint32_t x) {
  uint32_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

__device__ __forceinline__ void acc_add(uint32_t* p, uint32_t v) { atomicAdd(p, v); }
__device__ __forceinline__ void acc_add(double* p, double v) { atomicAdd(p, v); }

// Open addressing with linear probing; keys go EMPTY -> c once and never change again, so a
// non-empty slot read is final. Capacity >= 2 x inserts, so the probe bound is never reached
// in a correctly sized table; reaching it reports kErrTableFull instead of looping.
template <class Acc>
__device__ __forceinline__ bool table_add(uint32_t* keys, Acc* vals, uint32_t mask,
                                          uint32_t shift, uint32_t c, Acc w) {
  uint32_t h = hash_slot(c, shift);
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    uint32_t cur = ((volatile uint32_t*)keys)[h];
    if (cur == kEmpty) {
      cur = atomicCAS(&keys[h], kEmpty, c);
      if (cur == kEmpty) cur = c;
    }
    if (cur == c) {
      acc_add(&vals[h], w);
      return true;
    }
    h = (h + 1) & mask;
  }
  return false;
}

// The same insert, also telling where the key sits and whether this call created it:
// 0 = no free slot within the probe bound, 1 = the key was there, 2 = this call created it.
template <class Acc>
__device__ __forceinline__ int table_add_at(uint32_t* keys, Acc* vals, uint32_t mask, uint32_t shift,
                                            uint32_t c, Acc w, uint32_t& slot) {
  uint32_t h = hash_slot(c, shift);
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    uint32_t cur = ((volatile uint32_t*)keys)[h];
    int made = 1;
    if (cur == kEmpty) {
      cur = atomicCAS(&keys[h], kEmpty, c);
      if (cur == kEmpty) { cur = c; made = 2; }
    }
    if (cur == c) {
      acc_add(&vals[h], w);
      slot = h;
      return made;
    }
    h = (h + probe + 1u) & mask;  // triangular steps (see PackedTable::add_at)
  }
  return 0;
}

template <class Acc>
__device__ __forceinline__ Acc table_get(const uint32_t* keys, const Acc* vals, uint32_t mask,
                                         uint32_t shift, uint32_t c) {
  uint32_t h = hash_slot(c, shift);
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    const uint32_t cur = keys[h];
    if (cur == c) return vals[h];
    if (cur == kEmpty) return Acc(0);
    h = (h + 1) & mask;
  }
  return Acc(0);
}

// Table views for the insert / scan loops. SplitTable: keys and sums in two arrays (shared-memory
// tables, and global tables with fp32 weights). PackedTable: one u64 per slot, community id in
// the high word and the integer weight sum in the low word (global tables with integer weights:
// every sum is below 2m < 2^32, so adding to the low word never carries into the id); an
// insert is one 64-bit atomic on one 8-byte slot instead of a CAS and an add on two arrays.
constexpr unsigned long long kEmptySlot = 0xFFFFFFFF00000000ull;

template <class Acc>
struct SplitTable {
  uint32_t* keys;
  Acc* vals;
  uint32_t mask, shift;
  __device__ __forceinline__ bool add(uint32_t c, Acc w) const {
    return table_add(keys, vals, mask, shift, c, w);
  }
  __device__ __forceinline__ void load(uint32_t i, uint32_t& k, Acc& v) const {
    k = keys[i];
    v = vals[i];
  }
};

struct PackedTable {
  unsigned long long* slots;
  uint32_t mask, shift;
  __device__ __forceinline__ bool add(uint32_t c, uint32_t w) const {
    return add_from(hash_slot(c, shift), c, w);
  }
  // add() with the probe sequence starting at slot h (the home slot, or one past it)
  __device__ __forceinline__ bool add_from(uint32_t h, uint32_t c, uint32_t w) const {
    for (uint32_t probe = 0; probe <= mask; ++probe) {
      unsigned long long cur = ((volatile unsigned long long*)slots)[h];
      uint32_t key = (uint32_t)(cur >> 32);
      if (key == kEmpty) {
        cur = atomicCAS(&slots[h], kEmptySlot, ((unsigned long long)c << 32) | w);
        if (cur == kEmptySlot) return true;
        key = (uint32_t)(cur >> 32);
      }
      if (key == c) {
        atomicAdd(&slots[h], (unsigned long long)w);
        return true;
      }
      h = (h + 1) & mask;
    }
    return false;
  }
  __device__ __forceinline__ void load(uint32_t i, uint32_t& k, uint32_t& v) const {
    const unsigned long long x = slots[i];
    k = (uint32_t)(x >> 32);
    v = (uint32_t)x;
  }
  // add() that reports the slot and whether this call created the key (as table_add_at).
  // CAS_FIRST tries the CAS without reading the slot before: in a gain pass almost every insert
  // creates its key (a row's neighbours sit in distinct communities), and a CAS that fails
  // returns the slot's content anyway. Otherwise the slot is read first, which saves the failing
  // CAS when keys repeat (contraction: a community's members share neighbouring communities).
  template <bool CAS_FIRST = false>
  __device__ __forceinline__ int add_at(uint32_t c, uint32_t w, uint32_t& slot) const {
    uint32_t h = hash_slot(c, shift);
    for (uint32_t probe = 0; probe <= mask; ++probe) {
      unsigned long long cur;
      if (CAS_FIRST) {
        cur = atomicCAS(&slots[h], kEmptySlot, ((unsigned long long)c << 32) | w);
        if (cur == kEmptySlot) { slot = h; return 2; }
      } else {
        cur = ((volatile unsigned long long*)slots)[h];
        if (cur == kEmptySlot) {
          cur = atomicCAS(&slots[h], kEmptySlot, ((unsigned long long)c << 32) | w);
          if (cur == kEmptySlot) { slot = h; return 2; }
        }
      }
      const uint32_t key = (uint32_t)(cur >> 32);
      if (key == c) {
        atomicAdd(&slots[h], (unsigned long long)w);
        slot = h;
        return 1;
      }
      // triangular steps (offsets 1, 3, 6, ... from the home slot): they visit every slot of a
      // power-of-two table within `mask + 1` probes and break up the runs of occupied slots that
      // linear probing builds, so the longest probe of a warp's inserts -- the one every lane
      // waits for -- stays short
      h = (h + probe + 1u) & mask;
    }
    return 0;
  }
};

// A shared-memory table in the layout of the weight mode: packed slots for integer weights,
// split key / sum arrays for fp32 weights (both 4 + sizeof(sum) bytes per slot on average).
template <bool WINT>
struct ScratchTable {
  using Acc = typename WTraits<WINT>::Acc;
  uint32_t* keys;              // split layout
  Acc* vals;
  unsigned long long* slots;   // packed layout
  uint32_t mask, shift;
  __device__ __forceinline__ void clear(uint32_t i) const {
    if constexpr (WINT) {
      slots[i] = kEmptySlot;
    } else {
      keys[i] = kEmpty;
      vals[i] = Acc(0);
    }
  }
  __device__ __forceinline__ bool add(uint32_t c, Acc w) const {
    if constexpr (WINT) return PackedTable{slots, mask, shift}.add(c, w);
    else return table_add(keys, vals, mask, shift, c, w);
  }
  template <bool CAS_FIRST = false>
  __device__ __forceinline__ int add_at(uint32_t c, Acc w, uint32_t& slot) const {
    if constexpr (WINT) return PackedTable{slots, mask, shift}.template add_at<CAS_FIRST>(c, w, slot);
    else return table_add_at(keys, vals, mask, shift, c, w, slot);
  }
  __device__ __forceinline__ void load(uint32_t i, uint32_t& k, Acc& v) const {
    if constexpr (WINT) {
      const unsigned long long x = slots[i];
      k = (uint32_t)(x >> 32);
      v = (uint32_t)x;
    } else {
      k = keys[i];
      v = vals[i];
    }
  }
};

// ---- warp / block reductions -------------------------------------------------------------------
template <int T>
__device__ __forceinline__ unsigned long long team_max(unsigned long long x, unsigned mask) {
#pragma unroll
  for (int o = T / 2; o > 0; o >>= 1) {
    const unsigned long long y = __shfl_xor_sync(mask, x, o);
    x = y > x ? y : x;
  }
  return x;
}

// Load-balanced walk over the rows of up to 32 vertices held one per lane: calls
// f(entry index, pa, pb) for every entry of every row -- pa/pb being the payload of the lane
// that owns the row -- with all 32 lanes busy however the row lengths are spread. Lane i holds
// (rs_i, len_i, pa_i, pb_i); every lane of the warp must call it.
template <class F>
__device__ __forceinline__ void warp_expand_rows(uint32_t rs, uint32_t len, uint32_t pa, uint32_t pb,
                                                 F&& f) {
  const int lane = threadIdx.x & 31;
  uint32_t incl = len;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += y;
  }
  const uint32_t total = __shfl_sync(kFull, incl, 31);
  const uint32_t excl = incl - len;
  for (uint32_t jb = 0; jb < total; jb += 32) {
    const uint32_t j = jb + lane;
    // owner lane: the last lane whose exclusive offset is <= j
    int k = 0;
#pragma unroll
    for (int step = 16; step >= 1; step >>= 1) {
      const uint32_t ex = __shfl_sync(kFull, excl, k + step);
      if (ex <= j) k += step;
    }
    const uint32_t base = __shfl_sync(kFull, rs, k) - __shfl_sync(kFull, excl, k);
    const uint32_t a = __shfl_sync(kFull, pa, k), b = __shfl_sync(kFull, pb, k);
    if (j < total) f(base + j, a, b);
  }
}

// warp_expand_rows that calls f(entry index, valid) on every lane in every step (lanes past
// the last entry with valid = false), so that f may use warp-wide votes.
template <class F>
__device__ __forceinline__ void warp_expand_rows_all(uint32_t rs, uint32_t len, F&& f) {
  const int lane = threadIdx.x & 31;
  uint32_t incl = len;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += y;
  }
  const uint32_t total = __shfl_sync(kFull, incl, 31);
  const uint32_t excl = incl - len;
  for (uint32_t jb = 0; jb < total; jb += 32) {
    const uint32_t j = jb + lane;
    int k = 0;
#pragma unroll
    for (int step = 16; step >= 1; step >>= 1) {
      const uint32_t ex = __shfl_sync(kFull, excl, k + step);
      if (ex <= j) k += step;
    }
    const uint32_t base = __shfl_sync(kFull, rs, k) - __shfl_sync(kFull, excl, k);
    f(base + j, j < total);
  }
}

// The same with three payload words per row: f(entry index, pa, pb, pc).
template <class F>
__device__ __forceinline__ void warp_expand_rows3(uint32_t rs, uint32_t len, uint32_t pa, uint32_t pb,
                                                  uint32_t pc, F&& f) {
  const int lane = threadIdx.x & 31;
  uint32_t incl = len;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += y;
  }
  const uint32_t total = __shfl_sync(kFull, incl, 31);
  const uint32_t excl = incl - len;
  for (uint32_t jb = 0; jb < total; jb += 32) {
    const uint32_t j = jb + lane;
    int k = 0;
#pragma unroll
    for (int step = 16; step >= 1; step >>= 1) {
      const uint32_t ex = __shfl_sync(kFull, excl, k + step);
      if (ex <= j) k += step;
    }
    const uint32_t base = __shfl_sync(kFull, rs, k) - __shfl_sync(kFull, excl, k);
    const uint32_t a = __shfl_sync(kFull, pa, k), b = __shfl_sync(kFull, pb, k),
                   c = __shfl_sync(kFull, pc, k);
    if (j < total) f(base + j, a, b, c);
  }
}

// Sum over the aligned group of T lanes (every lane of the warp must call it).
template <int T, class V>
__device__ __forceinline__ V team_sum(V x) {
#pragma unroll
  for (int o = T / 2; o > 0; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
  return x;
}

template <class T>
__device__ __forceinline__ T warp_sum(T x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
  return x;
}

template <class T>
__device__ __forceinline__ T warp_incl_scan(T x, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T y = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += y;
  }
  return x;
}

// Exclusive block scan; every thread of the block must call it. `sh` holds >= 33 T.
template <class T, int NT>
__device__ __forceinline__ T block_excl_scan(T x, T* sh, T* total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const T inc = warp_incl_scan(x, lane);
  if (lane == 31) sh[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    T s = lane < NT / 32 ? sh[lane] : T(0);
    s = warp_incl_scan(s, lane);
    if (lane < NT / 32) sh[lane] = s;
    if (lane == NT / 32 - 1) sh[32] = s;
  }
  __syncthreads();
  const T base = wid > 0 ? sh[wid - 1] : T(0);
  if (total) *total = sh[32];
  const T out = base + inc - x;
  __syncthreads();
  return out;
}

}  // namespace lv
