// lv_ingest.cuh -- edge-list text to symmetric CSR on the GPU (lv_ingest_* in
// include/louvain_b200.h). Included at the end of lv_engine.cu.
//
// The reference reads a graph with GraphHost(name, weighted = false, skip_line) (graph.cu:17-87):
// skip `skip_line` lines, then read integers pairwise (`while (f >> a >> b)`) until the first
// failed extraction, collect the distinct unordered pairs (self-loop pairs included) and the
// distinct ids, and emit every pair in both directions with weight 1; GraphDevice later indexes
// vertices by id - min_id (graph.cuh:60-91), so ids must be contiguous. It runs on one host
// thread through std::set and dominates the reference's wall-clock on large graphs (outside
// its timed window). Here the same result is built on the device:
//   tokens   : per-thread byte chunks count token starts, a scan places them, one thread per
//              token parses it (optional sign and decimal digits, int32 range); the input ends
//              at the first token that is not an integer, and an unpaired last token is dropped
//   ids      : min / max reduction; every pair counts one entry into the row of each end,
//              and every id in [min, max] must have a row (ids must be contiguous)
//   rows     : a scan of the counts places the rows; every pair writes each end into the
//              other's row (a self-loop pair writes its id twice into its own row)
//   CSR      : each row sorted and deduplicated on its own -- a warp bitonic sort in registers
//              for rows of up to 32 entries (one per lane), 256 (eight per lane) and 1024 (32
//              per lane), a block bitonic sort in shared memory up to kIngestBlockRow, and above
//              that a bitmap of the row's id range in global memory
//              whose set bits read out in order are the sorted distinct ids; a row keeps its
//              own id twice when the graph has that self-loop pair (graph.cu:68-79 emits both
//              directions of it); a second scan of the row lengths gives the row offsets
// Every scan is the file's own (k_iscan_*), so no library sort or scan is on this path.
#pragma once

namespace lv {

constexpr uint32_t kIngestChunk = 64;  // bytes per thread when counting token starts

__device__ __forceinline__ bool is_space(unsigned char c) {
  return c == ' ' || c == '\n' || c == '\t' || c == '\r' || c == '\v' || c == '\f';
}

__global__ void k_tok_count(const unsigned char* text, uint64_t len, uint32_t* counts, uint64_t nchunks) {
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < nchunks;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t b = t * kIngestChunk, e = min(len, b + kIngestChunk);
    bool prev_space = b == 0 ? true : is_space(text[b - 1]);
    uint32_t c = 0;
    for (uint64_t i = b; i < e; ++i) {
      const bool sp = is_space(text[i]);
      c += (!sp && prev_space);
      prev_space = sp;
    }
    counts[t] = c;
  }
}

__global__ void k_tok_place(const unsigned char* text, uint64_t len, const uint32_t* offs, uint64_t nchunks,
                            uint64_t* pos) {
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < nchunks;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t b = t * kIngestChunk, e = min(len, b + kIngestChunk);
    bool prev_space = b == 0 ? true : is_space(text[b - 1]);
    uint32_t o = offs[t];
    for (uint64_t i = b; i < e; ++i) {
      const bool sp = is_space(text[i]);
      if (!sp && prev_space) pos[o++] = i;
      prev_space = sp;
    }
  }
}

// Token k -> its value; the first token that is not an int32 is recorded in *first_bad.
__global__ void k_tok_parse(const unsigned char* text, uint64_t len, const uint64_t* pos, uint64_t ntok,
                            int32_t* val, unsigned long long* first_bad) {
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < ntok;
       k += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t i = pos[k];
    bool neg = false;
    if (text[i] == '-' || text[i] == '+') {
      neg = text[i] == '-';
      ++i;
    }
    long long v = 0;
    int digits = 0;
    bool ok = true;
    while (i < len && !is_space(text[i])) {
      const unsigned char c = text[i];
      if (c < '0' || c > '9' || digits >= 11) { ok = false; break; }
      v = v * 10 + (c - '0');
      ++digits;
      ++i;
    }
    if (neg) v = -v;
    ok = ok && digits > 0 && v >= INT32_MIN && v <= INT32_MAX;
    if (ok) val[k] = (int32_t)v;
    else atomicMin(first_bad, (unsigned long long)k);
  }
}

__global__ void k_ids_minmax(const int32_t* val, uint64_t nt, int* mn, int* mx) {
  int lo = INT32_MAX, hi = INT32_MIN;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < nt; k += (uint64_t)gridDim.x * blockDim.x) {
    lo = min(lo, val[k]);
    hi = max(hi, val[k]);
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(kFull, lo, o));
    hi = max(hi, __shfl_xor_sync(kFull, hi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(mn, lo);
    atomicMax(mx, hi);
  }
}

// ---- device-wide exclusive scan (u32 in, T out) over tiles of kIScanTile elements ------------
constexpr int kIScanNT = 256;
constexpr int kIScanPer = 8;
constexpr uint32_t kIScanTile = kIScanNT * kIScanPer;

template <class T>
__global__ void __launch_bounds__(kIScanNT) k_iscan_tiles(const uint32_t* in, uint64_t n, T* tile_sums) {
  __shared__ T sh[33];
  const uint64_t ntiles = (n + kIScanTile - 1) / kIScanTile;
  for (uint64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const uint64_t b = t * kIScanTile + (uint64_t)threadIdx.x * kIScanPer;
    T x = 0;
#pragma unroll
    for (int i = 0; i < kIScanPer; ++i)
      if (b + i < n) x += (T)in[b + i];
    T tot;
    block_excl_scan<T, kIScanNT>(x, sh, &tot);
    if (threadIdx.x == 0) tile_sums[t] = tot;
  }
}

// One block: tile sums -> exclusive tile offsets (in place); *total = the sum of everything.
template <class T>
__global__ void __launch_bounds__(1024) k_iscan_sums(T* tile_sums, uint64_t ntiles, T* total) {
  __shared__ T sh[33];
  const uint64_t per = (ntiles + 1023) / 1024;
  const uint64_t b = (uint64_t)threadIdx.x * per, e = min(ntiles, b + per);
  T x = 0;
  for (uint64_t i = b; i < e; ++i) x += tile_sums[i];
  T tot;
  T run = block_excl_scan<T, 1024>(x, sh, &tot);
  for (uint64_t i = b; i < e; ++i) {
    const T y = tile_sums[i];
    tile_sums[i] = run;
    run += y;
  }
  if (threadIdx.x == 0) *total = tot;
}

template <class T>
__global__ void __launch_bounds__(kIScanNT) k_iscan_apply(const uint32_t* in, uint64_t n, const T* tile_offs,
                                                          T* out) {
  __shared__ T sh[33];
  const uint64_t ntiles = (n + kIScanTile - 1) / kIScanTile;
  for (uint64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const uint64_t b = t * kIScanTile + (uint64_t)threadIdx.x * kIScanPer;
    T v[kIScanPer];
    T x = 0;
#pragma unroll
    for (int i = 0; i < kIScanPer; ++i) {
      v[i] = b + i < n ? (T)in[b + i] : T(0);
      x += v[i];
    }
    T run = block_excl_scan<T, kIScanNT>(x, sh, nullptr) + tile_offs[t];
#pragma unroll
    for (int i = 0; i < kIScanPer; ++i)
      if (b + i < n) {
        out[b + i] = run;
        run += v[i];
      }
  }
}

// ---- rows ----------------------------------------------------------------------------------
// Entries per row: each pair puts one entry into the row of each end (ids relative to the
// minimum); a row with no entry means a missing id. Lanes of a warp that add to the same row
// (hub rows of a skewed graph are hit often) combine their counts into one atomic.
__device__ __forceinline__ void warp_add_row(uint32_t* cnt, uint32_t r) {
  const unsigned m = __match_any_sync(__activemask(), r);
  if ((int)(threadIdx.x & 31) == __ffs(m) - 1) atomicAdd(&cnt[r], (uint32_t)__popc(m));
}
// The position of this lane's entry in row r: one atomic per group of lanes writing row r.
__device__ __forceinline__ uint32_t warp_claim_row(uint32_t* cursor, uint32_t r) {
  const unsigned m = __match_any_sync(__activemask(), r);
  const int leader = __ffs(m) - 1;
  uint32_t base = 0;
  if ((int)(threadIdx.x & 31) == leader) base = atomicAdd(&cursor[r], (uint32_t)__popc(m));
  base = __shfl_sync(m, base, leader);
  return base + __popc(m & lanemask_lt());
}

__global__ void k_pair_count(const int32_t* val, uint64_t npairs, int mn, uint32_t* cnt) {
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < npairs;
       p += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t a = (uint32_t)((long long)val[2 * p] - mn), b = (uint32_t)((long long)val[2 * p + 1] - mn);
    warp_add_row(cnt, a);
    warp_add_row(cnt, b);
  }
}

__global__ void k_count_present(const uint32_t* cnt, uint64_t range, unsigned long long* count) {
  unsigned long long c = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < range; i += (uint64_t)gridDim.x * blockDim.x)
    c += cnt[i] != 0u;
  c = warp_sum(c);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

// Every pair writes each end into the other end's row (cursor starts at the row starts).
__global__ void k_pair_scatter(const int32_t* val, uint64_t npairs, int mn, uint32_t* cursor, uint32_t* buf) {
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < npairs;
       p += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t a = (uint32_t)((long long)val[2 * p] - mn), b = (uint32_t)((long long)val[2 * p + 1] - mn);
    buf[warp_claim_row(cursor, a)] = b;
    buf[warp_claim_row(cursor, b)] = a;
  }
}

constexpr uint32_t kIngestWarpRow = 32;     // rows sorted by one warp, one entry per lane
constexpr uint32_t kIngestWarp8Row = 256;   // rows sorted by one warp, eight entries per lane
constexpr uint32_t kIngestWarp32Row = 1024; // rows sorted by one warp, 32 entries per lane
constexpr uint32_t kIngestBlockRow = 4096;  // rows sorted by one block in shared memory
constexpr int kIngestBlockNT = 512;

// Rows longer than a warp's: appended to the block list (counts[0]), the bitmap list
// (counts[1]), the eight-per-lane list (counts[2]) or the 32-per-lane list (counts[3]).
__global__ void k_rows_classify(const uint32_t* cnt, uint32_t range, uint32_t* mid, uint32_t* big,
                                uint32_t* mid8, uint32_t* mid32, uint32_t* counts) {
  for (uint32_t base = blockIdx.x * blockDim.x; base < range; base += gridDim.x * blockDim.x) {
    const uint32_t v = base + threadIdx.x;
    const uint32_t c = v < range ? cnt[v] : 0u;
    const int cls = c > kIngestBlockRow ? 1
                    : c > kIngestWarp32Row ? 0
                    : c > kIngestWarp8Row ? 3
                    : c > kIngestWarpRow ? 2 : -1;
    uint32_t* lists[4] = {mid, big, mid8, mid32};
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const uint32_t pos = warp_append(cls, b, &counts[b]);
      if (pos != kEmpty) lists[b][pos] = v;
    }
  }
}

// Rows of up to 32 * PER entries, one warp each: the row padded to 32 * PER held as PER
// registers per lane (element q * 32 + lane in register q), sorted by a bitonic network whose
// partners at distance 32 and more sit in the lane's own registers and below 32 in another
// lane's (shuffles); then the distinct ids in order, the row's own id twice, back at the row's
// start. `rows` lists the rows (count *n_rows).
template <int PER>
__global__ void k_rows_warpn(const uint32_t* start, const uint32_t* cnt, const uint32_t* rows,
                             const uint32_t* n_rows, uint32_t* buf, uint32_t* ulen) {
  constexpr int P = 32 * PER;
  const int lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t nr = *n_rows;
  for (uint32_t r = warp; r < nr; r += nwarps) {
    const uint32_t v = rows[r];
    const uint32_t c = cnt[v], s0 = start[v];
    uint32_t x[PER];
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const uint32_t i = (uint32_t)q * 32u + lane;
      x[q] = i < c ? buf[s0 + i] : kEmpty;
    }
#pragma unroll
    for (int k = 2; k <= P; k <<= 1) {
#pragma unroll
      for (int j = k >> 1; j > 0; j >>= 1) {
        if (j >= 32) {
          const int jq = j >> 5;
#pragma unroll
          for (int q = 0; q < PER; ++q) {
            if (q & jq) continue;
            const int q2 = q | jq;
            const bool up = ((q * 32 + lane) & k) == 0;
            const uint32_t a = x[q], b = x[q2];
            if ((a > b) == up) { x[q] = b; x[q2] = a; }
          }
        } else {
#pragma unroll
          for (int q = 0; q < PER; ++q) {
            const uint32_t y = __shfl_xor_sync(kFull, x[q], j);
            const bool up = ((q * 32 + lane) & k) == 0, low = (lane & j) == 0;
            x[q] = (low == up) ? min(x[q], y) : max(x[q], y);
          }
        }
      }
    }
    // distinct ids in element order: the previous element of q*32+lane is lane-1 in register q,
    // or for lane 0 lane 31 in register q-1
    uint32_t emit[PER], off[PER];
    uint32_t run = 0;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const uint32_t up1 = __shfl_up_sync(kFull, x[q], 1);
      const uint32_t last_prev = q > 0 ? __shfl_sync(kFull, x[q > 0 ? q - 1 : 0], 31) : kEmpty;
      const uint32_t prev = lane > 0 ? up1 : last_prev;
      const bool first = q == 0 && lane == 0;
      const bool keep = x[q] != kEmpty && (first || x[q] != prev);
      emit[q] = keep ? (x[q] == v ? 2u : 1u) : 0u;
      const uint32_t incl = warp_incl_scan(emit[q], lane);
      off[q] = run + incl - emit[q];
      run += __shfl_sync(kFull, incl, 31);
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < PER; ++q)
      for (uint32_t t = 0; t < emit[q]; ++t) buf[s0 + off[q] + t] = x[q];
    if (lane == 0) ulen[v] = run;
  }
}

// Rows of up to 32 entries, one warp each: bitonic sort across the lanes, then the distinct
// ids written back to the row's start in order (the row's own id twice), length to ulen.
__global__ void k_rows_warp(const uint32_t* start, const uint32_t* cnt, uint32_t range, uint32_t* buf,
                            uint32_t* ulen) {
  const int lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t v = warp; v < range; v += nwarps) {
    const uint32_t c = cnt[v];
    if (c > kIngestWarpRow) continue;  // (warp-uniform)
    const uint32_t s0 = start[v];
    uint32_t x = (uint32_t)lane < c ? buf[s0 + lane] : kEmpty;
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
      for (int j = k >> 1; j > 0; j >>= 1) {
        const uint32_t y = __shfl_xor_sync(kFull, x, j);
        const bool up = (lane & k) == 0, low = (lane & j) == 0;
        x = (low == up) ? min(x, y) : max(x, y);
      }
    }
    const uint32_t prev = __shfl_up_sync(kFull, x, 1);
    const bool keep = x != kEmpty && (lane == 0 || x != prev);
    const uint32_t emit = keep ? (x == v ? 2u : 1u) : 0u;
    const uint32_t incl = warp_incl_scan(emit, lane);
    const uint32_t tot = __shfl_sync(kFull, incl, 31);
    __syncwarp();
    for (uint32_t i = 0; i < emit; ++i) buf[s0 + incl - emit + i] = x;
    if (lane == 0) ulen[v] = tot;
  }
}

// Rows of 1025..kIngestBlockRow entries, one block each: bitonic sort in shared memory.
__global__ void __launch_bounds__(kIngestBlockNT) k_rows_block(const uint32_t* start, const uint32_t* cnt,
                                                               const uint32_t* mid, const uint32_t* counts,
                                                               uint32_t* buf, uint32_t* ulen) {
  __shared__ uint32_t sv[kIngestBlockRow];
  __shared__ uint32_t sh[33];
  constexpr uint32_t PER = kIngestBlockRow / kIngestBlockNT;
  const uint32_t nmid = counts[0];
  for (uint32_t r = blockIdx.x; r < nmid; r += gridDim.x) {
    const uint32_t v = mid[r];
    const uint32_t c = cnt[v], s0 = start[v];
    uint32_t P = 64;
    while (P < c) P <<= 1;
    for (uint32_t i = threadIdx.x; i < P; i += kIngestBlockNT) sv[i] = i < c ? buf[s0 + i] : kEmpty;
    __syncthreads();
    for (uint32_t k = 2; k <= P; k <<= 1) {
      for (uint32_t j = k >> 1; j > 0; j >>= 1) {
        for (uint32_t i = threadIdx.x; i < P; i += kIngestBlockNT) {
          const uint32_t ixj = i ^ j;
          if (ixj > i) {
            const uint32_t a = sv[i], b = sv[ixj];
            const bool up = (i & k) == 0;
            if ((a > b) == up) {
              sv[i] = b;
              sv[ixj] = a;
            }
          }
        }
        __syncthreads();
      }
    }
    // thread t owns elements [t*PER, t*PER + PER) of the sorted row
    uint32_t emit = 0;
    const uint32_t b0 = threadIdx.x * PER;
#pragma unroll
    for (uint32_t i = 0; i < PER; ++i) {
      const uint32_t q = b0 + i;
      if (q < P) {
        const uint32_t x = sv[q];
        if (x != kEmpty && (q == 0 || sv[q - 1] != x)) emit += x == v ? 2u : 1u;
      }
    }
    uint32_t tot;
    uint32_t off = block_excl_scan<uint32_t, kIngestBlockNT>(emit, sh, &tot);
#pragma unroll
    for (uint32_t i = 0; i < PER; ++i) {
      const uint32_t q = b0 + i;
      if (q < P) {
        const uint32_t x = sv[q];
        if (x != kEmpty && (q == 0 || sv[q - 1] != x)) {
          buf[s0 + off++] = x;
          if (x == v) buf[s0 + off++] = x;
        }
      }
    }
    if (threadIdx.x == 0) ulen[v] = tot;
    __syncthreads();
  }
}

// Rows above kIngestBlockRow entries, one block each with its own bitmap (bmw words) of the
// row's id range [lo, hi]: set bits, then read them out in order.
__global__ void __launch_bounds__(kIngestBlockNT) k_rows_bitmap(const uint32_t* start, const uint32_t* cnt,
                                                                const uint32_t* big, const uint32_t* counts,
                                                                uint32_t* bitmaps, uint64_t bmw,
                                                                uint32_t* buf, uint32_t* ulen) {
  __shared__ uint32_t sh[33];
  __shared__ uint32_t lo_sh, hi_sh;
  uint32_t* bm = bitmaps + (uint64_t)blockIdx.x * bmw;
  const uint32_t nbig = counts[1];
  for (uint32_t r = blockIdx.x; r < nbig; r += gridDim.x) {
    const uint32_t v = big[r];
    const uint32_t c = cnt[v], s0 = start[v];
    uint32_t lo = kEmpty, hi = 0;
    for (uint32_t i = threadIdx.x; i < c; i += kIngestBlockNT) {
      const uint32_t x = buf[s0 + i];
      lo = min(lo, x);
      hi = max(hi, x);
    }
    for (int o = 16; o > 0; o >>= 1) {
      lo = min(lo, __shfl_xor_sync(kFull, lo, o));
      hi = max(hi, __shfl_xor_sync(kFull, hi, o));
    }
    if (threadIdx.x == 0) { lo_sh = kEmpty; hi_sh = 0; }
    __syncthreads();
    if ((threadIdx.x & 31) == 0) { atomicMin(&lo_sh, lo); atomicMax(&hi_sh, hi); }
    __syncthreads();
    lo = lo_sh;
    hi = hi_sh;
    const uint32_t words = ((hi - lo) >> 5) + 1;  // <= bmw
    for (uint32_t i = threadIdx.x; i < words; i += kIngestBlockNT) bm[i] = 0u;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < c; i += kIngestBlockNT) {
      const uint32_t d = buf[s0 + i] - lo;
      atomicOr(&bm[d >> 5], 1u << (d & 31));
    }
    __syncthreads();
    // thread t reads a contiguous run of words; counts, block scan, then the ids in order
    const uint32_t per = (words + kIngestBlockNT - 1) / kIngestBlockNT;
    const uint32_t w0 = threadIdx.x * per, w1 = min(words, w0 + per);
    const uint32_t self_w = v >= lo && v <= hi ? (v - lo) >> 5 : kEmpty;
    uint32_t emit = 0;
    for (uint32_t i = w0; i < w1; ++i) {
      const uint32_t m = bm[i];
      emit += __popc(m);
      if (i == self_w && ((m >> ((v - lo) & 31)) & 1u)) emit += 1;  // the self-loop twice
    }
    uint32_t tot;
    uint32_t off = block_excl_scan<uint32_t, kIngestBlockNT>(emit, sh, &tot);
    __syncthreads();  // every id was read into the bitmap before any is overwritten
    for (uint32_t i = w0; i < w1; ++i) {
      uint32_t m = bm[i];
      while (m) {
        const uint32_t bit = __ffs(m) - 1;
        m &= m - 1;
        const uint32_t x = lo + (i << 5) + bit;
        buf[s0 + off++] = x;
        if (x == v) buf[s0 + off++] = x;
      }
    }
    if (threadIdx.x == 0) ulen[v] = tot;
    __syncthreads();
  }
}

// Distinct, sorted rows (at their bucket starts) -> the dense CSR. The output is cut into chunks
// of kRowsCopyChunk entries, one block per chunk: the block stages the dense and bucket starts
// of the rows that overlap its chunk and finds each entry's row by binary search there (most
// rows are short, so a warp per row would leave most lanes idle).
constexpr uint32_t kRowsCopyChunk = 2048;

__global__ void __launch_bounds__(256) k_rows_copy(const uint32_t* start, const int64_t* row_ptr, uint32_t range,
                                                   uint64_t ne, const uint32_t* buf, int32_t* col) {
  __shared__ uint32_t rs[kRowsCopyChunk + 2], src0[kRowsCopyChunk + 1];
  __shared__ uint32_t r0_sh, nr_sh;
  const uint64_t nchunks = (ne + kRowsCopyChunk - 1) / kRowsCopyChunk;
  for (uint64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const uint32_t cs = (uint32_t)(ch * kRowsCopyChunk);
    const uint32_t ce = (uint32_t)min((uint64_t)cs + kRowsCopyChunk, ne);
    if (threadIdx.x == 0) {
      uint32_t lo = 0, hi = range;  // last row with row_ptr[r] <= cs
      while (hi - lo > 1) { const uint32_t mid = (lo + hi) >> 1; if ((uint64_t)row_ptr[mid] <= cs) lo = mid; else hi = mid; }
      uint32_t lo2 = lo;            // last row with row_ptr[r] < ce
      hi = range;
      while (hi - lo2 > 1) { const uint32_t mid = (lo2 + hi) >> 1; if ((uint64_t)row_ptr[mid] < ce) lo2 = mid; else hi = mid; }
      r0_sh = lo;
      nr_sh = lo2 + 1 - lo;  // every row has an entry, so at most kRowsCopyChunk rows
    }
    __syncthreads();
    const uint32_t r0 = r0_sh, nr = nr_sh;
    for (uint32_t i = threadIdx.x; i <= nr; i += blockDim.x) {
      rs[i] = (uint32_t)row_ptr[r0 + i];
      if (i < nr) src0[i] = start[r0 + i];
    }
    __syncthreads();
    for (uint32_t p = cs + threadIdx.x; p < ce; p += blockDim.x) {
      uint32_t lo = 0, hi = nr;  // rs[lo] <= p < rs[lo + 1]
      while (hi - lo > 1) { const uint32_t mid = (lo + hi) >> 1; if (rs[mid] <= p) lo = mid; else hi = mid; }
      col[p] = (int32_t)buf[src0[lo] + (p - rs[lo])];
    }
    __syncthreads();
  }
}

}  // namespace lv

struct lv_ingest {
  lv_context* ctx = nullptr;
  int64_t n = 0, n_links = 0, E = 0, min_id = 0;
  int64_t* row_ptr = nullptr;  // device, n + 1
  int32_t* col = nullptr;      // device, E
};

namespace lv {

// A device allocation of a single temporary buffer (plain cudaMalloc/cudaFree: ingest runs
// once per graph, outside the engine's pool).
struct DevBuf {
  void* p = nullptr;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { reset(); }
  void reset() {
    if (p) cudaFree(p);
    p = nullptr;
  }
  template <class T>
  T* alloc(size_t count) {
    reset();
    LV_CUDA(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)));
    return reinterpret_cast<T*>(p);
  }
};

// Exclusive scan of n u32 counts into out (T = u32 or i64): tile sums, one block over them,
// then each tile again with its offset. `tmp` holds the tile sums.
template <class T>
static void iscan(lv_context* ctx, cudaStream_t st, DevBuf& tmp, const uint32_t* in, uint64_t n, T* out) {
  const uint64_t ntiles = (n + kIScanTile - 1) / kIScanTile;
  T* sums = tmp.alloc<T>(ntiles + 1);
  const unsigned grid = (unsigned)std::min<uint64_t>(ntiles, (uint64_t)ctx->sms * 8);
  k_iscan_tiles<T><<<grid, kIScanNT, 0, st>>>(in, n, sums);
  k_iscan_sums<T><<<1, 1024, 0, st>>>(sums, ntiles, sums + ntiles);
  k_iscan_apply<T><<<grid, kIScanNT, 0, st>>>(in, n, sums, out);
}

static void ingest_run(lv_context* ctx, const char* text_in, int64_t len, int32_t skip_line, int32_t in_mem,
                       lv_ingest* out) {
  cudaStream_t st = ctx->stream;
  const int grid = ctx->sms * 8;
  // skip the header lines (std::getline semantics: up to and including '\n')
  int64_t start = 0;
  if (skip_line > 0) {
    std::vector<char> host;
    const char* h = text_in;
    if (in_mem == LV_MEM_DEVICE) {
      // the header is at the front: copy a growing prefix until enough newlines are seen
      int64_t got = std::min<int64_t>(len, 1 << 20);
      for (;;) {
        host.resize((size_t)got);
        LV_CUDA(cudaMemcpy(host.data(), text_in, (size_t)got, cudaMemcpyDeviceToHost));
        int seen = 0;
        int64_t i = 0;
        for (; i < got && seen < skip_line; ++i)
          if (host[(size_t)i] == '\n') ++seen;
        if (seen == skip_line || got == len) { start = seen == skip_line ? i : got; break; }
        got = std::min<int64_t>(len, got * 4);
      }
    } else {
      int seen = 0;
      int64_t i = 0;
      for (; i < len && seen < skip_line; ++i)
        if (h[i] == '\n') ++seen;
      start = i;
    }
  }
  const uint64_t L = (uint64_t)(len - start);
  if (L == 0) throw Fail{LV_ERR_INPUT, "Error during parsing: no node found"};
  DevBuf btext;
  const unsigned char* text;
  if (in_mem == LV_MEM_DEVICE) {
    text = reinterpret_cast<const unsigned char*>(text_in) + start;
  } else {
    unsigned char* t = btext.alloc<unsigned char>(L);
    LV_CUDA(cudaMemcpyAsync(t, text_in + start, L, cudaMemcpyHostToDevice, st));
    text = t;
  }
  // token starts
  const uint64_t nchunks = (L + kIngestChunk - 1) / kIngestChunk;
  if (nchunks >= 0xFFFFFFFFull) throw Fail{LV_ERR_RANGE, "edge-list text too large"};
  DevBuf bcnt, boff, btmp;
  uint32_t* cnt = bcnt.alloc<uint32_t>(nchunks + 1);
  uint32_t* off = boff.alloc<uint32_t>(nchunks + 1);
  k_tok_count<<<grid, 256, 0, st>>>(text, L, cnt, nchunks);
  LV_CUDA(cudaMemsetAsync(cnt + nchunks, 0, 4, st));
  iscan<uint32_t>(ctx, st, btmp, cnt, nchunks + 1, off);
  uint32_t ntok32 = 0;
  LV_CUDA(cudaMemcpyAsync(&ntok32, off + nchunks, 4, cudaMemcpyDeviceToHost, st));
  LV_CUDA(cudaStreamSynchronize(st));
  const uint64_t ntok = ntok32;
  if (ntok < 2) throw Fail{LV_ERR_INPUT, "Error during parsing: no node found"};
  DevBuf bpos, bval, bbad;
  uint64_t* pos = bpos.alloc<uint64_t>(ntok);
  k_tok_place<<<grid, 256, 0, st>>>(text, L, off, nchunks, pos);
  int32_t* val = bval.alloc<int32_t>(ntok);
  unsigned long long* bad = bbad.alloc<unsigned long long>(1);
  const unsigned long long none = ntok;
  LV_CUDA(cudaMemcpyAsync(bad, &none, 8, cudaMemcpyHostToDevice, st));
  k_tok_parse<<<grid, 256, 0, st>>>(text, L, pos, ntok, val, bad);
  unsigned long long first_bad = 0;
  LV_CUDA(cudaMemcpyAsync(&first_bad, bad, 8, cudaMemcpyDeviceToHost, st));
  LV_CUDA(cudaStreamSynchronize(st));
  const uint64_t npairs = first_bad / 2;  // an unpaired last token is dropped
  if (npairs == 0) throw Fail{LV_ERR_INPUT, "Error during parsing: no node found"};
  if (npairs > (1ull << 29)) throw Fail{LV_ERR_RANGE, "more than 2^29 pairs"};
  bcnt.reset();
  boff.reset();
  bpos.reset();
  // id range
  DevBuf bmm;
  int* mm = bmm.alloc<int>(2);
  const int init[2] = {INT32_MAX, INT32_MIN};
  LV_CUDA(cudaMemcpyAsync(mm, init, 8, cudaMemcpyHostToDevice, st));
  k_ids_minmax<<<grid, 256, 0, st>>>(val, 2 * npairs, mm, mm + 1);
  int hmm[2];
  LV_CUDA(cudaMemcpyAsync(hmm, mm, 8, cudaMemcpyDeviceToHost, st));
  LV_CUDA(cudaStreamSynchronize(st));
  const uint64_t range = (uint64_t)((long long)hmm[1] - (long long)hmm[0] + 1);
  // contiguous ids: at most one id per token, so a wider range cannot be filled
  if (range > 2 * npairs) throw Fail{LV_ERR_INPUT, "vertex IDs must be contiguous (the reference indexes by id - min_id)"};
  if (range >= 0x7FFFFFFFull) throw Fail{LV_ERR_RANGE, "more than 2^31-1 vertices"};
  // entries per row (both ends of every pair); every id must have one
  DevBuf bcntr, bstart, bcount;
  uint32_t* cntr = bcntr.alloc<uint32_t>(range + 1);
  LV_CUDA(cudaMemsetAsync(cntr, 0, (range + 1) * 4, st));
  k_pair_count<<<grid, 256, 0, st>>>(val, npairs, hmm[0], cntr);
  unsigned long long* pc = bcount.alloc<unsigned long long>(2);
  LV_CUDA(cudaMemsetAsync(pc, 0, 16, st));
  k_count_present<<<grid, 256, 0, st>>>(cntr, range, pc);
  unsigned long long nn = 0;
  LV_CUDA(cudaMemcpyAsync(&nn, pc, 8, cudaMemcpyDeviceToHost, st));
  LV_CUDA(cudaStreamSynchronize(st));
  if (nn != range) throw Fail{LV_ERR_INPUT, "vertex IDs must be contiguous (the reference indexes by id - min_id)"};
  // rows placed by a scan of the counts, filled by the pairs
  uint32_t* rstart = bstart.alloc<uint32_t>(range + 1);
  iscan<uint32_t>(ctx, st, btmp, cntr, range + 1, rstart);
  DevBuf bcur, bbuf;
  uint32_t* cursor = bcur.alloc<uint32_t>(range);
  LV_CUDA(cudaMemcpyAsync(cursor, rstart, range * 4, cudaMemcpyDeviceToDevice, st));
  uint32_t* buf = bbuf.alloc<uint32_t>(2 * npairs);
  k_pair_scatter<<<grid, 256, 0, st>>>(val, npairs, hmm[0], cursor, buf);
  bval.reset();
  // each row sorted and deduplicated in place: warp, block or bitmap by its length
  DevBuf bmid, bbig, bmid8, bmid32, bcls, bulen;
  uint32_t* mid = bmid.alloc<uint32_t>(range);
  uint32_t* big = bbig.alloc<uint32_t>(range);
  uint32_t* mid8 = bmid8.alloc<uint32_t>(range);
  uint32_t* mid32 = bmid32.alloc<uint32_t>(range);
  uint32_t* cls = bcls.alloc<uint32_t>(4);
  LV_CUDA(cudaMemsetAsync(cls, 0, 16, st));
  k_rows_classify<<<grid, 256, 0, st>>>(cntr, (uint32_t)range, mid, big, mid8, mid32, cls);
  uint32_t hcls[4] = {0, 0, 0, 0};
  LV_CUDA(cudaMemcpyAsync(hcls, cls, 16, cudaMemcpyDeviceToHost, st));
  uint32_t* ulen = bulen.alloc<uint32_t>(range + 1);
  LV_CUDA(cudaMemsetAsync(ulen + range, 0, 4, st));
  k_rows_warp<<<grid, 256, 0, st>>>(rstart, cntr, (uint32_t)range, buf, ulen);
  k_rows_warpn<8><<<grid, 256, 0, st>>>(rstart, cntr, mid8, cls + 2, buf, ulen);
  k_rows_warpn<32><<<grid, 256, 0, st>>>(rstart, cntr, mid32, cls + 3, buf, ulen);
  k_rows_block<<<ctx->sms * 2, kIngestBlockNT, 0, st>>>(rstart, cntr, mid, cls, buf, ulen);
  LV_CUDA(cudaStreamSynchronize(st));
  DevBuf bbm;
  if (hcls[1] > 0) {
    // a bitmap per block, each as wide as the whole id range; blocks limited to 1 GiB of them
    const uint64_t bmw = (range >> 5) + 1;
    const uint64_t nb = std::max<uint64_t>(1, std::min<uint64_t>({(uint64_t)hcls[1], (uint64_t)ctx->sms,
                                                                   (1ull << 28) / bmw}));
    uint32_t* bitmaps = bbm.alloc<uint32_t>(nb * bmw);
    k_rows_bitmap<<<(unsigned)nb, kIngestBlockNT, 0, st>>>(rstart, cntr, big, cls, bitmaps, bmw, buf, ulen);
  }
  // the dense CSR: row offsets from a scan of the distinct lengths
  int64_t* row_ptr = nullptr;
  int32_t* col = nullptr;
  LV_CUDA(cudaMalloc(&row_ptr, (range + 1) * sizeof(int64_t)));
  iscan<int64_t>(ctx, st, btmp, ulen, range + 1, row_ptr);
  int64_t ne64 = 0;
  LV_CUDA(cudaMemcpyAsync(&ne64, row_ptr + range, 8, cudaMemcpyDeviceToHost, st));
  const cudaError_t e0 = cudaStreamSynchronize(st);
  if (e0 != cudaSuccess) {
    cudaFree(row_ptr);
    throw Fail{LV_ERR_CUDA, std::string("ingest: ") + cudaGetErrorString(e0)};
  }
  const uint64_t ne = (uint64_t)ne64;
  const int64_t nl = ne64 / 2;  // each distinct pair is two entries (a self-loop: its id twice)
  if (cudaMalloc(&col, std::max<uint64_t>(ne, 1) * sizeof(int32_t)) != cudaSuccess) {
    cudaFree(row_ptr);
    cudaGetLastError();
    throw Fail{LV_ERR_NOMEM, "cudaMalloc of the CSR destinations failed"};
  }
  k_rows_copy<<<grid, 256, 0, st>>>(rstart, row_ptr, (uint32_t)range, ne, buf, col);
  const cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    cudaFree(row_ptr);
    cudaFree(col);
    throw Fail{LV_ERR_CUDA, std::string("ingest: ") + cudaGetErrorString(e)};
  }
  out->ctx = ctx;
  out->n = (int64_t)range;
  out->n_links = nl;
  out->E = (int64_t)ne;
  out->min_id = hmm[0];
  out->row_ptr = row_ptr;
  out->col = col;
}

}  // namespace lv

extern "C" {

lv_status lv_ingest_edge_list(lv_context* ctx, const char* text, int64_t len, int32_t skip_line, int32_t in_mem,
                              lv_ingest** out) {
  if (!ctx || !out || !text || len <= 0 || skip_line < 0 || (in_mem != LV_MEM_HOST && in_mem != LV_MEM_DEVICE))
    return LV_ERR_ARGUMENT;
  *out = nullptr;
  std::lock_guard<std::mutex> lk(ctx->mu);
  auto g = std::make_unique<lv_ingest>();
  const lv_status s = guarded(ctx, [&] {
    cudaSetDevice(ctx->device);
    lv::ingest_run(ctx, text, len, skip_line, in_mem, g.get());
  });
  if (s == LV_OK) *out = g.release();
  return s;
}

lv_status lv_ingest_info(const lv_ingest* g, int64_t* n_nodes, int64_t* n_links, int64_t* entries, int64_t* min_id) {
  if (!g) return LV_ERR_ARGUMENT;
  if (n_nodes) *n_nodes = g->n;
  if (n_links) *n_links = g->n_links;
  if (entries) *entries = g->E;
  if (min_id) *min_id = g->min_id;
  return LV_OK;
}

lv_status lv_ingest_copy_csr(const lv_ingest* g, int64_t* row_ptr, int32_t* col, int32_t out_mem) {
  if (!g || !row_ptr || !col) return LV_ERR_ARGUMENT;
  const cudaMemcpyKind k = out_mem == LV_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  cudaSetDevice(g->ctx->device);
  if (cudaMemcpy(row_ptr, g->row_ptr, (size_t)(g->n + 1) * 8, k) != cudaSuccess ||
      cudaMemcpy(col, g->col, (size_t)g->E * 4, k) != cudaSuccess) {
    cudaGetLastError();
    return LV_ERR_CUDA;
  }
  return LV_OK;
}

lv_status lv_ingest_run(lv_ingest* g, int32_t* out_comm, int32_t out_mem, double* out_modularity, lv_stats* stats) {
  if (!g) return LV_ERR_ARGUMENT;
  return lv_run_csr(g->ctx, g->n, g->row_ptr, g->col, nullptr, LV_MEM_DEVICE, out_comm, out_mem, out_modularity,
                    stats);
}

lv_status lv_ingest_destroy(lv_ingest* g) {
  if (!g) return LV_ERR_ARGUMENT;
  if (g->ctx) cudaSetDevice(g->ctx->device);
  if (g->row_ptr) cudaFree(g->row_ptr);
  if (g->col) cudaFree(g->col);
  delete g;
  return LV_OK;
}

}  // extern "C"
