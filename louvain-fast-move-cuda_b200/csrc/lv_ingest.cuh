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
//   ids      : min / max reduction, a presence bitmap over [min, max] (ids must fill it)
//   pairs    : (min, max) keys radix-sorted and deduplicated (n_links)
//   CSR      : both directions of every pair (a self-loop pair gives two (u, u) entries),
//              radix-sorted by (source, destination), row offsets from the sorted sources
#pragma once

#include <cub/cub.cuh>

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

// Presence of every id, and the pair keys (min id << 32 | max id), ids relative to the minimum.
__global__ void k_ids_mark(const int32_t* val, uint64_t npairs, int mn, uint8_t* present, uint64_t* keys) {
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < npairs;
       p += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t a = (uint32_t)((long long)val[2 * p] - mn), b = (uint32_t)((long long)val[2 * p + 1] - mn);
    present[a] = 1;
    present[b] = 1;
    keys[p] = a < b ? ((uint64_t)a << 32) | b : ((uint64_t)b << 32) | a;
  }
}

__global__ void k_count_present(const uint8_t* present, uint64_t range, unsigned long long* count) {
  unsigned long long c = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < range; i += (uint64_t)gridDim.x * blockDim.x)
    c += present[i];
  c = warp_sum(c);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

// Distinct sorted pair keys -> both directions as (source << 32 | destination).
__global__ void k_pairs_both(const uint64_t* uniq, uint64_t nl, uint64_t* both) {
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < nl; p += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = uniq[p];
    both[2 * p] = k;
    both[2 * p + 1] = (k << 32) | (k >> 32);
  }
}

// Sorted (source, destination) keys -> col, and each row's first entry index.
__global__ void k_csr_fill(const uint64_t* sorted, uint64_t ne, int32_t* col, unsigned long long* rowstart) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < ne; e += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = sorted[e];
    col[e] = (int32_t)(uint32_t)k;
    const uint32_t s = (uint32_t)(k >> 32);
    if (e == 0 || (uint32_t)(sorted[e - 1] >> 32) != s) rowstart[s] = e;
  }
}

// Row starts recorded at each row's first entry; every vertex has at least one entry (the ids
// are contiguous and each appears in a pair), so every row was written.
__global__ void k_csr_rows(const unsigned long long* rowstart, uint32_t n, uint64_t ne, int64_t* row_ptr) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v <= n; v += gridDim.x * blockDim.x)
    row_ptr[v] = v == n ? (int64_t)ne : (int64_t)rowstart[v];
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
  size_t tb = 0;
  LV_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt, off, (int)(nchunks + 1), st));
  void* tmp = btmp.alloc<unsigned char>(tb);
  LV_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, cnt, off, (int)(nchunks + 1), st));
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
  DevBuf bpres, bkeys, bcount;
  uint8_t* present = bpres.alloc<uint8_t>(range);
  LV_CUDA(cudaMemsetAsync(present, 0, range, st));
  uint64_t* keys = bkeys.alloc<uint64_t>(npairs);
  k_ids_mark<<<grid, 256, 0, st>>>(val, npairs, hmm[0], present, keys);
  unsigned long long* pc = bcount.alloc<unsigned long long>(1);
  LV_CUDA(cudaMemsetAsync(pc, 0, 8, st));
  k_count_present<<<grid, 256, 0, st>>>(present, range, pc);
  unsigned long long nn = 0;
  LV_CUDA(cudaMemcpyAsync(&nn, pc, 8, cudaMemcpyDeviceToHost, st));
  LV_CUDA(cudaStreamSynchronize(st));
  if (nn != range) throw Fail{LV_ERR_INPUT, "vertex IDs must be contiguous (the reference indexes by id - min_id)"};
  if (range >= 0x7FFFFFFFull) throw Fail{LV_ERR_RANGE, "more than 2^31-1 vertices"};
  bval.reset();
  bpres.reset();
  // distinct pairs
  int bits = 1;
  while (bits < 32 && (1ull << bits) < range) ++bits;
  DevBuf bsorted, bsel;
  uint64_t* sorted = bsorted.alloc<uint64_t>(npairs);
  tb = 0;
  LV_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, keys, sorted, (int)npairs, 0, 32 + bits, st));
  tmp = btmp.alloc<unsigned char>(tb);
  LV_CUDA(cub::DeviceRadixSort::SortKeys(tmp, tb, keys, sorted, (int)npairs, 0, 32 + bits, st));
  int* nsel = bsel.alloc<int>(1);
  tb = 0;
  LV_CUDA(cub::DeviceSelect::Unique(nullptr, tb, sorted, keys, nsel, (int)npairs, st));
  tmp = btmp.alloc<unsigned char>(tb);
  LV_CUDA(cub::DeviceSelect::Unique(tmp, tb, sorted, keys, nsel, (int)npairs, st));
  int nl = 0;
  LV_CUDA(cudaMemcpyAsync(&nl, nsel, 4, cudaMemcpyDeviceToHost, st));
  LV_CUDA(cudaStreamSynchronize(st));
  const uint64_t ne = 2ull * (uint64_t)nl;
  // both directions, sorted by (source, destination)
  DevBuf bboth, bsorted2;
  uint64_t* both = bboth.alloc<uint64_t>(ne);
  k_pairs_both<<<grid, 256, 0, st>>>(keys, (uint64_t)nl, both);
  bkeys.reset();
  bsorted.reset();
  uint64_t* sorted2 = bsorted2.alloc<uint64_t>(ne);
  tb = 0;
  LV_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, both, sorted2, (int)ne, 0, 32 + bits, st));
  tmp = btmp.alloc<unsigned char>(tb);
  LV_CUDA(cub::DeviceRadixSort::SortKeys(tmp, tb, both, sorted2, (int)ne, 0, 32 + bits, st));
  bboth.reset();
  // CSR
  int64_t* row_ptr = nullptr;
  int32_t* col = nullptr;
  LV_CUDA(cudaMalloc(&row_ptr, (range + 1) * sizeof(int64_t)));
  if (cudaMalloc(&col, ne * sizeof(int32_t)) != cudaSuccess) {
    cudaFree(row_ptr);
    cudaGetLastError();
    throw Fail{LV_ERR_NOMEM, "cudaMalloc of the CSR destinations failed"};
  }
  DevBuf bstart;
  unsigned long long* rstart = bstart.alloc<unsigned long long>(range);
  k_csr_fill<<<grid, 256, 0, st>>>(sorted2, ne, col, rstart);
  k_csr_rows<<<grid, 256, 0, st>>>(rstart, (uint32_t)range, ne, row_ptr);
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
