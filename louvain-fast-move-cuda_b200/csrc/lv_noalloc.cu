// lv_noalloc.cu -- lv_modularity_noalloc: modularity of a given partition without allocating.
//
// Some callers cannot allocate device memory at the moment they need an answer: a host
// framework that has reserved all of HBM for its own caching pool and forbids allocations
// behind its back, a latency-bound serving loop that must never stall on cudaMalloc (which
// synchronises the whole device), or code running while another component holds the device
// in a state where allocation calls are not allowed. For them this entry point evaluates
// Q = I/(2m) - S/(4 m m) for a partition using only the caller's buffers plus one fixed
// scratch array compiled into this library.
//
// Scratch: `g_noalloc_scratch`, a file-scope __device__ array of LV_NOALLOC_MAX_VERTICES + 64
// eight-byte words (8 MiB + 512 B). Every GPU that loads this library keeps that array until
// the process exits. It holds one community total per label and five accumulators. Every call
// uses the same array and leaves its own values in it; the call clears the part it uses
// before accumulating. Two calls that run on the GPU at the same time (on different streams,
// or from different host threads) use the same array and race: serialise them.
//
// Set-up: host code cannot pass the array's name to a kernel (in host code that name is only a
// stand-in, not a device address). The first call on each device, with that device current,
// asks the runtime for the array's device address with cudaGetSymbolAddress and keeps it.
// Under CUDA's default lazy module loading, that first call is also the moment this file's
// module is loaded onto the device: the 8 MiB array and the kernels' code are reserved in
// device memory then, not when the library is opened. So make the first call on each device
// before the caller's own pool claims the rest of HBM (otherwise it returns LV_ERR_CUDA), and
// before any stream capture on the device.
//
// Input checks happen on the device (the call never synchronises): a label or a column
// outside [0, n), or, with integer weights, a total weight 2m of 2^32 or more (the sum of
// squared totals is exact in u64 only below it), makes out[0] (Q) and out[3] (m) NaN. A graph
// whose weights sum to zero has m = 0 and Q = 0/0: out[0] is NaN and out[3] is 0, so the two
// cases stay apart.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/louvain_b200.h"

namespace {

constexpr int kWords = LV_NOALLOC_MAX_VERTICES + 64;
constexpr int kMaxDevices = 64;

// [0, n): community totals (u64 for integer weights, double bits otherwise);
// [LV_NOALLOC_MAX_VERTICES + 0..4]: internal weight, sum of totals^2, sum of k, flags, result.
static __device__ __align__(256) unsigned long long g_noalloc_scratch[kWords];

void* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mu;

__device__ __forceinline__ double dq(double I, double S, double m) {
  return __dsub_rn(__ddiv_rn(I, __dmul_rn(2.0, m)), __ddiv_rn(S, __dmul_rn(__dmul_rn(4.0, m), m)));
}

__global__ void k_na_clear(unsigned long long* s, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s[i] = 0ull;
  if (blockIdx.x == 0 && threadIdx.x < 5) s[LV_NOALLOC_MAX_VERTICES + threadIdx.x] = 0ull;
}

// One warp per vertex: k_v, its community's total, the internal weight (entries whose ends
// share a community, community.h:87-100) and the total weight. Labels and columns outside
// [0, n) set a flag instead of being used.
template <bool WINT>
__global__ void k_na_rows(const long long* row, const int32_t* col, const float* w,
                          const int32_t* comm, uint32_t n, unsigned long long* s) {
  const int lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t v = warp; v < n; v += nwarps) {
    const int32_t cv = comm[v];
    if (cv < 0 || (uint32_t)cv >= n) {
      if (lane == 0) atomicOr(&s[LV_NOALLOC_MAX_VERTICES + 3], 1ull);
      continue;
    }
    unsigned long long ki = 0, ii = 0;
    double kf = 0.0, iff = 0.0;
    bool bad_col = false;
    for (long long e = row[v] + lane; e < row[v + 1]; e += 32) {
      const int32_t u = col[e];
      const float x = w ? w[e] : 1.0f;
      const bool in = u >= 0 && (uint32_t)u < n;
      bad_col |= !in;
      const bool same = in && comm[u] == cv;
      if (WINT) {
        ki += (unsigned long long)x;
        if (same) ii += (unsigned long long)x;
      } else {
        kf += (double)x;
        if (same) iff += (double)x;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      ki += __shfl_xor_sync(0xFFFFFFFFu, ki, o);
      ii += __shfl_xor_sync(0xFFFFFFFFu, ii, o);
      kf += __shfl_xor_sync(0xFFFFFFFFu, kf, o);
      iff += __shfl_xor_sync(0xFFFFFFFFu, iff, o);
    }
    if (__any_sync(0xFFFFFFFFu, bad_col) && lane == 0) atomicOr(&s[LV_NOALLOC_MAX_VERTICES + 3], 2ull);
    if (lane == 0) {
      if (WINT) {
        atomicAdd(&s[cv], ki);
        atomicAdd(&s[LV_NOALLOC_MAX_VERTICES + 0], ii);
        atomicAdd(&s[LV_NOALLOC_MAX_VERTICES + 2], ki);
      } else {
        atomicAdd(reinterpret_cast<double*>(&s[cv]), kf);
        atomicAdd(reinterpret_cast<double*>(&s[LV_NOALLOC_MAX_VERTICES + 0]), iff);
        atomicAdd(reinterpret_cast<double*>(&s[LV_NOALLOC_MAX_VERTICES + 2]), kf);
      }
    }
  }
}

// Sum of squared totals (community.h:71-83), exact in u64 for integer weights.
template <bool WINT>
__global__ void k_na_squares(uint32_t n, unsigned long long* s) {
  unsigned long long su = 0;
  double sf = 0.0;
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    if (WINT) su += s[c] * s[c];
    else { const double x = __longlong_as_double((long long)s[c]); sf = __dadd_rn(sf, __dmul_rn(x, x)); }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    su += __shfl_xor_sync(0xFFFFFFFFu, su, o);
    sf += __shfl_xor_sync(0xFFFFFFFFu, sf, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (WINT) atomicAdd(&s[LV_NOALLOC_MAX_VERTICES + 1], su);
    else atomicAdd(reinterpret_cast<double*>(&s[LV_NOALLOC_MAX_VERTICES + 1]), sf);
  }
}

template <bool WINT>
__global__ void k_na_result(const unsigned long long* s, double* out) {
  if (threadIdx.x || blockIdx.x) return;
  const unsigned long long* acc = s + LV_NOALLOC_MAX_VERTICES;
  double I, S, k;
  if (WINT) { I = (double)acc[0]; S = (double)acc[1]; k = (double)acc[2]; }
  else {
    I = __longlong_as_double((long long)acc[0]);
    S = __longlong_as_double((long long)acc[1]);
    k = __longlong_as_double((long long)acc[2]);
  }
  const double m = k / 2.0;
  // flags: 1 a label out of range, 2 a column out of range, 4 integer total weight 2m >= 2^32
  const unsigned long long flags = acc[3] | (WINT && acc[2] >= (1ull << 32) ? 4ull : 0ull);
  const double nan = __longlong_as_double(0x7FF8000000000000ll);
  out[0] = flags ? nan : dq(I, S, m);  // m = 0 gives 0/0 = NaN with out[3] = 0
  out[1] = I;
  out[2] = S;
  out[3] = flags ? nan : m;
}

}  // namespace

extern "C" lv_status lv_modularity_noalloc(int64_t n, const int64_t* row_ptr, const int32_t* col,
                                           const float* w, const int32_t* comm, int32_t weights_integer,
                                           double* out, void* stream) {
  if (n <= 0 || !row_ptr || !col || !comm || !out) return LV_ERR_ARGUMENT;
  if (n > LV_NOALLOC_MAX_VERTICES) return LV_ERR_RANGE;  // more labels than the fixed scratch holds
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return LV_ERR_CUDA;
  }
  void* base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p) {
        cudaGetLastError();
        return LV_ERR_CUDA;
      }
      g_scratch_addr[dev] = p;
    }
    base = g_scratch_addr[dev];
  }
  unsigned long long* s = static_cast<unsigned long long*>(base);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const bool wint = weights_integer != 0 || w == nullptr;
  const uint32_t un = (uint32_t)n;
  k_na_clear<<<148, 256, 0, st>>>(s, un);
  if (wint) {
    k_na_rows<true><<<148 * 8, 256, 0, st>>>(reinterpret_cast<const long long*>(row_ptr), col, w, comm, un, s);
    k_na_squares<true><<<148 * 2, 256, 0, st>>>(un, s);
    k_na_result<true><<<1, 32, 0, st>>>(s, out);
  } else {
    k_na_rows<false><<<148 * 8, 256, 0, st>>>(reinterpret_cast<const long long*>(row_ptr), col, w, comm, un, s);
    k_na_squares<false><<<148 * 2, 256, 0, st>>>(un, s);
    k_na_result<false><<<1, 32, 0, st>>>(s, out);
  }
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? LV_OK : LV_ERR_CUDA;
}
