// Fuzz check of gain_fast (csrc/lv_device.cuh) against gain_exact, the reference's gain
// (operatorsDelta.h:29-45) evaluated with IEEE double divisions: both must give the same float,
// bit for bit, on every input. Compiled and run by tests/test_gain_fuzz_gpu.py.
//
// usage: gain_fuzz <log2 cases>   prints "cases mismatches fallbacks" and, for a mismatch,
// its inputs; exit status 1 on any mismatch.
#include <cstdio>
#include <cstdlib>

#include "lv_device.cuh"

using namespace lv;

__device__ __forceinline__ unsigned long long mix(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
__device__ __forceinline__ double unit(unsigned long long x) { return (double)(x >> 11) * 0x1p-53; }

struct Bad {
  unsigned long long count, fallbacks, first;
  float diff;
  double p, m;
};

__global__ void k_fuzz(unsigned long long n, Bad* bad) {
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long r0 = mix(i), r1 = mix(r0), r2 = mix(r1), r3 = mix(r2);
    // total weight m: integers from 1 to 2^31 (log-uniform), or fp32 sums with fractions
    double m = floor(exp2(unit(r0) * 31.0));
    if (m < 1.0) m = 1.0;
    if (r3 & 1) m = m + unit(r3) * 0.5;
    const double two_m2 = __dmul_rn(__dmul_rn(2.0, m), m);
    const double inv_m = __drcp_rn(m), inv_2m2 = __drcp_rn(two_m2);
    // diff = w_vc - self_v: integers up to 2m (either sign), sometimes fractional
    float diff = (float)floor((unit(r1) * 2.0 - 1.0) * fmin(2.0 * m, 16777216.0) * unit(r2));
    if (r3 & 2) diff = __fmul_rn(diff, 1.0f + (float)unit(r3 >> 8) * 0.25f);
    const int kind = (int)((r3 >> 2) & 3);
    double p;
    if (kind == 0) {
      // generic: k (a_own - k - a_c) with totals up to 2m
      const double k = floor(unit(r2 >> 3) * m) + 1.0;
      p = __dmul_rn(k, floor((unit(r1 >> 5) * 2.0 - 1.0) * 2.0 * m));
    } else if (kind == 1) {
      // near cancellation: p / (2 m^2) close to -diff / m
      p = floor(-(double)diff * 2.0 * m * (1.0 + (unit(r2 >> 7) - 0.5) * 1e-6));
    } else {
      // the sum aimed at a float rounding boundary: the midpoint between two floats
      const float f = (float)((unit(r1 >> 9) - 0.5) * 4.0 * (double)fabsf(diff) / m + 1e-30);
      const double mid = (double)f + 0.5 * (double)(nextafterf(f, 1e30f) - f);
      p = __dmul_rn(__dsub_rn(mid, __ddiv_rn((double)diff, m)), two_m2);
      if (kind == 3) p = floor(p);
    }
    const float a = gain_fast(diff, p, inv_m, inv_2m2, m, two_m2);
    const float b = gain_exact(diff, p, m, two_m2);
    const double t1 = __dmul_rn((double)diff, inv_m), t2 = __dmul_rn(p, inv_2m2);
    const double err = __fma_rn(__dadd_rn(fabs(t1), fabs(t2)), 0x1p-49, 0x1p-1000);
    const double s = __dadd_rn(t1, t2);
    if (__float_as_uint(__double2float_rn(__dsub_rd(s, err))) != __float_as_uint(__double2float_rn(__dadd_ru(s, err))))
      atomicAdd(&bad->fallbacks, 1ull);
    if (__float_as_uint(a) != __float_as_uint(b)) {
      if (atomicAdd(&bad->count, 1ull) == 0) {
        bad->first = i;
        bad->diff = diff;
        bad->p = p;
        bad->m = m;
      }
    }
  }
}

int main(int argc, char** argv) {
  const int lg = argc > 1 ? atoi(argv[1]) : 26;
  const unsigned long long n = 1ull << lg;
  Bad* d = nullptr;
  if (cudaMalloc(&d, sizeof(Bad)) != cudaSuccess) return 3;
  cudaMemset(d, 0, sizeof(Bad));
  k_fuzz<<<148 * 16, 256>>>(n, d);
  Bad h{};
  if (cudaMemcpy(&h, d, sizeof(Bad), cudaMemcpyDeviceToHost) != cudaSuccess) return 4;
  cudaFree(d);
  std::printf("%llu %llu %llu\n", n, h.count, h.fallbacks);
  if (h.count) std::printf("first mismatch #%llu diff=%.9g p=%.17g m=%.17g\n", h.first, h.diff, h.p, h.m);
  return h.count ? 1 : 0;
}
