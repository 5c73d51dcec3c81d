// Self-test of the reciprocal-based correctly rounded division used by the
// FP64 kernels: div_rcp(a, b, 1/b) must return the bits of the IEEE quotient
// a / b for every operand pair (Markstein's correction; see advect_fused.cuh).
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/fesom_tracer.h"
#include "advect_fused.cuh"

namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t x) {  // splitmix64 finaliser
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// double with a random 52-bit mantissa, random sign and exponent in [lo, hi]
__device__ __forceinline__ double rand_double(uint64_t r, int lo, int hi) {
  const uint64_t mant = r & ((1ull << 52) - 1);
  const int e = lo + (int)((r >> 52) % (uint64_t)(hi - lo + 1));
  const uint64_t sign = (r >> 63) << 63;
  const uint64_t bits = sign | ((uint64_t)(e + 1023) << 52) | mant;
  return __longlong_as_double((long long)bits);
}

__global__ void k_div_check(long long n, uint64_t seed, unsigned long long *bad, double *first) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (; i < n; i += stride) {
    const uint64_t r1 = mix64(seed ^ (uint64_t)(2 * i)), r2 = mix64(seed ^ (uint64_t)(2 * i + 1));
    double a, b;
    switch (i & 3) {
      case 0: a = rand_double(r1, -80, 80); b = rand_double(r2, -60, 60); break;       // general
      case 1: a = rand_double(r1, -40, 40); b = 6.0; break;                           // MUSCL /6
      case 2: a = rand_double(r1, -30, 50); b = fabs(rand_double(r2, 10, 30)); break;  // areas
      default: a = rand_double(r1, -30, 30); b = fabs(rand_double(r2, -4, 12)); break; // thicknesses
    }
    const double y = 1.0 / b;
    const double q = fesom::div_rcp(a, b, y), ref = a / b;
    if (__double_as_longlong(q) != __double_as_longlong(ref)) {
      unsigned long long k = atomicAdd(bad, 1ull);
      if (k == 0) { first[0] = a; first[1] = b; first[2] = q; first[3] = ref; }
    }
  }
}

}  // namespace

extern "C" int tracer_selftest_division(long long n, uint64_t seed, long long *mismatches, double *example4) {
  unsigned long long *d_bad = nullptr;
  double *d_first = nullptr;
  if (cudaMalloc(&d_bad, sizeof(unsigned long long)) != cudaSuccess) return -1;
  if (cudaMalloc(&d_first, 4 * sizeof(double)) != cudaSuccess) { cudaFree(d_bad); return -1; }
  cudaMemset(d_bad, 0, sizeof(unsigned long long));
  cudaMemset(d_first, 0, 4 * sizeof(double));
  k_div_check<<<148 * 8, 256>>>(n, seed, d_bad, d_first);
  cudaError_t e = cudaDeviceSynchronize();
  unsigned long long bad = 0;
  double first[4] = {0, 0, 0, 0};
  if (e == cudaSuccess) {
    cudaMemcpy(&bad, d_bad, sizeof(bad), cudaMemcpyDeviceToHost);
    cudaMemcpy(first, d_first, sizeof(first), cudaMemcpyDeviceToHost);
  }
  cudaFree(d_bad);
  cudaFree(d_first);
  if (e != cudaSuccess) return -1;
  if (mismatches) *mismatches = (long long)bad;
  if (example4)
    for (int k = 0; k < 4; k++) example4[k] = first[k];
  return 0;
}
