// Device self-tests of arithmetic primitives of the step kernels:
//  * the reciprocal-based correctly rounded division of the FP64 kernels:
//    div_rcp(a, b, 1/b) must return the bits of the IEEE quotient a / b for
//    every operand pair (Markstein's correction; see advect_fused.cuh);
//  * the stochastic rounding of 16-bit tracer stores (advect_ops.cuh): every
//    result is one of the two storage neighbours of the input, and the
//    fraction rounded up matches (remainder / spacing) without bias.
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

// storage neighbours of x toward zero (lo) and away from zero (hi)
__device__ __forceinline__ void nbrs_bf16(float x, float &lo, float &hi) {
  const uint32_t u = __float_as_uint(x) & 0xffff0000u;
  lo = __uint_as_float(u);
  hi = __uint_as_float(u + 0x10000u);
}
__device__ __forceinline__ void nbrs_f16(float x, float &lo, float &hi) {
  const __half l = __float2half_rz(x);
  lo = __half2float(l);
  hi = __half2float(__ushort_as_half((unsigned short)(__half_as_ushort(l) + 1)));
}

// fmt 0: BF16, 1: FP16.  Per input: `draws` roundings with the kernels'
// stream (per-step seed word, per-cell index); counts results outside
// {lo, hi} and accumulates (ups - draws p) and draws p (1 - p).
__global__ void k_sround_check(int fmt, long long n, int draws, uint32_t seed, unsigned long long *bad,
                               double *acc) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  double dev = 0.0, var = 0.0;
  for (; i < n; i += stride) {
    const uint64_t r = mix64((uint64_t)seed * 0x100000001ull ^ (uint64_t)i);
    // magnitudes 2^-6 .. 2^10 with random sign; one input in 16 exactly
    // representable in the format
    float x = ldexpf(1.0f + (float)(r & 0xffffff) * 0x1p-24f, (int)((r >> 24) % 16) - 6);
    if ((r >> 40) & 1) x = -x;
    float lo, hi;
    if (fmt == 0) nbrs_bf16(x, lo, hi);
    else nbrs_f16(x, lo, hi);
    if (((r >> 44) & 15) == 0) x = lo;
    const float gap = fabsf(hi - lo), rem = fabsf(x - lo);
    const double p = (double)rem / (double)gap;
    int ups = 0;
    for (int d = 0; d < draws; d++) {
      const uint32_t step_seed = fesom::mix32(seed + 0x9e3779b9u * (uint32_t)d);
      const uint32_t word = fesom::mix32(step_seed ^ fesom::mix32((uint32_t)i));
      const float y = fmt == 0 ? __bfloat162float(fesom::bf16_sround(x, word))
                               : __half2float(fesom::f16_sround(x, word));
      if (y == hi && rem > 0.0f) ups++;
      else if (y != lo) atomicAdd(bad, 1ull);
    }
    dev += (double)ups - draws * p;
    var += draws * p * (1.0 - p);
  }
  atomicAdd(&acc[0], dev);
  atomicAdd(&acc[1], var);
}

}  // namespace

extern "C" int tracer_selftest_sround(int fmt, long long n, int draws, uint32_t seed, long long *outside,
                                      double *z) {
  if (fmt < 0 || fmt > 1 || n < 1 || draws < 1) return -1;
  unsigned long long *d_bad = nullptr;
  double *d_acc = nullptr;
  if (cudaMalloc(&d_bad, sizeof(unsigned long long)) != cudaSuccess) return -1;
  if (cudaMalloc(&d_acc, 2 * sizeof(double)) != cudaSuccess) { cudaFree(d_bad); return -1; }
  cudaMemset(d_bad, 0, sizeof(unsigned long long));
  cudaMemset(d_acc, 0, 2 * sizeof(double));
  k_sround_check<<<148 * 4, 256>>>(fmt, n, draws, seed, d_bad, d_acc);
  cudaError_t e = cudaDeviceSynchronize();
  unsigned long long bad = 0;
  double acc[2] = {0, 0};
  if (e == cudaSuccess) {
    cudaMemcpy(&bad, d_bad, sizeof(bad), cudaMemcpyDeviceToHost);
    cudaMemcpy(acc, d_acc, sizeof(acc), cudaMemcpyDeviceToHost);
  }
  cudaFree(d_bad);
  cudaFree(d_acc);
  if (e != cudaSuccess) return -1;
  if (outside) *outside = (long long)bad;
  if (z) *z = acc[1] > 0.0 ? acc[0] / sqrt(acc[1]) : 0.0;
  return 0;
}

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
