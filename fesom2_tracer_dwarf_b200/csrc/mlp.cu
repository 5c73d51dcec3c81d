// Learned antidiffusive edge flux: a per-edge-level MLP (16 -> 64 -> 64 -> 1,
// GELU (tanh form), BF16 weights and activations, FP32 accumulation) on the fifth-
// generation tensor cores (tcgen05.mma, accumulators in TMEM).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "../../include/fesom_tracer.h"
#include "advect_fused.cuh"
#include "engine_impl.hpp"
#include "umma.cuh"

namespace fesom {
namespace {

constexpr long long kWaitLimit = 1ll << 26;  // mbarrier polls before giving up

// One CTA of 128 threads: D[128 x N] = A[128 x K] * B[N x K]^T with BF16
// inputs from global memory (row-major) and an FP32 result.
__global__ void __launch_bounds__(128, 1)
    k_umma_selftest(const __nv_bfloat16 *A, const __nv_bfloat16 *B, float *D, int N, int K, int *status) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tbase;
  const int tid = threadIdx.x, warp = tid >> 5;
  unsigned char *sA = sm;
  unsigned char *sB = sm + (((size_t)128 * K * 2 + 1023) & ~(size_t)1023);
  for (int i = tid; i < 128 * K; i += blockDim.x)
    *reinterpret_cast<__nv_bfloat16 *>(sA + umma::kmajor_offset(i / K, i % K, K)) = A[i];
  for (int i = tid; i < N * K; i += blockDim.x)
    *reinterpret_cast<__nv_bfloat16 *>(sB + umma::kmajor_offset(i / K, i % K, K)) = B[i];
  umma::fence_async_smem();
  uint32_t ncols = 32;
  while ((int)ncols < N) ncols <<= 1;
  if (warp == 0) {
    umma::tmem_alloc(&tbase, ncols);
    umma::tmem_relinquish();
  }
  if (tid == 0) {
    umma::mbar_init(&mbar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  const uint32_t tmem = tbase;
  if (tid == 0) {
    const uint32_t idesc = umma::idesc_bf16_f32(128, N);
    const uint32_t sbo = (uint32_t)(K / 8) * 128;
    for (int s = 0; s < K / 16; s++) {
      const uint64_t ad = umma::smem_desc(umma::smem_u32(sA) + s * 256, 128, sbo);
      const uint64_t bd = umma::smem_desc(umma::smem_u32(sB) + s * 256, 128, sbo);
      umma::mma_bf16(tmem, ad, bd, idesc, s > 0 ? 1u : 0u);
    }
    umma::mma_commit(&mbar);
  }
  const bool ok = umma::mbar_wait(&mbar, 0, kWaitLimit);
  umma::tc_fence_after();
  if (ok) {
    float v[16];
    for (int c = 0; c < N; c += 16) {
      umma::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
      for (int i = 0; i < 16; i++) D[(size_t)tid * N + c + i] = v[i];
    }
  } else if (tid == 0) {
    atomicExch(status, 2);
  }
  umma::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    umma::tc_fence_after();
    umma::tmem_dealloc(tmem, ncols);
  }
}

// ---------------------------------------------------------------------------
// MLP 16 -> 64 -> 64 -> 1 (GELU).  Parameters (FP32 master copy, packed):
// W1[64][16], b1[64], W2[64][64], b2[64], w3[64], b3 -- W1 and W2 also as
// BF16 for the tensor cores.  One CTA of 128 threads handles 128-sample
// tiles; thread m owns sample row m (TMEM lane m).
// ---------------------------------------------------------------------------
constexpr int kF = 16, kH = 64;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kH * kF, kOffW2 = kOffB1 + kH, kOffB2 = kOffW2 + kH * kH,
              kOffW3 = kOffB2 + kH, kOffB3 = kOffW3 + kH, kParams = kOffB3 + 1;

// GELU in its tanh form (Hendrycks & Gimpel 2016),
// g(z) = z/2 (1 + tanh(c (z + 0.044715 z^3))), c = sqrt(2/pi), with the
// hardware tanh approximation
__device__ __forceinline__ float tanh_fast(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
constexpr float kGeluC = 0.7978845608028654f, kGeluA = 0.044715f;
__device__ __forceinline__ float gelu(float z) {
  const float t = tanh_fast(kGeluC * (z + kGeluA * z * z * z));
  return 0.5f * z * (1.0f + t);
}
// acc + GELU(z) w3 with hw3 = w3 / 2, i.e. acc + hw3 z (1 + tanh u):
// u = z (c + c a z^2), then one add and one FMA
__device__ __forceinline__ float gelu_out(float z, float hw3, float acc) {
  const float t = tanh_fast(z * fmaf(kGeluC * kGeluA, z * z, kGeluC));
  const float hz = z * hw3;
  return fmaf(hz, t, acc + hz);
}
__device__ __forceinline__ float gelu_grad(float z) {
  const float t = tanh_fast(kGeluC * (z + kGeluA * z * z * z));
  return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * kGeluC * (1.0f + 3.0f * kGeluA * z * z);
}

// The first inference epilogue evaluates GELU on packed FP16 pairs (two
// values per instruction, hardware tanh.approx.f16x2): its activations are
// stored as BF16 for the second MMA anyway, whose 8-bit mantissa is coarser
// than FP16's 11 bits.  The second epilogue, which feeds the FP32 output
// layer directly, keeps the FP32 form (with the FP16 form there, the
// output's error against the exact network doubled).  Training keeps the
// FP32 form throughout.
__device__ __forceinline__ __half2 tanh_fast2(__half2 x) {
  uint32_t y, xi = *reinterpret_cast<uint32_t *>(&x);
  asm("tanh.approx.f16x2 %0, %1;" : "=r"(y) : "r"(xi));
  return *reinterpret_cast<__half2 *>(&y);
}
__device__ __forceinline__ __half2 gelu2(__half2 z) {
  const __half2 c = __float2half2_rn(kGeluC), ca = __float2half2_rn(kGeluC * kGeluA), h = __float2half2_rn(0.5f);
  const __half2 z2 = __hmul2(z, z);
  const __half2 u = __hmul2(z, __hfma2(ca, z2, c));  // c z + c a z^3
  const __half2 hz = __hmul2(h, z);
  return __hfma2(hz, tanh_fast2(u), hz);             // z/2 (1 + tanh u)
}
// 16 FP32 pre-activations (bias added) -> GELU -> 16 BF16 in two 16-byte stores
// (bias: 16-byte aligned shared memory, read as four 16-byte vectors)
__device__ __forceinline__ void gelu_store16(unsigned char *base, uint32_t off_lo, uint32_t off_hi, const float *v,
                                             const float *bias_s) {
  __align__(16) __nv_bfloat162 o[8];
  float bias[16];
  for (int i = 0; i < 4; i++) reinterpret_cast<float4 *>(bias)[i] = reinterpret_cast<const float4 *>(bias_s)[i];
  for (int i = 0; i < 8; i++) {
    const __half2 g = gelu2(__floats2half2_rn(v[2 * i] + bias[2 * i], v[2 * i + 1] + bias[2 * i + 1]));
    o[i] = __float22bfloat162_rn(__half22float2(g));
  }
  *reinterpret_cast<uint4 *>(base + off_lo) = *reinterpret_cast<const uint4 *>(o);
  *reinterpret_cast<uint4 *>(base + off_hi) = *reinterpret_cast<const uint4 *>(o + 4);
}

struct MlpDev {
  const __nv_bfloat16 *W1b, *W2b;  // [64][16], [64][64] BF16
  const float *p;                  // FP32 packed parameters
};

// byte offsets of the shared-memory tiles (all 1024-aligned)
struct FwdSmem {
  static constexpr uint32_t W1 = 0, W2 = 2048, X = W2 + 8192, H1 = X + 4096, END = H1 + 16384;
};
struct TrainSmem {
  static constexpr uint32_t W1 = 0, W2 = 2048, W2T = W2 + 8192, X = W2T + 8192, XT = X + 4096, H1 = XT + 4096,
                            H1T = H1 + 16384, DZ2 = H1T + 16384, DZ2T = DZ2 + 16384, DZ1T = DZ2T + 32768,
                            END = DZ1T + 32768;
};

__device__ __forceinline__ void st_bf16(unsigned char *base, uint32_t off, float v) {
  *reinterpret_cast<__nv_bfloat16 *>(base + off) = __float2bfloat16_rn(v);
}
// 8 consecutive K elements of one row: one 16-byte store
__device__ __forceinline__ void st_bf16x8(unsigned char *base, uint32_t off, const float *v) {
  __align__(16) __nv_bfloat16 h[8];
  for (int i = 0; i < 8; i++) h[i] = __float2bfloat16_rn(v[i]);
  *reinterpret_cast<uint4 *>(base + off) = *reinterpret_cast<const uint4 *>(h);
}

__device__ __forceinline__ void load_weights(unsigned char *sm, const MlpDev &w, uint32_t oW1, uint32_t oW2,
                                             uint32_t oW2T) {
  for (int i = threadIdx.x; i < kH * kF; i += blockDim.x)
    *reinterpret_cast<__nv_bfloat16 *>(sm + oW1 + umma::kmajor_offset(i / kF, i % kF, kF)) = w.W1b[i];
  for (int i = threadIdx.x; i < kH * kH; i += blockDim.x) {
    const int j = i / kH, k = i % kH;  // W2[j][k]: output j, input k
    *reinterpret_cast<__nv_bfloat16 *>(sm + oW2 + umma::kmajor_offset(j, k, kH)) = w.W2b[i];
    if (oW2T != 0xffffffffu)
      *reinterpret_cast<__nv_bfloat16 *>(sm + oW2T + umma::kmajor_offset(k, j, kH)) = w.W2b[i];
  }
}

// this thread's sample: 16 BF16 features as two 16-byte loads (zeros past S)
__device__ __forceinline__ void load_sample(const __nv_bfloat16 *X, long long S, long long sample, uint4 &lo,
                                            uint4 &hi) {
  if (sample < S) {
    const uint4 *p = reinterpret_cast<const uint4 *>(X + sample * kF);
    lo = p[0];
    hi = p[1];
  } else {
    lo = make_uint4(0, 0, 0, 0);
    hi = lo;
  }
}

__device__ __forceinline__ void mma_tiles(uint32_t tmem_d, uint32_t a, uint32_t b, int K, int N, bool accumulate) {
  const uint32_t idesc = umma::idesc_bf16_f32(128, N), sbo = (uint32_t)(K / 8) * 128;
  for (int s = 0; s < K / 16; s++)
    umma::mma_bf16(tmem_d, umma::smem_desc(a + s * 256, 128, sbo), umma::smem_desc(b + s * 256, 128, sbo), idesc,
                   (accumulate || s > 0) ? 1u : 0u);
}

// every thread waits; all agree on the outcome
__device__ __forceinline__ bool wait_all(uint64_t *mbar, uint32_t &phase) {
  const bool ok = umma::mbar_wait(mbar, phase, kWaitLimit);
  phase ^= 1u;
  umma::tc_fence_after();
  return __syncthreads_and(ok ? 1 : 0) != 0;
}

__device__ __forceinline__ void smem_to_tc() {
  umma::fence_async_smem();
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
}

// TMEM columns of one forward CTA (the 64 FP32 accumulator columns of a
// 128 x 64 layer output).  With 64 columns, eight CTAs fit an SM's 512 TMEM
// columns, so shared memory (about 32 KB per CTA) sets how many run side by
// side; their tiles' load, MMA and epilogue phases overlap one another.
constexpr uint32_t kFwdTmemCols = 64;

__global__ void __launch_bounds__(128, 1)
    k_mlp_fwd(const __nv_bfloat16 *X, long long S, MlpDev w, float *y, int *status) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tbase;
  __shared__ __align__(16) float sb1[kH];
  __shared__ __align__(16) float sb2[kH];
  __shared__ __align__(16) float shw3[kH];
  const int tid = threadIdx.x, warp = tid >> 5;
  load_weights(sm, w, FwdSmem::W1, FwdSmem::W2, 0xffffffffu);
  if (tid < kH) {
    sb1[tid] = w.p[kOffB1 + tid];
    sb2[tid] = w.p[kOffB2 + tid];
    shw3[tid] = 0.5f * w.p[kOffW3 + tid];  // the GELU's 1/2 folded into the output weights
  }
  const float b3 = w.p[kOffB3];
  if (warp == 0) {
    umma::tmem_alloc(&tbase, kFwdTmemCols);
    umma::tmem_relinquish();
  }
  if (tid == 0) {
    umma::mbar_init(&mbar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  smem_to_tc();
  const uint32_t tmem = tbase, lane = (uint32_t)(warp * 32) << 16;
  // both layers accumulate into the same 64 columns: every thread has read
  // the first layer's result (tcgen05.ld + wait::ld) before the barrier that
  // precedes the second MMA, and has read the second's before the barrier
  // that ends the tile
  const uint32_t D1 = tmem, D2 = tmem;
  const uint32_t aX = umma::smem_u32(sm + FwdSmem::X), aH1 = umma::smem_u32(sm + FwdSmem::H1);
  const uint32_t aW1 = umma::smem_u32(sm + FwdSmem::W1), aW2 = umma::smem_u32(sm + FwdSmem::W2);
  uint32_t phase = 0;
  bool ok = true;
  const long long ntiles = (S + 127) / 128;
  for (long long t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
    const long long sample = t * 128 + tid;
    uint4 lo, hi;
    load_sample(X, S, sample, lo, hi);
    *reinterpret_cast<uint4 *>(sm + FwdSmem::X + umma::kmajor_offset(tid, 0, kF)) = lo;
    *reinterpret_cast<uint4 *>(sm + FwdSmem::X + umma::kmajor_offset(tid, 8, kF)) = hi;
    smem_to_tc();
    if (tid == 0) {
      mma_tiles(D1, aX, aW1, kF, kH, false);
      umma::mma_commit(&mbar);
    }
    if (!(ok = wait_all(&mbar, phase))) break;
    for (int c = 0; c < kH; c += 16) {
      float v[16];
      umma::tmem_ld16(D1 + lane + c, v);
      gelu_store16(sm + FwdSmem::H1, umma::kmajor_offset(tid, c, kH), umma::kmajor_offset(tid, c + 8, kH), v, sb1 + c);
    }
    smem_to_tc();
    if (tid == 0) {
      mma_tiles(D2, aH1, aW2, kH, kH, false);
      umma::mma_commit(&mbar);
    }
    if (!(ok = wait_all(&mbar, phase))) break;
    float acc = 0.f;
    for (int c = 0; c < kH; c += 16) {
      float v[16];
      umma::tmem_ld16(D2 + lane + c, v);
      float b[16], hw[16];
      for (int i = 0; i < 4; i++) {
        reinterpret_cast<float4 *>(b)[i] = reinterpret_cast<const float4 *>(sb2 + c)[i];
        reinterpret_cast<float4 *>(hw)[i] = reinterpret_cast<const float4 *>(shw3 + c)[i];
      }
      for (int i = 0; i < 16; i++) acc = gelu_out(v[i] + b[i], hw[i], acc);
    }
    if (sample < S) y[sample] = acc + b3;
    umma::tc_fence_before();
    __syncthreads();
    umma::tc_fence_after();
  }
  if (!ok) {
    if (tid == 0) atomicExch(status, 2);
    umma::mbar_wait(&mbar, phase ^ 1u, kWaitLimit);  // bounded: let the MMA in flight finish
  }
  umma::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    umma::tc_fence_after();
    umma::tmem_dealloc(tmem, kFwdTmemCols);
  }
}

__device__ __forceinline__ float warp_sum(float v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Gradients of sum_s dy[s] * y(x_s) with respect to every parameter, added
// to grad (FP32, packed like the parameters).
__global__ void __launch_bounds__(128, 1)
    k_mlp_train(const __nv_bfloat16 *X, const float *dy, long long S, MlpDev w, float *grad, int *status) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tbase;
  __shared__ float sb1[kH], sb2[kH], sw3[kH], gdb1[kH], gdb2[kH], gdw3[kH], gdb3;
  const int tid = threadIdx.x, warp = tid >> 5, lid = tid & 31;
  load_weights(sm, w, TrainSmem::W1, TrainSmem::W2, TrainSmem::W2T);
  // padded rows 64..127 of the transposed gradient operands stay zero
  for (int i = tid; i < 64 * 128 * 2 / 16; i += blockDim.x) {
    reinterpret_cast<uint4 *>(sm + TrainSmem::DZ2T + 64 * 128 * 2)[i] = make_uint4(0, 0, 0, 0);
    reinterpret_cast<uint4 *>(sm + TrainSmem::DZ1T + 64 * 128 * 2)[i] = make_uint4(0, 0, 0, 0);
  }
  if (tid < kH) {
    sb1[tid] = w.p[kOffB1 + tid];
    sb2[tid] = w.p[kOffB2 + tid];
    sw3[tid] = w.p[kOffW3 + tid];
    gdb1[tid] = gdb2[tid] = gdw3[tid] = 0.f;
  }
  if (tid == 0) gdb3 = 0.f;
  if (warp == 0) {
    umma::tmem_alloc(&tbase, 512);
    umma::tmem_relinquish();
  }
  if (tid == 0) {
    umma::mbar_init(&mbar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  smem_to_tc();
  const uint32_t tmem = tbase, lane = (uint32_t)(warp * 32) << 16;
  const uint32_t D1 = tmem, D2 = tmem + 64, DH1 = tmem + 128, DW2 = tmem + 192, DW1 = tmem + 256;
  auto A = [&](uint32_t off) { return umma::smem_u32(sm + off); };
  uint32_t phase = 0;
  bool ok = true, first = true;
  const long long ntiles = (S + 127) / 128;
  for (long long t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
    const long long sample = t * 128 + tid;
    const float g = sample < S ? dy[sample] : 0.f;
    uint4 lo, hi;
    load_sample(X, S, sample, lo, hi);
    *reinterpret_cast<uint4 *>(sm + TrainSmem::X + umma::kmajor_offset(tid, 0, kF)) = lo;
    *reinterpret_cast<uint4 *>(sm + TrainSmem::X + umma::kmajor_offset(tid, 8, kF)) = hi;
    {
      const __nv_bfloat16 *xv = reinterpret_cast<const __nv_bfloat16 *>(&lo);
      const __nv_bfloat16 *xw = reinterpret_cast<const __nv_bfloat16 *>(&hi);
      for (int f = 0; f < 8; f++) {
        *reinterpret_cast<__nv_bfloat16 *>(sm + TrainSmem::XT + umma::kmajor_offset(f, tid, 128)) = xv[f];
        *reinterpret_cast<__nv_bfloat16 *>(sm + TrainSmem::XT + umma::kmajor_offset(f + 8, tid, 128)) = xw[f];
      }
    }
    smem_to_tc();
    if (tid == 0) {
      mma_tiles(D1, A(TrainSmem::X), A(TrainSmem::W1), kF, kH, false);
      umma::mma_commit(&mbar);
    }
    if (!(ok = wait_all(&mbar, phase))) break;
    for (int c = 0; c < kH; c += 16) {
      float v[16];
      umma::tmem_ld16(D1 + lane + c, v);
      for (int i = 0; i < 16; i++) {
        v[i] = gelu(v[i] + sb1[c + i]);
        st_bf16(sm + TrainSmem::H1T, umma::kmajor_offset(c + i, tid, 128), v[i]);
      }
      st_bf16x8(sm + TrainSmem::H1, umma::kmajor_offset(tid, c, kH), v);
      st_bf16x8(sm + TrainSmem::H1, umma::kmajor_offset(tid, c + 8, kH), v + 8);
    }
    smem_to_tc();
    if (tid == 0) {
      mma_tiles(D2, A(TrainSmem::H1), A(TrainSmem::W2), kH, kH, false);
      umma::mma_commit(&mbar);
    }
    if (!(ok = wait_all(&mbar, phase))) break;
    // output layer and dZ2 = dy * w3 * gelu'(z2)
    for (int c = 0; c < kH; c += 16) {
      float v[16], dz[16];
      umma::tmem_ld16(D2 + lane + c, v);
      for (int i = 0; i < 16; i++) {
        const float z = v[i] + sb2[c + i];
        const float h2 = gelu(z);
        dz[i] = g * sw3[c + i] * gelu_grad(z);
        st_bf16(sm + TrainSmem::DZ2T, umma::kmajor_offset(c + i, tid, 128), dz[i]);
        const float a = warp_sum(g * h2), b = warp_sum(dz[i]);
        if (lid == 0) {
          atomicAdd(&gdw3[c + i], a);
          atomicAdd(&gdb2[c + i], b);
        }
      }
      st_bf16x8(sm + TrainSmem::DZ2, umma::kmajor_offset(tid, c, kH), dz);
      st_bf16x8(sm + TrainSmem::DZ2, umma::kmajor_offset(tid, c + 8, kH), dz + 8);
    }
    {
      const float a = warp_sum(g);
      if (lid == 0) atomicAdd(&gdb3, a);
    }
    smem_to_tc();
    if (tid == 0) {
      // dW2[j][i] += sum_m dZ2[m][j] H1[m][i];  dH1[m][i] = sum_j dZ2[m][j] W2[j][i]
      mma_tiles(DW2, A(TrainSmem::DZ2T), A(TrainSmem::H1T), 128, kH, !first);
      mma_tiles(DH1, A(TrainSmem::DZ2), A(TrainSmem::W2T), kH, kH, false);
      umma::mma_commit(&mbar);
    }
    if (!(ok = wait_all(&mbar, phase))) break;
    for (int c = 0; c < kH; c += 16) {
      float dh[16], z1[16];
      umma::tmem_ld16(DH1 + lane + c, dh);
      umma::tmem_ld16(D1 + lane + c, z1);
      for (int i = 0; i < 16; i++) {
        const float dz = dh[i] * gelu_grad(z1[i] + sb1[c + i]);
        st_bf16(sm + TrainSmem::DZ1T, umma::kmajor_offset(c + i, tid, 128), dz);
        const float b = warp_sum(dz);
        if (lid == 0) atomicAdd(&gdb1[c + i], b);
      }
    }
    smem_to_tc();
    if (tid == 0) {
      // dW1[i][f] += sum_m dZ1[m][i] X[m][f]
      mma_tiles(DW1, A(TrainSmem::DZ1T), A(TrainSmem::XT), 128, kF, !first);
      umma::mma_commit(&mbar);
    }
    if (!(ok = wait_all(&mbar, phase))) break;
    first = false;
  }
  if (!ok) {
    if (tid == 0) atomicExch(status, 2);
    umma::mbar_wait(&mbar, phase ^ 1u, kWaitLimit);  // bounded: let the MMA in flight finish
  } else if (!first) {
    // weight gradients: rows j (i) < 64 live in TMEM lanes 0..63 (warps 0, 1)
    if (warp < 2) {
      for (int c = 0; c < kH; c += 16) {
        float v[16];
        umma::tmem_ld16(DW2 + lane + c, v);
        for (int i = 0; i < 16; i++) atomicAdd(&grad[kOffW2 + tid * kH + c + i], v[i]);
      }
      float v[16];
      umma::tmem_ld16(DW1 + lane, v);
      for (int i = 0; i < 16; i++) atomicAdd(&grad[kOffW1 + tid * kF + i], v[i]);
    }
  }
  __syncthreads();
  if (tid < kH) {
    atomicAdd(&grad[kOffB1 + tid], gdb1[tid]);
    atomicAdd(&grad[kOffB2 + tid], gdb2[tid]);
    atomicAdd(&grad[kOffW3 + tid], gdw3[tid]);
  }
  if (tid == 0) atomicAdd(&grad[kOffB3], gdb3);
  umma::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    umma::tc_fence_after();
    umma::tmem_dealloc(tmem, 512);
  }
}

__global__ void k_params_to_bf16(const float *p, __nv_bfloat16 *W1b, __nv_bfloat16 *W2b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kH * kF + kH * kH; i += gridDim.x * blockDim.x) {
    if (i < kH * kF) W1b[i] = __float2bfloat16_rn(p[kOffW1 + i]);
    else W2b[i - kH * kF] = __float2bfloat16_rn(p[kOffW2 + i - kH * kF]);
  }
}

}  // namespace
}  // namespace fesom

using namespace fesom;

namespace fesom {

// Device state of one MLP: FP32 parameters (and gradients, Adam moments),
// BF16 copies of W1 and W2.
struct MlpState {
  float *p = nullptr, *grad = nullptr, *m1 = nullptr, *m2 = nullptr;
  __nv_bfloat16 *W1b = nullptr, *W2b = nullptr;
  int *status = nullptr;
  int adam_t = 0;
  int sms = 148;
};

static bool mlp_alloc(MlpState &s) {
  if (cudaMalloc(&s.p, kParams * 4) != cudaSuccess || cudaMalloc(&s.grad, kParams * 4) != cudaSuccess ||
      cudaMalloc(&s.m1, kParams * 4) != cudaSuccess || cudaMalloc(&s.m2, kParams * 4) != cudaSuccess ||
      cudaMalloc(&s.W1b, kH * kF * 2) != cudaSuccess || cudaMalloc(&s.W2b, kH * kH * 2) != cudaSuccess ||
      cudaMalloc(&s.status, 4) != cudaSuccess)
    return false;
  // until parameters are given the network is zero (y = 0: the plain scheme)
  cudaMemset(s.p, 0, kParams * 4);
  cudaMemset(s.grad, 0, kParams * 4);
  cudaMemset(s.W1b, 0, kH * kF * 2);
  cudaMemset(s.W2b, 0, kH * kH * 2);
  cudaMemset(s.m1, 0, kParams * 4);
  cudaMemset(s.m2, 0, kParams * 4);
  cudaMemset(s.status, 0, 4);
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&s.sms, cudaDevAttrMultiProcessorCount, dev);
  return true;
}
static void mlp_free(MlpState &s) {
  cudaFree(s.p); cudaFree(s.grad); cudaFree(s.m1); cudaFree(s.m2); cudaFree(s.W1b); cudaFree(s.W2b); cudaFree(s.status);
  s = MlpState();
}
static MlpDev mlp_view(const MlpState &s) { return MlpDev{s.W1b, s.W2b, s.p}; }

static void mlp_sync_bf16(const MlpState &s, cudaStream_t st) { k_params_to_bf16<<<8, 256, 0, st>>>(s.p, s.W1b, s.W2b); }

static size_t fwd_smem() { return FwdSmem::END; }
static size_t train_smem() { return TrainSmem::END; }

// y[S] = MLP(X[S][16]) on the device (X BF16, 16-byte aligned rows)
int mlp_forward_dev(const MlpState &s, const __nv_bfloat16 *X, long long S, float *y, cudaStream_t st) {
  static bool attr = false;
  static int per_sm = 1;
  if (!attr) {
    if (cudaFuncSetAttribute(k_mlp_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fwd_smem()) != cudaSuccess)
      return -1;
    // A CTA's tile loop is grid-strided, so the grid is exactly the CTAs that
    // are resident together (a CTA started after another one's exit would run
    // its whole share late): the CTAs an SM's shared memory, registers and
    // threads hold, at most 512 / kFwdTmemCols for TMEM.  (Counted here from
    // the kernel's attributes: the runtime's occupancy query answered one CTA
    // per SM for this kernel, which the shared memory does not require.)
    if (cudaFuncSetAttribute(k_mlp_fwd, cudaFuncAttributePreferredSharedMemoryCarveout,
                             (int)cudaSharedmemCarveoutMaxShared) != cudaSuccess)
      return -1;
    cudaFuncAttributes fa{};
    int dev = 0, smem_sm = 0, resv = 0, regs_sm = 0, thr_sm = 0;
    if (cudaFuncGetAttributes(&fa, k_mlp_fwd) != cudaSuccess || cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&resv, cudaDevAttrReservedSharedMemoryPerBlock, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&thr_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev) != cudaSuccess)
      return -1;
    const int per_cta_smem = (int)(fwd_smem() + fa.sharedSizeBytes) + resv;
    const int regs_cta = ((fa.numRegs + 7) / 8) * 8 * 128;
    per_sm = std::min({smem_sm / per_cta_smem, regs_sm / std::max(regs_cta, 1), thr_sm / 128,
                       512 / (int)kFwdTmemCols});
    if (per_sm < 1) return -1;
    attr = true;
  }
  if (S <= 0) return 0;
  const long long tiles = (S + 127) / 128;
  const int grid = (int)std::min<long long>(tiles, (long long)s.sms * per_sm);
  k_mlp_fwd<<<grid, 128, fwd_smem(), st>>>(X, S, mlp_view(s), y, s.status);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// grad += d/dparams sum_s dy[s] y(X[s])
int mlp_grads_dev(const MlpState &s, const __nv_bfloat16 *X, const float *dy, long long S, cudaStream_t st) {
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)train_smem()) !=
        cudaSuccess)
      return -1;
    attr = true;
  }
  if (S <= 0) return 0;
  const long long tiles = (S + 127) / 128;
  const int grid = (int)std::min<long long>(tiles, (long long)s.sms);
  k_mlp_train<<<grid, 128, train_smem(), st>>>(X, dy, S, mlp_view(s), s.grad, s.status);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

static int mlp_status(const MlpState &s) {
  int h = 0;
  if (cudaMemcpy(&h, s.status, 4, cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
  return h ? -2 : 0;
}

}  // namespace fesom

namespace fesom {

// ---------------------------------------------------------------------------
// learned flux inside the engine
// ---------------------------------------------------------------------------
struct LearnedState {
  MlpState mlp;
  bool on = false;
  long long ncells = 0;  // edge cells of the dense edge schedule
  __nv_bfloat16 *feat[kBatchMax] = {};
  float *fscale[kBatchMax] = {}, *y[kBatchMax] = {};
  float *dy = nullptr, *target = nullptr, *hp = nullptr, *hm = nullptr;
  double *red = nullptr;  // per-block partial sums
  double volume = 0.0;    // sum of areasvol * hnode_new over wet cells
  float adam_b1 = 0.9f, adam_b2 = 0.999f;
};

namespace {

// adf: tracer t's slot of the batch's tracer-interleaved antidiffusive fluxes
// (stride nt)
__global__ void __launch_bounds__(kThreads) k_learn_apply(DMeshT<float> m, float *adf, int nt, const float *scale,
                                                         const float *y) {
  extern __shared__ int smem[];
  int *s_off = smem, *s_item = smem + kMaxItemsPerBlock + 1;
  const CellMap cm = map_cells(m.edge_sched, blockIdx.x, s_off, s_item);
  for (int lc = threadIdx.x; lc < cm.nc; lc += blockDim.x) {
    const int j = s_item[lc], e = cm.i0 + j, k = lc - (s_off[j] - cm.c0), cell = cm.c0 + lc;
    adf[((size_t)e * m.S + k) * nt] += scale[cell] * y[cell];
  }
}

// dL/dy for L = sum_n V_n (T_n - target_n)^2 / sum V after an unlimited step:
// an edge flux f enters T_n1 with +dt/V and T_n2 with -dt/V, f = base + scale y
// With the FCT limiter (adf, rp, rm set; rp and rm point into one array of
// (R+, R-) pairs, stride 2), the flux entering the update is
// ae * f with the limiter's factor ae held at its forward value.
__global__ void __launch_bounds__(kThreads) k_learn_dy(DMeshT<float> m, const float *T, const float *target,
                                                      const float *scale, float c, const float *adf, const float *rp,
                                                      const float *rm, float *dy) {
  extern __shared__ int smem[];
  int *s_off = smem, *s_item = smem + kMaxItemsPerBlock + 1;
  const CellMap cm = map_cells(m.edge_sched, blockIdx.x, s_off, s_item);
  for (int lc = threadIdx.x; lc < cm.nc; lc += blockDim.x) {
    const int j = s_item[lc], e = cm.i0 + j, k = lc - (s_off[j] - cm.c0), cell = cm.c0 + lc;
    const int2 nn = m.edge_nodes[e];
    const size_t o1 = (size_t)nn.x * m.S + k, o2 = (size_t)nn.y * m.S + k;
    float ae = 1.0f;
    if (rp) {
      const float f = adf[(size_t)e * m.S + k];
      ae = f >= 0.0f ? fminf(1.0f, fminf(rp[2 * (o1)], rm[2 * (o2)])) : fminf(1.0f, fminf(rm[2 * (o1)], rp[2 * (o2)]));
    }
    dy[cell] = ae * scale[cell] * c * ((T[o1] - target[o1]) - (T[o2] - target[o2]));
  }
}

// ---- gradient through the FCT limiter (Zalesak) ------------------------------
// rho = dL/d(flux into a cell) = 2 dt (T - target) / sum V for every cell (the
// update divides a flux by areasvol * hnode_new, the loss weights by it).
__device__ __forceinline__ float learn_rho(const float *T, const float *target, size_t o, float c) {
  return c * (T[o] - target[o]);
}

// Per node level: G+/- = sum over every limited flux (incident edges, the
// column's interfaces) whose limiting factor is this cell's R+/- (the active
// argument of the min, ties as in k_col3) of dL/d(limited flux) * flux; then
// dL/dP+/- = G+/- * dR+/-/dP+/- where R+/- < 1 (R = Q / (P dt / V +- eps)).
__global__ void __launch_bounds__(kThreads) k_learn_fct_g(DMeshT<float> m, const float *T, const float *target,
                                                         float c, const float *adfh, const float *adfv,
                                                         const float *rp, const float *rm, float dt, float *hp,
                                                         float *hm) {
  extern __shared__ int smem[];
  int *s_off = smem, *s_item = smem + kMaxItemsPerBlock + 1;
  const CellMap cm = map_cells(m.node_sched, blockIdx.x, s_off, s_item);
  const int S = m.S;
  for (int lc = threadIdx.x; lc < cm.nc; lc += blockDim.x) {
    const int j = s_item[lc], n = cm.i0 + j, k = lc - (s_off[j] - cm.c0), nz = k + 1;
    const size_t col = (size_t)n * S, o = col + k;
    const int nlev = m.nlev_node[n];
    const float *av = adfv + col;
    const float rpn = rp[2 * (o)], rmn = rm[2 * (o)];
    const float rho = learn_rho(T, target, o, c);
    float gp = 0.f, gm = 0.f;
    float fp = 0.f + (fmax2(0.f, av[k]) + fmax2(0.f, -av[k + 1]));
    float fm = 0.f + (fmin2(0.f, av[k]) + fmin2(0.f, -av[k + 1]));
    for (int p = m.ne_ptr[n]; p < m.ne_ptr[n + 1]; p++) {
      const int4 q = m.ne4[p];
      if (nz > q.z) continue;
      const bool second = q.x & 1;
      const float f = adfh[(size_t)(q.x >> 1) * S + k];
      if (second) { fp = fp + fmax2(0.f, -f); fm = fm + fmin2(0.f, -f); }
      else { fp = fp + fmax2(0.f, f); fm = fm + fmin2(0.f, f); }
      const size_t oo = (size_t)q.y * S + k;
      const float rpo = rp[2 * (oo)], rmo = rm[2 * (oo)], rho_o = learn_rho(T, target, oo, c);
      const float rp1 = second ? rpo : rpn, rm1 = second ? rmo : rmn, rp2 = second ? rpn : rpo, rm2 = second ? rmn : rmo;
      const float dLdF = second ? (rho_o - rho) : (rho - rho_o);  // first node gains the flux
      if (f >= 0.f) {
        const float a1 = rp1 < 1.f ? rp1 : 1.f;
        if (rm2 < a1) { if (second) gm += dLdF * f; }       // node 2's R- limits
        else if (rp1 < 1.f) { if (!second) gp += dLdF * f; }  // node 1's R+ limits
      } else {
        const float a1 = rm1 < 1.f ? rm1 : 1.f;
        if (rp2 < a1) { if (second) gp += dLdF * f; }
        else if (rm1 < 1.f) { if (!second) gm += dLdF * f; }
      }
    }
    // interface i = nz (top of this cell): the cell is the limiter's "below" cell
    {
      const int i = nz;
      if (i < nlev) {
        const float f = av[i - 1];
        const float dLdF = rho - (i >= 2 ? learn_rho(T, target, col + i - 2, c) : 0.f);
        if (i == 1) {
          if (f >= 0.f) { if (rpn < 1.f) gp += dLdF * f; }
          else if (rmn < 1.f) gm += dLdF * f;
        } else if (f >= 0.f) {
          const float r_up = rm[2 * (col + i - 2)], a1 = r_up < 1.f ? r_up : 1.f;
          if (rpn < a1) gp += dLdF * f;
        } else {
          const float r_up = rp[2 * (col + i - 2)], a1 = r_up < 1.f ? r_up : 1.f;
          if (rmn < a1) gm += dLdF * f;
        }
      }
    }
    // interface i = nz + 1 (bottom of this cell): the cell is the "above" cell
    {
      const int i = nz + 1;
      if (i < nlev) {
        const float f = av[i - 1];
        const float dLdF = learn_rho(T, target, col + i - 1, c) - rho;
        if (f >= 0.f) {
          const float a1 = rmn < 1.f ? rmn : 1.f;
          if (!(rp[2 * (col + i - 1)] < a1) && rmn < 1.f) gm += dLdF * f;
        } else {
          const float a1 = rpn < 1.f ? rpn : 1.f;
          if (!(rm[2 * (col + i - 1)] < a1) && rpn < 1.f) gp += dLdF * f;
        }
      }
    }
    const double dtv = (double)dt / (double)m.areasvol[o], e64 = (double)1e-16f;
    const double fluxp = (double)fp * dtv + e64, fluxm = (double)fm * dtv - e64;
    hp[o] = rpn < 1.f ? (float)((double)gp * (-(double)rpn / fluxp) * dtv) : 0.f;
    hm[o] = rmn < 1.f ? (float)((double)gm * (-(double)rmn / fluxm) * dtv) : 0.f;
  }
}

// dL/dy per edge cell through the limited update: the limited flux ae * f
// plus f's share of both nodes' P+/- sums
__global__ void __launch_bounds__(kThreads) k_learn_dy_fct(DMeshT<float> m, const float *T, const float *target,
                                                          float c, const float *scale, const float *adfh,
                                                          const float *rp, const float *rm, const float *hp,
                                                          const float *hm, float *dy) {
  extern __shared__ int smem[];
  int *s_off = smem, *s_item = smem + kMaxItemsPerBlock + 1;
  const CellMap cm = map_cells(m.edge_sched, blockIdx.x, s_off, s_item);
  for (int lc = threadIdx.x; lc < cm.nc; lc += blockDim.x) {
    const int j = s_item[lc], e = cm.i0 + j, k = lc - (s_off[j] - cm.c0), cell = cm.c0 + lc;
    const int2 nn = m.edge_nodes[e];
    const size_t o1 = (size_t)nn.x * m.S + k, o2 = (size_t)nn.y * m.S + k;
    const float f = adfh[(size_t)e * m.S + k];
    const float ae = f >= 0.f ? fmin2(fmin2(1.f, rp[2 * (o1)]), rm[2 * (o2)]) : fmin2(fmin2(1.f, rm[2 * (o1)]), rp[2 * (o2)]);
    float g = ae * (learn_rho(T, target, o1, c) - learn_rho(T, target, o2, c));
    if (f > 0.f) g += hp[o1] - hm[o2];
    else if (f < 0.f) g += hm[o1] - hp[o2];
    dy[cell] = scale[cell] * g;
  }
}

__global__ void __launch_bounds__(kThreads) k_learn_loss(DMeshT<float> m, const float *T, const float *target,
                                                        double *part) {
  extern __shared__ int smem[];
  int *s_off = smem, *s_item = smem + kMaxItemsPerBlock + 1;
  __shared__ double red[kThreads];
  const CellMap cm = map_cells(m.node_sched, blockIdx.x, s_off, s_item);
  double acc = 0.0;
  for (int lc = threadIdx.x; lc < cm.nc; lc += blockDim.x) {
    const int j = s_item[lc], n = cm.i0 + j, k = lc - (s_off[j] - cm.c0);
    const size_t o = (size_t)n * m.S + k;
    const double r = (double)T[o] - (double)target[o];
    acc += (double)m.areasvol[o] * (double)m.hnode_new[o] * r * r;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void k_adam(float *p, const float *g, float *m1, float *m2, int n, float lr, float b1, float b2, float bc1,
                       float bc2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.f - b1) * gi, b = b2 * m2[i] + (1.f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    p[i] -= lr * (a / bc1) / (sqrtf(b / bc2) + 1e-8f);
  }
}

template <typename T>
T *dmalloc(size_t n) {
  void *p = nullptr;
  CK(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
  return (T *)p;
}

}  // namespace

void learned_release(EngineImpl &P) {
  if (!P.learn) return;
  LearnedState &L = *P.learn;
  mlp_free(L.mlp);
  for (int t = 0; t < kBatchMax; t++) {
    cudaFree(L.feat[t]);
    cudaFree(L.fscale[t]);
    cudaFree(L.y[t]);
  }
  cudaFree(L.dy);
  cudaFree(L.target);
  cudaFree(L.hp);
  cudaFree(L.hm);
  cudaFree(L.red);
  delete P.learn;
  P.learn = nullptr;
}

void learned_correct_f32(EngineImpl &P, int nt, const FusedArgs<float, float> &a) {
  LearnedState &L = *P.learn;
  for (int t = 0; t < nt; t++) {
    if (mlp_forward_dev(L.mlp, a.feat[t], L.ncells, L.y[t], P.stream) != 0)
      throw std::runtime_error("learned flux: MLP forward launch failed");
    if (P.dm32.edge_sched.nblk > 0)
      k_learn_apply<<<P.dm32.edge_sched.nblk, kThreads, smem_edge(), P.stream>>>(P.dm32, a.adf_h[t], nt, a.fscale[t],
                                                                                  L.y[t]);
    CK(cudaGetLastError());
  }
}

// feature / scale buffers of the batch slots, for the run_batch of engine.cu
void learned_slot_buffers(EngineImpl &P, int t, void **feat, void **scale) {
  LearnedState &L = *P.learn;
  if (!L.feat[t]) {
    L.feat[t] = dmalloc<__nv_bfloat16>((size_t)L.ncells * kF);
    L.fscale[t] = dmalloc<float>(L.ncells);
    L.y[t] = dmalloc<float>(L.ncells);
  }
  *feat = L.feat[t];
  *scale = L.fscale[t];
}
bool learned_active(const EngineImpl &P) { return P.learn && P.learn->on; }

void Engine::set_learned(const float *params, bool on) {
  EngineImpl &P = *p_;
  if (P.prec != Precision::FP32) throw std::invalid_argument("the learned flux runs in the FP32 mode");
  CK(cudaStreamSynchronize(P.stream));
  if (!P.learn) {
    P.learn = new LearnedState();
    LearnedState &L = *P.learn;
    if (!mlp_alloc(L.mlp)) throw std::runtime_error("learned flux: device allocation failed");
    const MeshHost &M = P.mesh;
    long long cells = 0;
    for (int e = 0; e < M.edge2D; e++) cells += M.edge_levels(e);
    L.ncells = cells;
    double vol = 0.0;
    const int L1 = M.nl - 1;
    for (int n = 0; n < M.nod2D; n++)
      for (int k = 0; k < M.nlev_node[n] - 1; k++)
        vol += M.areasvol[(size_t)n * M.nl + k] * M.hnode_new[(size_t)n * L1 + k];
    L.volume = vol;
    L.dy = dmalloc<float>(L.ncells);
    L.target = dmalloc<float>((size_t)M.nod2D * P.S);
    CK(cudaMemset(L.target, 0, (size_t)M.nod2D * P.S * sizeof(float)));
    L.red = dmalloc<double>(std::max(1, P.dm32.node_sched.nblk));
  }
  LearnedState &L = *P.learn;
  if (params) {
    CK(cudaMemcpy(L.mlp.p, params, kParams * sizeof(float), cudaMemcpyHostToDevice));
    CK(cudaMemset(L.mlp.m1, 0, kParams * sizeof(float)));
    CK(cudaMemset(L.mlp.m2, 0, kParams * sizeof(float)));
    L.mlp.adam_t = 0;
    mlp_sync_bf16(L.mlp, P.stream);
    CK(cudaStreamSynchronize(P.stream));
  }
  L.on = on;
}

bool Engine::learned() const { return learned_active(*p_); }

void Engine::get_learned_grad(float *grad) const {
  if (!p_->learn) throw std::runtime_error("no learned flux");
  CK(cudaMemcpy(grad, p_->learn->mlp.grad, kParams * sizeof(float), cudaMemcpyDeviceToHost));
}

void Engine::get_learned(float *params) const {
  if (!p_->learn) throw std::runtime_error("no learned flux");
  CK(cudaMemcpy(params, p_->learn->mlp.p, kParams * sizeof(float), cudaMemcpyDeviceToHost));
}

double Engine::learn_step(const double *T_in, const double *T_target, double dt, double lr, bool update, bool fct,
                          bool fct_grad) {
  EngineImpl &P = *p_;
  if (!P.learn) throw std::runtime_error("no learned flux: call set_learned first");
  if (P.tr.empty()) throw std::runtime_error("no tracers");
  LearnedState &L = *P.learn;
  const TracerScheme keep = P.tr[0].sch;
  const bool keep_on = L.on;
  TracerScheme sch;
  sch.hor = 1;  // MUSCL
  sch.ver = 1;  // PPM
  sch.lim = fct ? 1 : 0;  // without FCT the state is linear in the correction
  P.tr[0].sch = sch;
  L.on = true;
  try {
    set_values(0, T_in, true);
    step_tracer(0, dt, true);
  } catch (...) {
    P.tr[0].sch = keep;
    L.on = keep_on;
    throw;
  }
  P.tr[0].sch = keep;
  L.on = keep_on;
  stage_upload(P, T_target);
  stage_pack(P, 0.0, L.target, nullptr, nullptr);
  const DMeshT<float> &m = P.dm32;
  const float *T = (const float *)P.tr[0].T;
  k_learn_loss<<<m.node_sched.nblk, kThreads, smem_edge(), P.stream>>>(m, T, L.target, L.red);
  CK(cudaGetLastError());
  std::vector<double> part(std::max(1, m.node_sched.nblk));
  CK(cudaMemcpyAsync(part.data(), L.red, part.size() * sizeof(double), cudaMemcpyDeviceToHost, P.stream));
  if (update) {
    const float c = (float)(2.0 * dt / L.volume);
    if (fct && fct_grad) {
      if (!L.hp) {
        L.hp = dmalloc<float>((size_t)P.mesh.nod2D * P.S);
        L.hm = dmalloc<float>((size_t)P.mesh.nod2D * P.S);
      }
      k_learn_fct_g<<<m.node_sched.nblk, kThreads, smem_edge(), P.stream>>>(
          m, T, L.target, c, (const float *)P.adfh[0], (const float *)P.adfv[0], (const float *)P.rpm[0],
          (const float *)P.rpm[0] + 1, (float)dt, L.hp, L.hm);
      CK(cudaGetLastError());
      k_learn_dy_fct<<<m.edge_sched.nblk, kThreads, smem_edge(), P.stream>>>(
          m, T, L.target, c, L.fscale[0], (const float *)P.adfh[0], (const float *)P.rpm[0], (const float *)P.rpm[0] + 1,
          L.hp, L.hm, L.dy);
    } else {
      k_learn_dy<<<m.edge_sched.nblk, kThreads, smem_edge(), P.stream>>>(
          m, T, L.target, L.fscale[0], c, (const float *)P.adfh[0], fct ? (const float *)P.rpm[0] : nullptr,
          fct ? (const float *)P.rpm[0] + 1 : nullptr, L.dy);
    }
    CK(cudaGetLastError());
    CK(cudaMemsetAsync(L.mlp.grad, 0, kParams * sizeof(float), P.stream));
    if (mlp_grads_dev(L.mlp, L.feat[0], L.dy, L.ncells, P.stream) != 0)
      throw std::runtime_error("learned flux: MLP backward launch failed");
    L.mlp.adam_t++;
    const float bc1 = 1.f - powf(L.adam_b1, (float)L.mlp.adam_t), bc2 = 1.f - powf(L.adam_b2, (float)L.mlp.adam_t);
    k_adam<<<8, 256, 0, P.stream>>>(L.mlp.p, L.mlp.grad, L.mlp.m1, L.mlp.m2, kParams, (float)lr, L.adam_b1, L.adam_b2,
                                   bc1, bc2);
    CK(cudaGetLastError());
    mlp_sync_bf16(L.mlp, P.stream);
  }
  CK(cudaStreamSynchronize(P.stream));
  if (mlp_status(L.mlp) != 0) throw std::runtime_error("learned flux: a tensor-core wait timed out");
  double s = 0.0;
  for (double x : part) s += x;
  return s / L.volume;
}

}  // namespace fesom

extern "C" int tracer_mlp_num_params(void) { return fesom::kParams; }

extern "C" int tracer_mlp_forward(const uint16_t *X, long long S, const float *params, float *y) {
  if (!X || !params || !y || S < 0) return -1;
  MlpState s;
  __nv_bfloat16 *dX = nullptr;
  float *dy = nullptr;
  int rc = -1;
  if (mlp_alloc(s) && cudaMalloc(&dX, std::max<long long>(S, 1) * kF * 2) == cudaSuccess &&
      cudaMalloc(&dy, std::max<long long>(S, 1) * 4) == cudaSuccess &&
      cudaMemcpy(s.p, params, kParams * 4, cudaMemcpyHostToDevice) == cudaSuccess &&
      cudaMemcpy(dX, X, (size_t)S * kF * 2, cudaMemcpyHostToDevice) == cudaSuccess) {
    mlp_sync_bf16(s, 0);
    if (mlp_forward_dev(s, dX, S, dy, 0) == 0 && cudaDeviceSynchronize() == cudaSuccess &&
        cudaMemcpy(y, dy, (size_t)S * 4, cudaMemcpyDeviceToHost) == cudaSuccess)
      rc = mlp_status(s);
  }
  cudaFree(dX);
  cudaFree(dy);
  mlp_free(s);
  return rc;
}

extern "C" int tracer_mlp_grads(const uint16_t *X, const float *dyv, long long S, const float *params, float *grads) {
  if (!X || !dyv || !params || !grads || S < 0) return -1;
  MlpState s;
  __nv_bfloat16 *dX = nullptr;
  float *ddy = nullptr;
  int rc = -1;
  if (mlp_alloc(s) && cudaMalloc(&dX, std::max<long long>(S, 1) * kF * 2) == cudaSuccess &&
      cudaMalloc(&ddy, std::max<long long>(S, 1) * 4) == cudaSuccess &&
      cudaMemcpy(s.p, params, kParams * 4, cudaMemcpyHostToDevice) == cudaSuccess &&
      cudaMemcpy(dX, X, (size_t)S * kF * 2, cudaMemcpyHostToDevice) == cudaSuccess &&
      cudaMemcpy(ddy, dyv, (size_t)S * 4, cudaMemcpyHostToDevice) == cudaSuccess &&
      cudaMemset(s.grad, 0, kParams * 4) == cudaSuccess) {
    mlp_sync_bf16(s, 0);
    if (mlp_grads_dev(s, dX, ddy, S, 0) == 0 && cudaDeviceSynchronize() == cudaSuccess &&
        cudaMemcpy(grads, s.grad, kParams * 4, cudaMemcpyDeviceToHost) == cudaSuccess)
      rc = mlp_status(s);
  }
  cudaFree(dX);
  cudaFree(ddy);
  mlp_free(s);
  return rc;
}

extern "C" int tracer_selftest_umma(int N, int K, const uint16_t *A, const uint16_t *B, float *D) {
  if (N < 16 || N > 256 || N % 16 || K < 16 || K > 256 || K % 16 || !A || !B || !D) return -1;
  const size_t na = (size_t)128 * K, nb = (size_t)N * K, nd = (size_t)128 * N;
  __nv_bfloat16 *dA = nullptr, *dB = nullptr;
  float *dD = nullptr;
  int *dst = nullptr;
  int rc = -1;
  const size_t smem = ((na * 2 + 1023) & ~(size_t)1023) + nb * 2 + 1024;
  if (cudaMalloc(&dA, na * 2) == cudaSuccess && cudaMalloc(&dB, nb * 2) == cudaSuccess &&
      cudaMalloc(&dD, nd * 4) == cudaSuccess && cudaMalloc(&dst, sizeof(int)) == cudaSuccess &&
      cudaMemcpy(dA, A, na * 2, cudaMemcpyHostToDevice) == cudaSuccess &&
      cudaMemcpy(dB, B, nb * 2, cudaMemcpyHostToDevice) == cudaSuccess &&
      cudaMemset(dst, 0, sizeof(int)) == cudaSuccess &&
      cudaFuncSetAttribute(k_umma_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) == cudaSuccess) {
    k_umma_selftest<<<1, 128, smem>>>(dA, dB, dD, N, K, dst);
    int st = 0;
    if (cudaDeviceSynchronize() == cudaSuccess && cudaMemcpy(&st, dst, sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess &&
        cudaMemcpy(D, dD, nd * 4, cudaMemcpyDeviceToHost) == cudaSuccess)
      rc = st ? -2 : 0;
  }
  cudaFree(dA);
  cudaFree(dB);
  cudaFree(dD);
  cudaFree(dst);
  return rc;
}
