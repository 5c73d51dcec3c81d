// Learned antidiffusive edge flux: a per-edge-level MLP (16 -> 64 -> 64 -> 1,
// GELU, BF16 weights and activations, FP32 accumulation) on the fifth-
// generation tensor cores (tcgen05.mma, accumulators in TMEM).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "../../include/fesom_tracer.h"
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

}  // namespace
}  // namespace fesom

using namespace fesom;

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
