// Host <-> device transfer of tracer fields.
//
// Tracers cross the C ABI as FP64 arrays in the reference's layout (nl-1,
// nod2D).  They travel over PCIe unchanged into a device staging array of the
// same layout; kernels then repack them into the engine's padded storage
// columns (stride S), converting to the storage type and applying the 16-bit
// storage offset on wet cells.  Reads run the same path backwards.
//
// Host buffers registered with tracer_host_register (page-locked) are copied
// by one DMA each way.  Pageable buffers go through a ring of pinned slots:
// host threads copy chunk i into a slot while the DMA engine moves chunk i-1.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <thread>
#include <type_traits>
#include <vector>

#include "engine_impl.hpp"

namespace fesom {

// ---------------------------------------------------------------------------
// registry of page-locked host ranges
// ---------------------------------------------------------------------------
namespace {
std::mutex g_pin_mu;
std::map<const char *, size_t> g_pinned;  // start -> bytes

bool range_pinned(const void *p, size_t bytes) {
  std::lock_guard<std::mutex> lk(g_pin_mu);
  const char *c = (const char *)p;
  auto it = g_pinned.upper_bound(c);
  if (it == g_pinned.begin()) return false;
  --it;
  return c >= it->first && c + bytes <= it->first + it->second;
}
}  // namespace

int host_register(void *p, size_t bytes) {
  if (!p || !bytes) return -1;
  if (cudaHostRegister(p, bytes, cudaHostRegisterDefault) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  std::lock_guard<std::mutex> lk(g_pin_mu);
  g_pinned[(const char *)p] = bytes;
  return 0;
}

int host_unregister(void *p) {
  {
    std::lock_guard<std::mutex> lk(g_pin_mu);
    auto it = g_pinned.find((const char *)p);
    if (it == g_pinned.end()) return -1;
    g_pinned.erase(it);
  }
  return cudaHostUnregister(p) == cudaSuccess ? 0 : -1;
}

// ---------------------------------------------------------------------------
// host side: parallel copies and the pinned ring
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kSlotBytes = size_t(32) << 20;  // 32 MiB per pinned slot

void parallel_copy(void *dst, const void *src, size_t bytes) {
  const size_t per = size_t(4) << 20;
  unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const int nt = (int)std::min<size_t>(std::min<unsigned>(hw, 16u), std::max<size_t>(1, bytes / per));
  if (nt <= 1) {
    std::memcpy(dst, src, bytes);
    return;
  }
  const size_t part = (bytes / nt + 63) / 64 * 64;
  std::vector<std::thread> th;
  th.reserve(nt - 1);
  for (int t = 1; t < nt; t++) {
    const size_t a = std::min(bytes, part * t), b = std::min(bytes, part * (t + 1));
    if (b > a) th.emplace_back([=] { std::memcpy((char *)dst + a, (const char *)src + a, b - a); });
  }
  std::memcpy(dst, src, std::min(bytes, part));
  for (auto &x : th) x.join();
}

void ensure_ring(EngineImpl &P) {
  if (P.ring[0]) return;
  for (int s = 0; s < EngineImpl::kRing; s++) {
    CK(cudaHostAlloc(&P.ring[s], kSlotBytes, cudaHostAllocDefault));
    CK(cudaEventCreateWithFlags(&P.ring_ev[s], cudaEventDisableTiming));
  }
}

void ensure_stage(EngineImpl &P) {
  const size_t n = (size_t)(P.mesh.nl - 1) * P.mesh.nod2D;
  if (!P.stage_d) P.stage_d = P.dalloc<double>(std::max<size_t>(n, 1));
}

const int *nlev_dev(const EngineImpl &P) {
  return P.prec == Precision::FP64 ? P.dm64.nlev_node : P.dm32.nlev_node;
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
template <typename TS>
__device__ __forceinline__ TS to_ts(double v) {
  if constexpr (std::is_same<TS, double>::value) return v;
  else if constexpr (std::is_same<TS, float>::value) return (float)v;
  else if constexpr (std::is_same<TS, __nv_bfloat16>::value) return __float2bfloat16_rn((float)v);
  else return __float2half_rn((float)v);
}
template <typename TS>
__device__ __forceinline__ double from_ts(TS v) {
  if constexpr (std::is_same<TS, double>::value) return v;
  else if constexpr (std::is_same<TS, float>::value) return (double)v;
  else if constexpr (std::is_same<TS, __nv_bfloat16>::value) return (double)__bfloat162float(v);
  else return (double)__half2float(v);
}

// (L, N) doubles -> up to three storage arrays of stride S; wet cells store
// v - off, dry cells v, padding 0
template <typename TS>
__global__ void k_pack(const double *__restrict__ src, const int *__restrict__ nlev, int L, int S, long long N,
                       double off, TS *d0, TS *d1, TS *d2) {
  const long long total = N * S;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long n = i / S;
    const int k = (int)(i - n * S);
    TS o = TS(0.0f);
    if (k < L) {
      const double v = src[n * L + k];
      o = to_ts<TS>(k < nlev[n] - 1 ? v - off : v);
    }
    d0[i] = o;
    if (d1) d1[i] = o;
    if (d2) d2[i] = o;
  }
}

// storage array of stride S -> (L, N) doubles (wet cells plus off)
template <typename TS>
__global__ void k_unpack(const TS *__restrict__ s, const int *__restrict__ nlev, int L, int S, long long N, double off,
                         double *dst) {
  const long long total = N * L;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long n = i / L;
    const int k = (int)(i - n * L);
    const double v = from_ts<TS>(s[n * S + k]);
    dst[i] = k < nlev[n] - 1 ? v + off : v;
  }
}

// wet cells of a storage array: anomaly re-expressed against a new offset
template <typename TS>
__global__ void k_reoffset(TS *s, const int *__restrict__ nlev, int S, long long N, double off_old, double off_new) {
  const long long total = N * S;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long n = i / S;
    const int k = (int)(i - n * S);
    if (k < nlev[n] - 1) s[i] = to_ts<TS>(from_ts<TS>(s[i]) + off_old - off_new);
  }
}

__device__ __forceinline__ void two_sum_d(double a, double b, double &s, double &e) {
  s = a + b;
  const double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}

// per block: compensated sum of the wet cells of (L, N) doubles and their count
__global__ void k_wet_sum(const double *__restrict__ src, const int *__restrict__ nlev, int L, long long N,
                          double *out) {
  double s = 0.0, c = 0.0, cnt = 0.0;
  for (long long n = (long long)blockIdx.x * blockDim.y + threadIdx.y; n < N; n += (long long)gridDim.x * blockDim.y) {
    const int w = nlev[n] - 1;
    for (int k = threadIdx.x; k < w; k += blockDim.x) {
      double t, e;
      two_sum_d(s, src[n * L + k], t, e);
      s = t;
      c += e;
      cnt += 1.0;
    }
  }
  __shared__ double sh[3][256];
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  sh[0][tid] = s;
  sh[1][tid] = c;
  sh[2][tid] = cnt;
  __syncthreads();
  if (tid == 0) {
    double S0 = 0.0, C0 = 0.0, K0 = 0.0;
    for (int t = 0; t < (int)(blockDim.x * blockDim.y); t++) {
      double u, e;
      two_sum_d(S0, sh[0][t], u, e);
      S0 = u;
      C0 += e + sh[1][t];
      K0 += sh[2][t];
    }
    out[3 * blockIdx.x] = S0;
    out[3 * blockIdx.x + 1] = C0;
    out[3 * blockIdx.x + 2] = K0;
  }
}

constexpr int kGrid = 148 * 8, kBlock = 256;

// Statistics of one tracer over the (nl-1, nod2D) values the host would read
// back (wet cells T = storage + off, dry cells the storage itself): per block
// the minimum and maximum of the non-NaN values, the NaN count and a
// Neumaier-compensated sum, in a fixed assignment of cells to threads and a
// fixed reduction order, so the result does not depend on scheduling.
constexpr int kStatBlocks = 296, kStatThreads = 256;
template <typename TS>
__global__ void __launch_bounds__(kStatThreads) k_stats(const TS *__restrict__ s, const int *__restrict__ nlev,
                                                        int L, int S, long long N, double off, double *out) {
  double mn = INFINITY, mx = -INFINITY, nan = 0.0, sm = 0.0, c = 0.0;
  const long long total = N * L;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long n = i / L;
    const int k = (int)(i - n * L);
    const double raw = from_ts<TS>(s[n * S + k]);
    const double v = k < nlev[n] - 1 ? raw + off : raw;
    if (v != v) {
      nan += 1.0;
      continue;
    }
    mn = fmin(mn, v);
    mx = fmax(mx, v);
    double t, e;
    two_sum_d(sm, v, t, e);
    sm = t;
    c += e;
  }
  __shared__ double sh[5][kStatThreads];
  const int tid = threadIdx.x;
  sh[0][tid] = mn; sh[1][tid] = mx; sh[2][tid] = nan; sh[3][tid] = sm; sh[4][tid] = c;
  __syncthreads();
  for (int w = kStatThreads / 2; w > 0; w >>= 1) {
    if (tid < w) {
      sh[0][tid] = fmin(sh[0][tid], sh[0][tid + w]);
      sh[1][tid] = fmax(sh[1][tid], sh[1][tid + w]);
      sh[2][tid] += sh[2][tid + w];
      double t, e;
      two_sum_d(sh[3][tid], sh[3][tid + w], t, e);
      sh[3][tid] = t;
      sh[4][tid] += sh[4][tid + w] + e;
    }
    __syncthreads();
  }
  if (tid < 5) out[5 * blockIdx.x + tid] = sh[tid][0];
}

template <typename TS>
void pack_t(EngineImpl &P, double off, void *d0, void *d1, void *d2) {
  k_pack<TS><<<kGrid, kBlock, 0, P.stream>>>(P.stage_d, nlev_dev(P), P.mesh.nl - 1, P.S, P.mesh.nod2D, off,
                                             (TS *)d0, (TS *)d1, (TS *)d2);
  CK(cudaGetLastError());
}
template <typename TS>
void unpack_t(EngineImpl &P, const void *s, double off) {
  k_unpack<TS><<<kGrid, kBlock, 0, P.stream>>>((const TS *)s, nlev_dev(P), P.mesh.nl - 1, P.S, P.mesh.nod2D, off,
                                               P.stage_d);
  CK(cudaGetLastError());
}
template <typename TS>
void reoffset_t(EngineImpl &P, void *s, double off_old, double off_new) {
  k_reoffset<TS><<<kGrid, kBlock, 0, P.stream>>>((TS *)s, nlev_dev(P), P.S, P.mesh.nod2D, off_old, off_new);
  CK(cudaGetLastError());
}

}  // namespace

// ---------------------------------------------------------------------------
// engine-facing functions
// ---------------------------------------------------------------------------
void stage_upload(EngineImpl &P, const double *host) {
  ensure_stage(P);
  const size_t bytes = sizeof(double) * (size_t)(P.mesh.nl - 1) * P.mesh.nod2D;
  if (!bytes) return;
  if (range_pinned(host, bytes)) {
    CK(cudaMemcpyAsync(P.stage_d, host, bytes, cudaMemcpyHostToDevice, P.stream));
    return;
  }
  ensure_ring(P);
  for (size_t a = 0, c = 0; a < bytes; a += kSlotBytes, c++) {
    const int s = (int)(c % EngineImpl::kRing);
    const size_t n = std::min(kSlotBytes, bytes - a);
    CK(cudaEventSynchronize(P.ring_ev[s]));  // the slot's previous DMA is done
    parallel_copy(P.ring[s], (const char *)host + a, n);
    CK(cudaMemcpyAsync((char *)P.stage_d + a, P.ring[s], n, cudaMemcpyHostToDevice, P.stream));
    CK(cudaEventRecord(P.ring_ev[s], P.stream));
  }
}

void stage_download(EngineImpl &P, double *host) {
  const size_t bytes = sizeof(double) * (size_t)(P.mesh.nl - 1) * P.mesh.nod2D;
  if (!bytes) return;
  if (range_pinned(host, bytes)) {
    CK(cudaMemcpyAsync(host, P.stage_d, bytes, cudaMemcpyDeviceToHost, P.stream));
    CK(cudaStreamSynchronize(P.stream));
    return;
  }
  ensure_ring(P);
  const size_t nchunks = (bytes + kSlotBytes - 1) / kSlotBytes;
  auto issue = [&](size_t c) {
    const int s = (int)(c % EngineImpl::kRing);
    const size_t a = c * kSlotBytes, n = std::min(kSlotBytes, bytes - a);
    CK(cudaMemcpyAsync(P.ring[s], (const char *)P.stage_d + a, n, cudaMemcpyDeviceToHost, P.stream));
    CK(cudaEventRecord(P.ring_ev[s], P.stream));
  };
  for (size_t c = 0; c < std::min<size_t>(nchunks, EngineImpl::kRing); c++) issue(c);
  for (size_t c = 0; c < nchunks; c++) {
    const int s = (int)(c % EngineImpl::kRing);
    const size_t a = c * kSlotBytes, n = std::min(kSlotBytes, bytes - a);
    CK(cudaEventSynchronize(P.ring_ev[s]));
    parallel_copy((char *)host + a, P.ring[s], n);
    if (c + EngineImpl::kRing < nchunks) issue(c + EngineImpl::kRing);
  }
}

double stage_wet_mean(EngineImpl &P) {
  const int blocks = 296;
  double *d = P.dalloc<double>(3 * blocks);
  k_wet_sum<<<blocks, dim3(32, 8), 0, P.stream>>>(P.stage_d, nlev_dev(P), P.mesh.nl - 1, P.mesh.nod2D, d);
  CK(cudaGetLastError());
  std::vector<double> h(3 * blocks);
  P.d2h(h.data(), d, h.size() * sizeof(double));
  P.dfree(d);
  double s = 0.0, c = 0.0, k = 0.0;
  for (int b = 0; b < blocks; b++) {
    const double x = h[3 * b], t = s + x;
    c += ((std::fabs(s) >= std::fabs(x)) ? (s - t) + x : (x - t) + s) + h[3 * b + 1];
    s = t;
    k += h[3 * b + 2];
  }
  return k > 0.0 ? (s + c) / k : 0.0;
}

void stage_pack(EngineImpl &P, double off, void *d0, void *d1, void *d2) {
  switch (P.prec) {
    case Precision::FP64: pack_t<double>(P, off, d0, d1, d2); break;
    case Precision::FP32: pack_t<float>(P, off, d0, d1, d2); break;
    case Precision::BF16: pack_t<__nv_bfloat16>(P, off, d0, d1, d2); break;
    case Precision::FP16: pack_t<__half>(P, off, d0, d1, d2); break;
  }
}

void stage_unpack(EngineImpl &P, const void *s, double off) {
  ensure_stage(P);
  switch (P.prec) {
    case Precision::FP64: unpack_t<double>(P, s, off); break;
    case Precision::FP32: unpack_t<float>(P, s, off); break;
    case Precision::BF16: unpack_t<__nv_bfloat16>(P, s, off); break;
    case Precision::FP16: unpack_t<__half>(P, s, off); break;
  }
}

void tracer_stats(EngineImpl &P, const void *s, double off, double out[4]) {
  if (!P.stats_d) P.stats_d = P.dalloc<double>(5 * kStatBlocks + 1);
  const int L = P.mesh.nl - 1;
  const long long N = P.mesh.nod2D;
  switch (P.prec) {
    case Precision::FP32:
      k_stats<float><<<kStatBlocks, kStatThreads, 0, P.stream>>>((const float *)s, nlev_dev(P), L, P.S, N, off, P.stats_d);
      break;
    case Precision::BF16:
      k_stats<__nv_bfloat16><<<kStatBlocks, kStatThreads, 0, P.stream>>>((const __nv_bfloat16 *)s, nlev_dev(P), L, P.S,
                                                                        N, off, P.stats_d);
      break;
    case Precision::FP16:
      k_stats<__half><<<kStatBlocks, kStatThreads, 0, P.stream>>>((const __half *)s, nlev_dev(P), L, P.S, N, off,
                                                                 P.stats_d);
      break;
    default:
      k_stats<double><<<kStatBlocks, kStatThreads, 0, P.stream>>>((const double *)s, nlev_dev(P), L, P.S, N, off,
                                                                 P.stats_d);
      break;
  }
  CK(cudaGetLastError());
  // the first cell as the host reads it: a NaN there makes min and max NaN,
  // like a host loop seeded with the first value
  std::vector<double> h(5 * kStatBlocks);
  P.d2h(h.data(), P.stats_d, h.size() * sizeof(double));
  double first = 0.0;
  if (L > 0 && N > 0) {
    double raw = 0.0;
    switch (P.prec) {
      case Precision::FP32: { float f; P.d2h(&f, s, 4); raw = f; break; }
      case Precision::BF16: { __nv_bfloat16 b; P.d2h(&b, s, 2); raw = (double)__bfloat162float(b); break; }
      case Precision::FP16: { __half b; P.d2h(&b, s, 2); raw = (double)__half2float(b); break; }
      default: P.d2h(&raw, s, 8); break;
    }
    first = (P.mesh.nlev_node[0] - 1 > 0) ? raw + off : raw;
  }
  double mn = INFINITY, mx = -INFINITY, nan = 0.0, sm = 0.0, c = 0.0;
  for (int b = 0; b < kStatBlocks; b++) {
    mn = std::fmin(mn, h[5 * b]);
    mx = std::fmax(mx, h[5 * b + 1]);
    nan += h[5 * b + 2];
    const double x = h[5 * b + 3], t = sm + x;
    c += (std::fabs(sm) >= std::fabs(x)) ? (sm - t) + x : (x - t) + sm;
    sm = t;
    c += h[5 * b + 4];
  }
  if (first != first || (L > 0 && N > 0 && nan == (double)L * N)) mn = mx = first;
  out[0] = (L > 0 && N > 0) ? mn : 0.0;
  out[1] = (L > 0 && N > 0) ? mx : 0.0;
  out[2] = sm + c;
  out[3] = nan;
}

bool host_range_pinned(const void *p, size_t bytes) { return range_pinned(p, bytes); }

void pack_from(EngineImpl &P, const double *src, cudaStream_t st, void *d0, void *d1, void *d2) {
  const int L = P.mesh.nl - 1;
  const long long N = P.mesh.nod2D;
  if (P.prec == Precision::FP64)
    k_pack<double><<<kGrid, kBlock, 0, st>>>(src, nlev_dev(P), L, P.S, N, 0.0, (double *)d0, (double *)d1, (double *)d2);
  else
    k_pack<float><<<kGrid, kBlock, 0, st>>>(src, nlev_dev(P), L, P.S, N, 0.0, (float *)d0, (float *)d1, (float *)d2);
  CK(cudaGetLastError());
}

void unpack_to(EngineImpl &P, const void *s, double *dst, cudaStream_t st) {
  const int L = P.mesh.nl - 1;
  const long long N = P.mesh.nod2D;
  if (P.prec == Precision::FP64)
    k_unpack<double><<<kGrid, kBlock, 0, st>>>((const double *)s, nlev_dev(P), L, P.S, N, 0.0, dst);
  else
    k_unpack<float><<<kGrid, kBlock, 0, st>>>((const float *)s, nlev_dev(P), L, P.S, N, 0.0, dst);
  CK(cudaGetLastError());
}

void storage_reoffset(EngineImpl &P, void *s, double off_old, double off_new) {
  if (P.prec == Precision::BF16) reoffset_t<__nv_bfloat16>(P, s, off_old, off_new);
  else if (P.prec == Precision::FP16) reoffset_t<__half>(P, s, off_old, off_new);
}

void release_ring(EngineImpl &P) {
  for (int s = 0; s < EngineImpl::kRing; s++) {
    if (P.ring_ev[s]) cudaEventDestroy(P.ring_ev[s]);
    if (P.ring[s]) cudaFreeHost(P.ring[s]);
    P.ring_ev[s] = nullptr;
    P.ring[s] = nullptr;
  }
}

}  // namespace fesom
