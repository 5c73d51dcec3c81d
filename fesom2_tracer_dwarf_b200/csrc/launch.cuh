// Templated dispatch of the step kernels for one (compute, storage) type
// pair; included by exactly one translation unit per pair.
#pragma once
#include <mutex>
#include <unordered_map>

// engine_impl.hpp first: its declarations name the non-variant FusedArgs
#include "engine_impl.hpp"
#include "advect_fused.cuh"
#include "tile.cuh"

namespace fesom {
FESOM_VARIANT_BEGIN

template <typename R>
const DMeshT<R> &dmesh(const EngineImpl &P);
template <>
inline const DMeshT<double> &dmesh<double>(const EngineImpl &P) { return P.dm64; }
template <>
inline const DMeshT<float> &dmesh<float>(const EngineImpl &P) { return P.dm32; }

// Raise the dynamic shared-memory limit of a kernel once (per kernel
// function; all kernels share one C++ function-pointer type).
template <typename K>
void set_smem(K kernel, size_t bytes) {
  static std::mutex mu;
  static std::unordered_map<const void *, size_t> done;
  std::lock_guard<std::mutex> lock(mu);
  auto it = done.find((const void *)kernel);
  if (it != done.end() && it->second >= bytes) return;
  CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  done[(const void *)kernel] = bytes;
}

template <typename R, typename TS, int NT, int HOR, int LIM>
void launch_edge(EngineImpl &P, const FusedArgs<R, TS> &a) {
  const DMeshT<R> &m = dmesh<R>(P);
  if (m.edge_sched.nblk <= 0) return;
  P.mark_begin(KK_EDGE);
  k_edge<R, TS, NT, HOR, LIM><<<m.edge_sched.nblk, kThreads, smem_edge(), P.stream>>>(m, a);
  P.mark_end();
}

template <typename R, typename TS, int NT, int VER, int LIM>
void launch_col1(EngineImpl &P, const FusedArgs<R, TS> &a) {
  const DMeshT<R> &m = dmesh<R>(P);
  const size_t sm = StageIncidence<R>::col1 ? smem_col_staged<R>(NT, 2) : smem_col<R>(NT, 2);
  set_smem(k_col1<R, TS, NT, VER, LIM>, sm);
  P.mark_begin(KK_COL1);
  k_col1<R, TS, NT, VER, LIM><<<m.node_sched.nblk, kThreads, sm, P.stream>>>(m, a);
  P.mark_end();
}

template <typename R, typename TS, int NT>
void launch_grad(EngineImpl &P, const FusedArgs<R, TS> &a) {
  const DMeshT<R> &m = dmesh<R>(P);
  if (m.grad_sched.nblk <= 0) return;
  P.mark_begin(KK_GRAD);
  k_grad<R, TS, NT><<<m.grad_sched.nblk, kThreads, smem_edge(), P.stream>>>(m, a);
  P.mark_end();
}

template <typename R, typename TS, int NT, int LIM>
void run_group(EngineImpl &P, const TracerScheme &sc, const FusedArgs<R, TS> &a) {
  if (sc.hor != 0) launch_grad<R, TS, NT>(P, a);
  switch (sc.hor) {
    case 1: launch_edge<R, TS, NT, HOR_MUSCL, LIM>(P, a); break;
    case 2: launch_edge<R, TS, NT, HOR_MFCT, LIM>(P, a); break;
    default: launch_edge<R, TS, NT, HOR_UPW1, LIM>(P, a); break;
  }
  if constexpr (std::is_same<R, float>::value && std::is_same<TS, float>::value) {
    if (a.feat[0] && sc.hor == 1) learned_correct_f32(P, NT, a);
  }
  switch (sc.ver) {
    case 1: launch_col1<R, TS, NT, VER_PPM, LIM>(P, a); break;
    case 2: launch_col1<R, TS, NT, VER_QR4C, LIM>(P, a); break;
    case 3: launch_col1<R, TS, NT, VER_CDIFF, LIM>(P, a); break;
    default: launch_col1<R, TS, NT, VER_UPW1, LIM>(P, a); break;
  }
  const DMeshT<R> &m = dmesh<R>(P);
  if (LIM == LIM_FCT) {
    const size_t sm2 = StageIncidence<R>::col2 ? smem_col_staged<R>(NT, 2) : smem_col<R>(NT, 2);
    set_smem(k_col2<R, TS, NT>, sm2);
    P.mark_begin(KK_COL2);
    k_col2<R, TS, NT><<<m.node_sched.nblk, kThreads, sm2, P.stream>>>(m, a);
    P.mark_end();
  }
  const size_t sm3 = StageIncidence<R>::col3 ? smem_col_staged<R>(NT, 0) : smem_col<R>(NT, 0);
  set_smem(k_col3<R, TS, NT, LIM>, sm3);
  P.mark_begin(KK_COL3);
  k_col3<R, TS, NT, LIM><<<m.node_sched.nblk, kThreads, sm3, P.stream>>>(m, a);
  P.mark_end();
}

// Geometry reciprocals of k_col3 (k_rcp_planes), once per mesh.
template <typename R>
void build_rcp_planes_t(EngineImpl &P, DMeshT<R> &d) {
  const size_t plane = (size_t)d.S * d.N;
  R *rcp = (R *)P.dalloc_bytes(2 * plane * sizeof(R));
  const int grid = (int)std::min<size_t>((plane + 255) / 256, (size_t)148 * 32);
  k_rcp_planes<R><<<std::max(grid, 1), 256, 0, P.stream>>>(d, rcp);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(P.stream));
  d.rcp = rcp;
  d.rcp_plane = plane;
}

// Edge volume fluxes of every edge level (the values k_edge computes and
// stores), for the fused kernel, which reads them.
template <typename R>
__global__ void __launch_bounds__(256) k_vflux(DMeshT<R> m, const R *vel, R *vflux) {
  const size_t n = (size_t)m.E * m.S;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const int s = (int)(q / m.S), k = (int)(q - (size_t)s * m.S);
    if (k >= m.edge_lev[s].y) continue;
    vflux[q] = edge_vflux(m, edge_ctx(m, s), vel, k);
  }
}

template <typename R, int LIM, bool AB>
void launch_tile(EngineImpl &P, const TileArgs<R> &a, const TileLayout &L) {
  set_smem(k_tile<R, LIM, AB>, L.bytes);
  k_tile<R, LIM, AB><<<P.tiles.np, kTileThreads, L.bytes, P.stream>>>(dmesh<R>(P), a, P.tiles, L);
}

// One batch through the fused patch kernel: the edge volume fluxes first
// when the batch does not find them stored, then one launch per tracer.
template <typename R>
void run_tiles(EngineImpl &P, const TracerScheme &sc, int nt, const BatchPtrs &b, double dt) {
  const DMeshT<R> &m = dmesh<R>(P);
  if (b.vflux_mode != 2) {
    const size_t n = (size_t)m.E * m.S;
    const int grid = (int)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, (size_t)148 * 16));
    P.mark_begin(KK_VFLUX);
    k_vflux<R><<<grid, 256, 0, P.stream>>>(m, (const R *)P.vel, (R *)b.vflux);
    P.mark_end();
  }
  for (int t = 0; t < nt; t++) {
    TileArgs<R> a{};
    a.T = (const R *)b.T[t];
    a.TAB = (const R *)b.TAB[t];
    a.T_out = (R *)b.T_out[t];
    a.vflux = (const R *)b.vflux;
    a.W = (const R *)P.W;
    a.dt = (R)dt;
    a.ph = (R)sc.ph;
    a.hor = sc.hor;
    a.ver = sc.ver;
    a.nonfinite = P.nonfinite_d;
    const bool ab = b.TAB[t] == b.T[t];
    const TileLayout L = tile_layout(P.tplan, (unsigned)sizeof(R), ab, sc.hor != 0, sc.lim == 1);
    P.mark_begin(KK_TILE);
    if (sc.lim == 1) ab ? launch_tile<R, LIM_FCT, true>(P, a, L) : launch_tile<R, LIM_FCT, false>(P, a, L);
    else ab ? launch_tile<R, LIM_NONE, true>(P, a, L) : launch_tile<R, LIM_NONE, false>(P, a, L);
    P.mark_end();
  }
}

template <typename R, typename TS>
void launch_batch_t(EngineImpl &P, const TracerScheme &sc, int nt, const BatchPtrs &b, double dt) {
  if constexpr (std::is_same<R, TS>::value) {
    if (fused_step(P, sc, b.feat[0] != nullptr)) {
      run_tiles<R>(P, sc, nt, b, dt);
      return;
    }
  }
  FusedArgs<R, TS> a{};
  for (int t = 0; t < nt; t++) {
    a.T[t] = (const TS *)b.T[t];
    a.TAB[t] = (const TS *)b.TAB[t];
    a.T_out[t] = (TS *)b.T_out[t];
    a.adf_h[t] = (R *)b.adf_h[t];
    a.adf_v[t] = (R *)b.adf_v[t];
    a.lo[t] = (R *)b.lo[t];
    a.rpm[t] = (R *)b.rpm[t];
    a.gradn[t] = (R *)b.gradn[t];
    a.feat[t] = (__nv_bfloat16 *)b.feat[t];
    a.fscale[t] = (float *)b.fscale[t];
  }
  a.vflux = (R *)b.vflux;
  a.vel = (const R *)P.vel;
  a.W = (const R *)P.W;
  a.dt = (R)dt;
  a.ph = (R)sc.ph;
  a.pv = (R)sc.pv;
  for (int t = 0; t < nt; t++) {
    a.off[t] = (R)b.off[t];
    a.seed[t] = b.seed[t];
  }
  a.sround = b.sround;
  a.vflux_mode = b.vflux_mode;
  a.nonfinite = P.nonfinite_d;
  const bool fct = sc.lim == 1;
  if (nt == 4) fct ? run_group<R, TS, 4, LIM_FCT>(P, sc, a) : run_group<R, TS, 4, LIM_NONE>(P, sc, a);
  else if (nt == 2) fct ? run_group<R, TS, 2, LIM_FCT>(P, sc, a) : run_group<R, TS, 2, LIM_NONE>(P, sc, a);
  else fct ? run_group<R, TS, 1, LIM_FCT>(P, sc, a) : run_group<R, TS, 1, LIM_NONE>(P, sc, a);
}

// ---------------------------------------------------------------------------
// compensated FP64 sums over the wet cells of one tracer
// ---------------------------------------------------------------------------
__device__ __forceinline__ void two_sum(double a, double b, double &s, double &e) {
  s = a + b;
  const double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}

template <typename R, typename TS>
__global__ void __launch_bounds__(256) k_volume_sum(DMeshT<R> m, const TS *T, double off, double *out) {
  // per thread: Neumaier-compensated partial sums of T and T*areasvol*hnode_new
  double s0 = 0, c0 = 0, s1 = 0, c1 = 0;
  for (int n = blockIdx.x * blockDim.y + threadIdx.y; n < m.N; n += gridDim.x * blockDim.y) {
    const int L = m.nlev_node[n] - 1;
    for (int k = threadIdx.x; k < L; k += blockDim.x) {
      const size_t o = (size_t)n * m.S + k;
      const double t = std::is_same<R, TS>::value ? (double)R(T[o]) : (double)R(T[o]) + off;
      const double v = t * (double)m.areasvol[o] * (double)m.hnode_new[o];
      double s, e;
      two_sum(s0, t, s, e); s0 = s; c0 += e;
      two_sum(s1, v, s, e); s1 = s; c1 += e;
    }
  }
  __shared__ double sh[4][256];
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  sh[0][tid] = s0; sh[1][tid] = c0; sh[2][tid] = s1; sh[3][tid] = c1;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (tid < w) {
      double s, e;
      two_sum(sh[0][tid], sh[0][tid + w], s, e);
      sh[0][tid] = s; sh[1][tid] += sh[1][tid + w] + e;
      two_sum(sh[2][tid], sh[2][tid + w], s, e);
      sh[2][tid] = s; sh[3][tid] += sh[3][tid + w] + e;
    }
    __syncthreads();
  }
  if (tid == 0) {
    out[4 * blockIdx.x + 0] = sh[0][0];
    out[4 * blockIdx.x + 1] = sh[1][0];
    out[4 * blockIdx.x + 2] = sh[2][0];
    out[4 * blockIdx.x + 3] = sh[3][0];
  }
}

template <typename R, typename TS>
void volume_sum_t(EngineImpl &P, const void *T, double off, double res[2]) {
  const int blocks = 296;
  double *d = P.dalloc<double>(4 * blocks);
  k_volume_sum<R, TS><<<blocks, dim3(32, 8), 0, P.stream>>>(dmesh<R>(P), (const TS *)T, off, d);
  CK(cudaGetLastError());
  std::vector<double> h(4 * blocks);
  P.d2h(h.data(), d, h.size() * sizeof(double));
  P.dfree(d);
  // final compensated combination on the host, in block order
  double s0 = 0, c0 = 0, s1 = 0, c1 = 0;
  for (int b = 0; b < blocks; b++) {
    for (int q = 0; q < 2; q++) {
      double &s = q ? s1 : s0, &c = q ? c1 : c0;
      const double x = h[4 * b + 2 * q], xc = h[4 * b + 2 * q + 1];
      const double t = s + x;
      c += (std::fabs(s) >= std::fabs(x)) ? (s - t) + x : (x - t) + s;
      s = t;
      c += xc;
    }
  }
  res[0] = s0 + c0;
  res[1] = s1 + c1;
}

FESOM_VARIANT_END
}  // namespace fesom
