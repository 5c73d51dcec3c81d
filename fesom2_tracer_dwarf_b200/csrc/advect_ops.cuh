// Per-cell operators of the tracer advection step, shared by every kernel.
//
// Each function evaluates one reference expression for one (column, level)
// with the reference's operand order, so that FP64 builds without FMA
// contraction (nvcc --fmad=false) reproduce the Fortran arithmetic bit for
// bit.  Levels are 0-based here (k = nz - 1); "nz" names the Fortran 1-based
// level where a formula depends on it.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "dmesh.hpp"

namespace fesom {

// Fortran MAX/MIN as evaluated by the oracle: the first argument wins ties.
template <typename R> __device__ __forceinline__ R fmax2(R a, R b) { return (b > a) ? b : a; }
template <typename R> __device__ __forceinline__ R fmin2(R a, R b) { return (b < a) ? b : a; }
template <typename R> __device__ __forceinline__ R fmax3(R a, R b, R c) { return fmax2(fmax2(a, b), c); }
template <typename R> __device__ __forceinline__ R fmin3(R a, R b, R c) { return fmin2(fmin2(a, b), c); }
__device__ __forceinline__ double sgn1(double w) { return copysign(1.0, w); }
__device__ __forceinline__ float sgn1(float w) { return copysignf(1.0f, w); }

enum HorScheme { HOR_UPW1 = 0, HOR_MUSCL = 1, HOR_MFCT = 2 };
enum VerScheme { VER_UPW1 = 0, VER_PPM = 1, VER_QR4C = 2, VER_CDIFF = 3 };
enum Limiter { LIM_NONE = 0, LIM_FCT = 1 };

constexpr double kREarthD = 6367500.0;

// ---------------------------------------------------------------------------
// horizontal edge fluxes (lib/oce_adv_tra_hor.F90)
// ---------------------------------------------------------------------------
template <typename R>
struct EdgeCtx {
  int e, n1, n2, el1, el2, shared, levels;
  R dX1, dY1, dX2, dY2;
};

template <typename R>
__device__ __forceinline__ EdgeCtx<R> edge_ctx(const DMeshT<R> &m, int e) {
  EdgeCtx<R> c;
  c.e = e;
  int2 nn = m.edge_nodes[e], tt = m.edge_tri[e], lv = m.edge_lev[e];
  c.n1 = nn.x; c.n2 = nn.y; c.el1 = tt.x; c.el2 = tt.y; c.shared = lv.x; c.levels = lv.y;
  c.dX1 = m.edge_cross[4 * e + 0]; c.dY1 = m.edge_cross[4 * e + 1];
  c.dX2 = m.edge_cross[4 * e + 2]; c.dY2 = m.edge_cross[4 * e + 3];
  return c;
}

// Volume flux through the edge's dual segments at level k: both segments on
// the shared levels (segment C), otherwise the one element that reaches that
// deep (segments D, E) -- lib/oce_adv_tra_hor.F90:171-253 with ulevels = 1.
template <typename R>
__device__ __forceinline__ R edge_vflux(const DMeshT<R> &m, const EdgeCtx<R> &c, const R *vel, int k) {
  const int nz = k + 1;
  const int S = m.S;
  if (nz <= c.shared) {
    const R u1 = vel[2 * ((size_t)c.el1 * S + k)], v1 = vel[2 * ((size_t)c.el1 * S + k) + 1];
    const R u2 = vel[2 * ((size_t)c.el2 * S + k)], v2 = vel[2 * ((size_t)c.el2 * S + k) + 1];
    return (-v1 * c.dX1 + u1 * c.dY1) * m.helem[(size_t)c.el1 * S + k] +
           (v2 * c.dX2 - u2 * c.dY2) * m.helem[(size_t)c.el2 * S + k];
  }
  const int nl1 = m.nlev_elem[c.el1] - 1;
  if (nz <= nl1) {
    const R u1 = vel[2 * ((size_t)c.el1 * S + k)], v1 = vel[2 * ((size_t)c.el1 * S + k) + 1];
    return (-v1 * c.dX1 + u1 * c.dY1) * m.helem[(size_t)c.el1 * S + k];
  }
  const R u2 = vel[2 * ((size_t)c.el2 * S + k)], v2 = vel[2 * ((size_t)c.el2 * S + k) + 1];
  return (v2 * c.dX2 - u2 * c.dY2) * m.helem[(size_t)c.el2 * S + k];
}

// first-order upwind edge flux, lib/oce_adv_tra_hor.F90:178-181
template <typename R>
__device__ __forceinline__ R upw1_flux(R vflux, R t1, R t2) {
  return R(-0.5) * (t1 * (vflux + fabs(vflux)) + t2 * (vflux - fabs(vflux)));
}

// ---------------------------------------------------------------------------
// vertical fluxes at interfaces (lib/oce_adv_tra_ver.F90); "i" is the
// 1-based interface index, interface i is the top of layer i; nlev is
// nlevels_nod2D of the column (bottom interface).
// ---------------------------------------------------------------------------
template <typename R, typename TS = R>
struct Col {
  const TS *T;  // tracer column (layers), storage type TS
  const R *W;   // vertical velocity column (interfaces)
  const R *A;   // area column (interfaces)
  const R *HN;  // hnode_new column
  const R *H;   // hnode column
  int nlev;
};

// adv_tra_ver_upw1 (lib/oce_adv_tra_ver.F90:300-327)
template <typename R, typename TS>
__device__ __forceinline__ R ver_upw1(const Col<R, TS> &c, int i) {
  if (i == 1) return -(c.W[0] * R(c.T[0]) * c.A[0]);
  if (i == c.nlev) return R(0);
  const R w = c.W[i - 1];
  return -(R(0.5) * (R(c.T[i - 1]) * (w + fabs(w)) + R(c.T[i - 2]) * (w - fabs(w))) * c.A[i - 1]);
}

// QR4C (lib/oce_adv_tra_ver.F90:397-436): the reference's assignments replayed
// in order for interface i, starting from the previous flux value v.
template <typename R, typename TS>
__device__ __forceinline__ R ver_qr4c(const Col<R, TS> &c, const R *zbar, const R *Z, int i, R num_ord, R v) {
  auto T = [&](int q) { return R(c.T[q - 1]); };  // 1-based views
  const R *W = c.W - 1;
  const R *A = c.A - 1;
  const int nzmin = 1, nzmax = c.nlev;
  if (i == nzmin) v = -(T(i) * W[i] * A[i]) - v;
  if (i == nzmin + 1) v = -(R(0.5) * (T(i - 1) + T(i)) * W[i] * A[i]) - v;
  if (i == nzmax - 1) v = -(R(0.5) * (T(i - 1) + T(i)) * W[i] * A[i]) - v;
  if (i == nzmax) v = R(0) - v;
  if (i >= nzmin + 2 && i <= nzmax - 2) {
    const R *Zc = Z - 1;
    const R *ZB = zbar - 1;
    const R qc = (T(i - 1) - T(i)) / (Zc[i - 1] - Zc[i]);
    const R qu = (T(i) - T(i + 1)) / (Zc[i] - Zc[i + 1]);
    const R qd = (T(i - 2) - T(i - 1)) / (Zc[i - 2] - Zc[i - 1]);
    const R Tmean1 = T(i) + (R(2) * qc + qu) * (ZB[i] - Zc[i]) / R(3);
    const R Tmean2 = T(i - 1) + (R(2) * qc + qd) * (ZB[i] - Zc[i - 1]) / R(3);
    const R Tmean = (W[i] + fabs(W[i])) * Tmean1 + (W[i] - fabs(W[i])) * Tmean2;
    v = (-(R(0.5) * (R(1) - num_ord) * Tmean) - num_ord * (R(0.5) * (Tmean1 + Tmean2)) * W[i]) * A[i] - v;
  }
  return v;
}

// CDIFF (lib/oce_adv_tra_ver.F90:679-704): interfaces 1..nlev-1 are written,
// the bottom interface keeps its previous value v.
template <typename R, typename TS>
__device__ __forceinline__ R ver_cdiff(const Col<R, TS> &c, int i, R v) {
  if (i == c.nlev) return v;
  if (i == 1) return -(c.W[0] * R(c.T[0]) * c.A[0]) - v;
  const R tv = R(0.5) * (R(c.T[i - 2]) + R(c.T[i - 1]));
  return -(tv * c.W[i - 1] * c.A[i - 1]) - v;
}

}  // namespace fesom
