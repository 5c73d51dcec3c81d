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

#include <cstdint>
#include <type_traits>

#include "dmesh.hpp"

// The FP64 kernels are compiled twice: without FMA contraction (bit-identical
// to the reference's arithmetic) and, in a translation unit that defines
// FESOM_KERNEL_VARIANT, with it (step_f64fma.cu).  The variant's kernels and
// their launch templates live in an inline namespace of that name, so the two
// builds of the same templates do not collide at link time.
#ifndef FESOM_VARIANT_BEGIN
#ifdef FESOM_KERNEL_VARIANT
#define FESOM_VARIANT_BEGIN inline namespace FESOM_KERNEL_VARIANT {
#define FESOM_VARIANT_END }
#else
#define FESOM_VARIANT_BEGIN
#define FESOM_VARIANT_END
#endif
#endif

namespace fesom {
FESOM_VARIANT_BEGIN

// Fortran MAX/MIN as evaluated by the oracle: the first argument wins ties.
template <typename R> __device__ __forceinline__ R fmax2(R a, R b) { return (b > a) ? b : a; }
template <typename R> __device__ __forceinline__ R fmin2(R a, R b) { return (b < a) ? b : a; }
template <typename R> __device__ __forceinline__ R fmax3(R a, R b, R c) { return fmax2(fmax2(a, b), c); }
template <typename R> __device__ __forceinline__ R fmin3(R a, R b, R c) { return fmin2(fmin2(a, b), c); }
__device__ __forceinline__ double sgn1(double w) { return copysign(1.0, w); }
__device__ __forceinline__ float sgn1(float w) { return copysignf(1.0f, w); }

// Cell index within a (S, N) or (S, E) array: 32-bit unsigned, so that
// address arithmetic stays one multiply-add (the engine refuses meshes with
// E x S or N x S of 2^32 cells or more).
using cix = unsigned;

// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// tracer storage.  FP64 and FP32 storage hold the tracer T itself; 16-bit
// storage holds the anomaly T - off on wet cells, with off a per-tracer FP32
// constant near the field's mean, so that the storage ulp follows the
// anomaly's magnitude.  Arithmetic is always in R.
// ---------------------------------------------------------------------------
template <typename R, typename TS, typename I>
__device__ __forceinline__ R ldT(const TS *p, I i, R off) {
  if constexpr (std::is_same<R, TS>::value) {
    (void)off;
    return p[i];
  } else {
    return R(p[i]) + off;
  }
}

// 32-bit integer hash (Wellons' "lowbias32" finalizer, a published
// xorshift-multiply mix); used as a counter-based random stream.
__device__ __forceinline__ uint32_t mix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

// Stochastic rounding of an FP32 value to BF16: add 16 random bits below the
// kept mantissa and truncate, so the value rounds up with probability equal
// to its distance from the lower neighbour over the spacing (Connolly, Higham
// & Mary 2021).  Inf and NaN pass through unchanged.
__device__ __forceinline__ __nv_bfloat16 bf16_sround(float x, uint32_t r) {
  uint32_t u = __float_as_uint(x);
  if ((u & 0x7f800000u) != 0x7f800000u) u += (r & 0xffffu);
  return __ushort_as_bfloat16((unsigned short)(u >> 16));
}

// Stochastic rounding of an FP32 value to FP16: round toward zero, then step
// one FP16 ulp away from zero with probability (remainder / spacing).
__device__ __forceinline__ __half f16_sround(float x, uint32_t r) {
  const __half lo = __float2half_rz(x);
  const float flo = __half2float(lo);
  const float rem = fabsf(x - flo);                 // exact: x - (x cut to 11 bits)
  if (!(rem > 0.0f)) return (x == x) ? lo : __float2half_rn(x);
  const __half hi = __ushort_as_half((unsigned short)(__half_as_ushort(lo) + 1));  // next magnitude
  const float gap = fabsf(__half2float(hi) - flo);  // a power of two (or inf past the range)
  const float u = (float)(r >> 8) * 0x1p-24f;       // [0, 1)
  return (u * gap < rem) ? hi : lo;
}

// Store of a new tracer value: identity for FP64/FP32 storage; for 16-bit
// storage the anomaly v - off rounded to nearest or stochastically with the
// random word r.
template <typename R, typename TS>
__device__ __forceinline__ TS stT(R v, R off, bool sround, uint32_t r) {
  if constexpr (std::is_same<R, TS>::value) {
    (void)off; (void)sround; (void)r;
    return v;
  } else if constexpr (std::is_same<TS, __nv_bfloat16>::value) {
    const float x = float(v - off);
    return sround ? bf16_sround(x, r) : __float2bfloat16_rn(x);
  } else {
    const float x = float(v - off);
    return sround ? f16_sround(x, r) : __float2half_rn(x);
  }
}

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
  R off;        // storage offset (16-bit storage only)
};

// adv_tra_ver_upw1 (lib/oce_adv_tra_ver.F90:300-327)
template <typename R, typename TS>
__device__ __forceinline__ R ver_upw1(const Col<R, TS> &c, int i) {
  if (i == 1) return -(c.W[0] * ldT(c.T, 0, c.off) * c.A[0]);
  if (i == c.nlev) return R(0);
  const R w = c.W[i - 1];
  return -(R(0.5) * (ldT(c.T, i - 1, c.off) * (w + fabs(w)) + ldT(c.T, i - 2, c.off) * (w - fabs(w))) * c.A[i - 1]);
}

// QR4C (lib/oce_adv_tra_ver.F90:397-436): the reference's assignments replayed
// in order for interface i, starting from the previous flux value v.
template <typename R, typename TS>
__device__ __forceinline__ R ver_qr4c(const Col<R, TS> &c, const R *zbar, const R *Z, int i, R num_ord, R v) {
  auto T = [&](int q) { return ldT(c.T, q - 1, c.off); };  // 1-based views
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
  if (i == 1) return -(c.W[0] * ldT(c.T, 0, c.off) * c.A[0]) - v;
  const R tv = R(0.5) * (ldT(c.T, i - 2, c.off) + ldT(c.T, i - 1, c.off));
  return -(tv * c.W[i - 1] * c.A[i - 1]) - v;
}

FESOM_VARIANT_END
}  // namespace fesom
