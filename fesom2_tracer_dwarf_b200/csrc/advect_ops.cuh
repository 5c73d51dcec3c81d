// Per-cell operators of the tracer advection step, shared by every kernel.
//
// Each function evaluates one reference expression for one (column, level)
// with the reference's operand order, so that FP64 builds without FMA
// contraction (nvcc --fmad=false) reproduce the Fortran arithmetic bit for
// bit.  Levels are 0-based here (k = nz - 1); "nz" names the Fortran 1-based
// level where a formula depends on it.
#pragma once
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
// cell schedules
// ---------------------------------------------------------------------------
__device__ __forceinline__ int find_item(const int *s_off, int nitems, int c) {
  int lo = 0, hi = nitems;
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (s_off[mid] <= c) lo = mid; else hi = mid;
  }
  return lo;
}

// Calls f(item, level) for every wet cell of this block's items.
template <class F>
__device__ __forceinline__ void for_each_cell(const DSched &sc, int *s_off, F &&f) {
  const int i0 = sc.blk[blockIdx.x], i1 = sc.blk[blockIdx.x + 1], ni = i1 - i0;
  for (int t = threadIdx.x; t <= ni; t += blockDim.x) s_off[t] = sc.cell_off[i0 + t];
  __syncthreads();
  const int c0 = s_off[0], c1 = s_off[ni];
  for (int c = c0 + (int)threadIdx.x; c < c1; c += blockDim.x) {
    int j = find_item(s_off, ni, c);
    f(i0 + j, c - s_off[j]);
  }
}

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

// element tracer gradient: sum(gradient_sca(1:3)*T), sum(gradient_sca(4:6)*T)
template <typename R>
__device__ __forceinline__ void tr_xy(const DMeshT<R> &m, const R *tab, int elem, int k, R &gx, R &gy) {
  const int *en = m.elem_nodes + 3 * elem;
  const R *gs = m.grad_sca + 6 * elem;
  const R t1 = tab[(size_t)en[0] * m.S + k], t2 = tab[(size_t)en[1] * m.S + k], t3 = tab[(size_t)en[2] * m.S + k];
  gx = (gs[0] * t1 + gs[1] * t2) + gs[2] * t3;
  gy = (gs[3] * t1 + gs[4] * t2) + gs[5] * t3;
}

// area-weighted ring mean of tr_xy (lib/oce_muscl_adv.F90:394-409)
template <typename R>
__device__ __forceinline__ void ring_mean(const DMeshT<R> &m, const R *tab, int n, int k, R &gx, R &gy) {
  R tvol = R(0), tx = R(0), ty = R(0);
  const int nz = k + 1;
  for (int p = m.ring_ptr[n]; p < m.ring_ptr[n + 1]; p++) {
    const int el = m.ring_elem[p];
    if (m.nlev_elem[el] - 1 < nz) continue;
    R ax, ay;
    tr_xy(m, tab, el, k, ax, ay);
    const R a = m.elem_area[el];
    tvol = tvol + a;
    tx = tx + ax * a;
    ty = ty + ay * a;
  }
  gx = tx / tvol;
  gy = ty / tvol;
}

// edge_up_dn_grad(1:4, nz, edge) of fill_up_dn_grad (lib/oce_muscl_adv.F90:383-527)
template <typename R>
__device__ __forceinline__ void up_dn_grad(const DMeshT<R> &m, const EdgeCtx<R> &c, const R *tab, int k, R g[4]) {
  const int2 ud = m.up_dn[c.e];
  bool shared = false;
  if (ud.x >= 0 && ud.y >= 0) {
    const int nzmax = min(m.nlev_node_min[c.n1], m.nlev_node_min[c.n2]);
    shared = (k + 1) <= nzmax - 1;
  }
  if (shared) {
    tr_xy(m, tab, ud.x, k, g[0], g[2]);
    tr_xy(m, tab, ud.y, k, g[1], g[3]);
  } else {
    ring_mean(m, tab, c.n1, k, g[0], g[2]);
    ring_mean(m, tab, c.n2, k, g[1], g[3]);
  }
}

// MUSCL / MFCT high-order edge flux (lib/oce_adv_tra_hor.F90:454-497)
template <typename R, int HOR>
__device__ __forceinline__ R muscl_flux(const DMeshT<R> &m, const EdgeCtx<R> &c, const R *tab, R vflux, R num_ord, int k) {
  R g[4];
  up_dn_grad(m, c, tab, k, g);
  const R t1 = tab[(size_t)c.n1 * m.S + k], t2 = tab[(size_t)c.n2 * m.S + k];
  const R ex = m.edge_dxdy[2 * c.e], ey = m.edge_dxdy[2 * c.e + 1], a = m.edge_a[c.e];
  const R re = R(kREarthD);
  R Tmean1, Tmean2;
  if (HOR == HOR_MUSCL) {
    const int nz = k + 1;
    const R c_lo1 = (m.nbl[c.n1] - nz >= 0) ? R(1) : R(0);
    const R c_lo2 = (m.nbl[c.n2] - nz >= 0) ? R(1) : R(0);
    Tmean2 = t2 - (R(2) * (t2 - t1) + ex * a * g[1] + ey * re * g[3]) / R(6) * c_lo2;
    Tmean1 = t1 + (R(2) * (t2 - t1) + ex * a * g[0] + ey * re * g[2]) / R(6) * c_lo1;
  } else {
    Tmean2 = t2 - (R(2) * (t2 - t1) + ex * a * g[1] + ey * re * g[3]) / R(6);
    Tmean1 = t1 + (R(2) * (t2 - t1) + ex * a * g[0] + ey * re * g[2]) / R(6);
  }
  const R cHO = (vflux + fabs(vflux)) * Tmean1 + (vflux - fabs(vflux)) * Tmean2;
  return -(R(0.5) * (R(1) - num_ord) * cHO) - vflux * num_ord * R(0.5) * (Tmean1 + Tmean2);
}

// ---------------------------------------------------------------------------
// vertical fluxes at interfaces (lib/oce_adv_tra_ver.F90); "i" is the
// 1-based interface index, interface i is the top of layer i; nlev is
// nlevels_nod2D of the column (bottom interface).
// ---------------------------------------------------------------------------
template <typename R>
struct Col {
  const R *T;   // tracer column (layers)
  const R *W;   // vertical velocity column (interfaces)
  const R *A;   // area column (interfaces)
  const R *HN;  // hnode_new column
  const R *H;   // hnode column
  int nlev;
};

template <typename R>
__device__ __forceinline__ Col<R> column(const DMeshT<R> &m, const R *T, const R *W, int n) {
  Col<R> c;
  const size_t o = (size_t)n * m.S;
  c.T = T + o; c.W = W + o; c.A = m.area + o; c.HN = m.hnode_new + o; c.H = m.hnode + o;
  c.nlev = m.nlev_node[n];
  return c;
}

// adv_tra_ver_upw1 (lib/oce_adv_tra_ver.F90:300-327)
template <typename R>
__device__ __forceinline__ R ver_upw1(const Col<R> &c, int i) {
  if (i == 1) return -(c.W[0] * c.T[0] * c.A[0]);
  if (i == c.nlev) return R(0);
  const R w = c.W[i - 1];
  return -(R(0.5) * (c.T[i - 1] * (w + fabs(w)) + c.T[i - 2] * (w - fabs(w))) * c.A[i - 1]);
}

// PPM interface value tv(i) (lib/oce_adv_tra_ver.F90:510-594)
template <typename R>
__device__ __forceinline__ R ppm_tv(const Col<R> &c, int i) {
  const R *T = c.T - 1;   // 1-based views
  const R *HN = c.HN - 1;
  const int nzmax = c.nlev;
  if (i == 1) return T[1];
  if (i == nzmax) return T[nzmax - 1];
  if (i == nzmax - 1) {
    const R s = sgn1(c.W[nzmax - 2]);
    return -T[nzmax - 2] * fmin2(s, R(0)) + T[nzmax - 1] * fmax2(s, R(0));
  }
  if (i == 2) return R(0.5) * (T[1] + T[2]);
  const int nz = i - 1;
  const R dzjm1 = HN[nz - 1], dzj = HN[nz], dzjp1 = HN[nz + 1], dzjp2 = HN[nz + 2];
  R deltaj = dzj / (dzjm1 + dzj + dzjp1) *
             ((R(2) * dzjm1 + dzj) / (dzjp1 + dzj) * (T[nz + 1] - T[nz]) +
              (dzj + R(2) * dzjp1) / (dzjm1 + dzj) * (T[nz] - T[nz - 1]));
  R deltajp1 = dzjp1 / (dzj + dzjp1 + dzjp2) *
               ((R(2) * dzj + dzjp1) / (dzjp2 + dzjp1) * (T[nz + 2] - T[nz + 1]) +
                (dzjp1 + R(2) * dzjp2) / (dzj + dzjp1) * (T[nz + 1] - T[nz]));
  if ((T[nz + 1] - T[nz]) * (T[nz] - T[nz - 1]) > R(0))
    deltaj = fmin3(fabs(deltaj), R(2) * fabs(T[nz + 1] - T[nz]), R(2) * fabs(T[nz] - T[nz - 1])) * sgn1(deltaj);
  else
    deltaj = R(0);
  if ((T[nz + 2] - T[nz + 1]) * (T[nz + 1] - T[nz]) > R(0))
    deltajp1 = fmin3(fabs(deltajp1), R(2) * fabs(T[nz + 2] - T[nz + 1]), R(2) * fabs(T[nz + 1] - T[nz])) * sgn1(deltajp1);
  else
    deltajp1 = R(0);
  return T[nz] + dzj / (dzj + dzjp1) * (T[nz + 1] - T[nz]) +
         R(1) / (dzjm1 + dzj + dzjp1 + dzjp2) *
             ((R(2) * dzjp1 * dzj) / (dzj + dzjp1) *
                  ((dzjm1 + dzj) / (R(2) * dzj + dzjp1) - (dzjp2 + dzjp1) / (R(2) * dzjp1 + dzj)) *
                  (T[nz + 1] - T[nz]) -
              dzj * (dzjm1 + dzj) / (R(2) * dzj + dzjp1) * deltajp1 +
              dzjp1 * (dzjp1 + dzjp2) / (dzj + R(2) * dzjp1) * deltaj);
}

// PPM flux through interface i (lib/oce_adv_tra_ver.F90:597-639).  The flux
// through an inner interface comes from the layer below it when W > 0 and
// from the layer above it when W < 0, each with that layer's monotonised
// parabola.
template <typename R>
__device__ __forceinline__ R ver_ppm(const Col<R> &c, int i, R dt) {
  const int nzmax = c.nlev;
  if (i == 1) return -(ppm_tv(c, 1) * c.W[0] * c.A[0]);
  if (i == nzmax) return R(0);
  const R w = c.W[i - 1];
  if (!(w > R(0)) && !(w < R(0))) return R(0);
  const int nz = (w > R(0)) ? i : i - 1;  // layer that supplies the flux
  const R Tc = c.T[nz - 1];
  R aL = ppm_tv(c, nz), aR = ppm_tv(c, nz + 1);
  if ((aR - Tc) * (Tc - aL) <= R(0)) { aL = Tc; aR = Tc; }
  if ((aR - aL) * (Tc - R(0.5) * (aL + aR)) > (aR - aL) * (aR - aL) / R(6)) aL = R(3) * Tc - R(2) * aR;
  if ((aR - aL) * (Tc - R(0.5) * (aR + aL)) < -((aR - aL) * (aR - aL) / R(6))) aR = R(3) * Tc - R(2) * aL;
  const R dzj = c.H[nz - 1];
  const R aj = R(6) * (Tc - R(0.5) * (aL + aR));
  const R two3 = R(2.0 / 3.0);
  if (w > R(0)) {
    const R x = fmin2(w * dt / dzj, R(1));
    const R t = (-aL - R(0.5) * x * (aR - aL + (R(1) - two3 * x) * aj));
    return t * c.A[i - 1] * w;
  }
  const R x = fmin2(-(w * dt / dzj), R(1));
  const R t = (-aR + R(0.5) * x * (aR - aL - (R(1) - two3 * x) * aj));
  return t * c.A[i - 1] * w;
}

// QR4C (lib/oce_adv_tra_ver.F90:397-436): the reference's assignments replayed
// in order for interface i, starting from the previous flux value v.
template <typename R>
__device__ __forceinline__ R ver_qr4c(const Col<R> &c, const R *zbar, const R *Z, int i, R num_ord, R v) {
  const R *T = c.T - 1;
  const R *W = c.W - 1;
  const R *A = c.A - 1;
  const int nzmin = 1, nzmax = c.nlev;
  if (i == nzmin) v = -(T[i] * W[i] * A[i]) - v;
  if (i == nzmin + 1) v = -(R(0.5) * (T[i - 1] + T[i]) * W[i] * A[i]) - v;
  if (i == nzmax - 1) v = -(R(0.5) * (T[i - 1] + T[i]) * W[i] * A[i]) - v;
  if (i == nzmax) v = R(0) - v;
  if (i >= nzmin + 2 && i <= nzmax - 2) {
    const R *Zc = Z - 1;
    const R *ZB = zbar - 1;
    const R qc = (T[i - 1] - T[i]) / (Zc[i - 1] - Zc[i]);
    const R qu = (T[i] - T[i + 1]) / (Zc[i] - Zc[i + 1]);
    const R qd = (T[i - 2] - T[i - 1]) / (Zc[i - 2] - Zc[i - 1]);
    const R Tmean1 = T[i] + (R(2) * qc + qu) * (ZB[i] - Zc[i]) / R(3);
    const R Tmean2 = T[i - 1] + (R(2) * qc + qd) * (ZB[i] - Zc[i - 1]) / R(3);
    const R Tmean = (W[i] + fabs(W[i])) * Tmean1 + (W[i] - fabs(W[i])) * Tmean2;
    v = (-(R(0.5) * (R(1) - num_ord) * Tmean) - num_ord * (R(0.5) * (Tmean1 + Tmean2)) * W[i]) * A[i] - v;
  }
  return v;
}

// CDIFF (lib/oce_adv_tra_ver.F90:679-704): interfaces 1..nlev-1 are written,
// the bottom interface keeps its previous value v.
template <typename R>
__device__ __forceinline__ R ver_cdiff(const Col<R> &c, int i, R v) {
  if (i == c.nlev) return v;
  if (i == 1) return -(c.W[0] * c.T[0] * c.A[0]) - v;
  const R tv = R(0.5) * (c.T[i - 2] + c.T[i - 1]);
  return -(tv * c.W[i - 1] * c.A[i - 1]) - v;
}

}  // namespace fesom
