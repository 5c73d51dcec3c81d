// Kernels of the tracer advection step (do_oce_adv_tra,
// lib/oce_adv_tra_driver.F90:23-294, with FCT from lib/oce_adv_tra_fct.F90).
//
// Every edge scatter of the reference is rewritten as a node-centric gather
// over the node's incident edges in ascending edge id, so each node sums its
// contributions in exactly the order of the reference's serial edge loop and
// no float atomics are used: results are deterministic and bit-reproducible.
//
// Step structure (per tracer, FCT on):
//   edge_flux  : per edge level, LO upwind flux on T and the antidiffusive
//                flux HO(T_AB) - LO (MUSCL/MFCT/UPW1)                [edge]
//   node_lo    : LO solution (horizontal gather + upwind vertical)   [node]
//   node_vert  : vertical antidiffusive flux HO(T_AB) - LO at the
//                column's interfaces (PPM/QR4C/CDIFF/UPW1)            [node]
//   node_bounds: a1-a3 cluster max/min of (LO, T)                     [node]
//   node_ratio : b1-b2 limiter ratios R+, R-                          [node]
//   node_apply : b3 limiting, flux2dtracer and T += del/h_new         [node]
// The two global dependencies (LO before the bounds, R+- before limiting)
// fall on kernel boundaries.
#pragma once
#include "advect_ops.cuh"

namespace fesom {

template <typename R>
struct StepArgs {
  const R *T;       // tracer at step n (values)
  const R *TAB;     // tracer used for the high-order fluxes (valuesAB)
  const R *vel;     // (2, S, elem)
  const R *W;       // (S, node), interfaces
  R dt, ph, pv;
  R *flo;           // (S, edge) LO horizontal flux
  R *adf_h;         // (S, edge) antidiffusive (or, without FCT, HO) horizontal flux
  R *adf_v;         // (S, node) antidiffusive (or HO) vertical flux at interfaces
  R *lo;            // (S, node) LO solution
  R *tmax, *tmin;   // (S, node) cluster bounds (a3, first half)
  R *rp, *rm;       // (S, node) limiter ratios
  R *T_out;         // (S, node) tracer at step n+1
};

// ---------------------------------------------------------------------------
template <typename R, int HOR, int LIM>
__global__ void __launch_bounds__(256) k_edge_flux(DMeshT<R> m, StepArgs<R> a) {
  extern __shared__ int s_off[];
  for_each_cell(m.edge_sched, s_off, [&](int e, int k) {
    const EdgeCtx<R> c = edge_ctx(m, e);
    const R vflux = edge_vflux(m, c, a.vel, k);
    R flo = R(0);
    if (LIM == LIM_FCT) flo = upw1_flux(vflux, a.T[(size_t)c.n1 * m.S + k], a.T[(size_t)c.n2 * m.S + k]);
    R ho;
    if (HOR == HOR_UPW1)
      ho = upw1_flux(vflux, a.TAB[(size_t)c.n1 * m.S + k], a.TAB[(size_t)c.n2 * m.S + k]);
    else
      ho = muscl_flux<R, HOR>(m, c, a.TAB, vflux, a.ph, k);
    const size_t o = (size_t)e * m.S + k;
    if (LIM == LIM_FCT) {
      a.flo[o] = flo;
      a.adf_h[o] = ho - flo;
    } else {
      a.adf_h[o] = ho - R(0);
    }
  });
}

// LO solution (lib/oce_adv_tra_driver.F90:95-211)
template <typename R>
__global__ void __launch_bounds__(256) k_node_lo(DMeshT<R> m, StepArgs<R> a) {
  extern __shared__ int s_off[];
  for_each_cell(m.node_sched, s_off, [&](int n, int k) {
    const int nz = k + 1;
    R acc = R(0);
    for (int p = m.ne_ptr[n]; p < m.ne_ptr[n + 1]; p++) {
      const int code = m.ne[p], e = code >> 1;
      if (nz > m.edge_lev[e].y) continue;
      const R F = a.flo[(size_t)e * m.S + k];
      acc = (code & 1) ? acc - F : acc + F;
    }
    const Col<R> c = column(m, a.T, a.W, n);
    const R fk = ver_upw1(c, nz), fk1 = ver_upw1(c, nz + 1);
    const size_t o = (size_t)n * m.S + k;
    a.lo[o] = (c.T[k] * c.H[k] + (acc + (fk - fk1)) * a.dt / m.areasvol[o]) / c.HN[k];
  });
}

// vertical HO (and antidiffusive) fluxes at the interfaces of each column.
// The thread of layer k writes interface k+1 (1-based), the thread of the
// deepest layer also writes the bottom interface.
template <typename R, int VER, int LIM>
__global__ void __launch_bounds__(256) k_node_vert(DMeshT<R> m, StepArgs<R> a) {
  extern __shared__ int s_off[];
  for_each_cell(m.node_sched, s_off, [&](int n, int k) {
    const Col<R> cT = column(m, a.T, a.W, n);
    const Col<R> cA = column(m, a.TAB, a.W, n);
    const int last = (k + 2 == cT.nlev);
    for (int i = k + 1; i <= k + 1 + last; i++) {
      const R lo = (LIM == LIM_FCT) ? ver_upw1(cT, i) : R(0);
      R v;
      if (VER == VER_PPM) v = ver_ppm(cA, i, a.dt) - lo;
      else if (VER == VER_QR4C) v = ver_qr4c(cA, m.zbar, m.Z, i, a.pv, lo);
      else if (VER == VER_CDIFF) v = ver_cdiff(cA, i, lo);
      else v = ver_upw1(cA, i) - lo;
      a.adf_v[(size_t)n * m.S + (i - 1)] = v;
    }
  });
}

// a1-a3 (first half): max/min over the node's element ring of each element's
// 3-node max/min of (LO, T); elements shallower than the level give -/+1e3
// (lib/oce_adv_tra_fct.F90:105-184)
template <typename R>
__global__ void __launch_bounds__(256) k_node_bounds(DMeshT<R> m, StepArgs<R> a) {
  extern __shared__ int s_off[];
  for_each_cell(m.node_sched, s_off, [&](int n, int k) {
    const int nz = k + 1;
    const R big = R(1e3);
    R tmx = R(0), tmn = R(0);
    for (int p = m.ring_ptr[n]; p < m.ring_ptr[n + 1]; p++) {
      const int el = m.ring_elem[p];
      R amx, amn;
      if (nz <= m.nlev_elem[el] - 1) {
        const int *en = m.elem_nodes + 3 * el;
        const size_t o0 = (size_t)en[0] * m.S + k, o1 = (size_t)en[1] * m.S + k, o2 = (size_t)en[2] * m.S + k;
        const R l0 = a.lo[o0], l1 = a.lo[o1], l2 = a.lo[o2];
        const R t0 = a.T[o0], t1 = a.T[o1], t2 = a.T[o2];
        amx = fmax3(fmax2(l0, t0), fmax2(l1, t1), fmax2(l2, t2));
        amn = fmin3(fmin2(l0, t0), fmin2(l1, t1), fmin2(l2, t2));
      } else {
        amx = -big;
        amn = big;
      }
      if (p == m.ring_ptr[n]) { tmx = amx; tmn = amn; }
      else { tmx = fmax2(tmx, amx); tmn = fmin2(tmn, amn); }
    }
    const size_t o = (size_t)n * m.S + k;
    a.tmax[o] = tmx;
    a.tmin[o] = tmn;
  });
}

// a3 (second half), b1, b2: admissible increments and limiter ratios
// (lib/oce_adv_tra_fct.F90:196-374)
template <typename R>
__global__ void __launch_bounds__(256) k_node_ratio(DMeshT<R> m, StepArgs<R> a) {
  extern __shared__ int s_off[];
  for_each_cell(m.node_sched, s_off, [&](int n, int k) {
    const int nz = k + 1;
    const size_t o = (size_t)n * m.S + k;
    const int nl1 = m.nlev_node[n];
    const R LO = a.lo[o];
    R bmax, bmin;
    if (nz == 1 || nz == nl1 - 1) {
      bmax = a.tmax[o] - LO;
      bmin = a.tmin[o] - LO;
    } else {
      bmax = fmax3(a.tmax[o - 1], a.tmax[o], a.tmax[o + 1]) - LO;
      bmin = fmin3(a.tmin[o - 1], a.tmin[o], a.tmin[o + 1]) - LO;
    }
    const R *av = a.adf_v + (size_t)n * m.S;
    R fp = R(0) + (fmax2(R(0), av[k]) + fmax2(R(0), -av[k + 1]));
    R fm = R(0) + (fmin2(R(0), av[k]) + fmin2(R(0), -av[k + 1]));
    for (int p = m.ne_ptr[n]; p < m.ne_ptr[n + 1]; p++) {
      const int code = m.ne[p], e = code >> 1;
      if (nz > m.edge_lev[e].y) continue;
      const R f = a.adf_h[(size_t)e * m.S + k];
      if (code & 1) {
        fp = fp + fmax2(R(0), -f);
        fm = fm + fmin2(R(0), -f);
      } else {
        fp = fp + fmax2(R(0), f);
        fm = fm + fmin2(R(0), f);
      }
    }
    const R eps = R((double)1e-16f);  // real(MP) :: flux_eps = 1e-16 (default-real literal)
    const R asv = m.areasvol[o];
    R flux = fp * a.dt / asv + eps;
    a.rp[o] = fmin2(R(1), bmax / flux);
    flux = fm * a.dt / asv - eps;
    a.rm[o] = fmin2(R(1), bmin / flux);
  });
}

// limited vertical flux at interface i (lib/oce_adv_tra_fct.F90:396-427)
template <typename R>
__device__ __forceinline__ R limit_v(const R *av, const R *rp, const R *rm, int i, int nlev) {
  const R f = av[i - 1];
  if (i == nlev) return f;
  R ae = R(1);
  if (i == 1) {
    ae = (f >= R(0)) ? fmin2(ae, rp[0]) : fmin2(ae, rm[0]);
  } else if (f >= R(0)) {
    ae = fmin2(ae, rm[i - 2]);
    ae = fmin2(ae, rp[i - 1]);
  } else {
    ae = fmin2(ae, rp[i - 2]);
    ae = fmin2(ae, rm[i - 1]);
  }
  return ae * f;
}

// b3 limiting + oce_tra_adv_flux2dtracer + host update
// (lib/oce_adv_tra_fct.F90:396-471, lib/oce_adv_tra_driver.F90:298-450,
//  src/fesom_analytic.F90:407-437)
template <typename R, int LIM>
__global__ void __launch_bounds__(256) k_node_apply(DMeshT<R> m, StepArgs<R> a) {
  extern __shared__ int s_off[];
  for_each_cell(m.node_sched, s_off, [&](int n, int k) {
    const int nz = k + 1;
    const size_t col = (size_t)n * m.S, o = col + k;
    const int nlev = m.nlev_node[n];
    const R asv = m.areasvol[o];
    const R *av = a.adf_v + col;
    R dv = R(0);
    if (LIM == LIM_FCT) {
      dv = dv - a.T[o] * m.hnode[o] + a.lo[o] * m.hnode_new[o];
      const R *rp = a.rp + col, *rm = a.rm + col;
      const R fk = limit_v(av, rp, rm, nz, nlev), fk1 = limit_v(av, rp, rm, nz + 1, nlev);
      dv = dv + (fk - fk1) * a.dt / asv;
    } else {
      dv = dv + (av[k] - av[k + 1]) * a.dt / asv;
    }
    R dh = R(0);
    for (int p = m.ne_ptr[n]; p < m.ne_ptr[n + 1]; p++) {
      const int code = m.ne[p], e = code >> 1;
      if (nz > m.edge_lev[e].y) continue;
      R f = a.adf_h[(size_t)e * m.S + k];
      if (LIM == LIM_FCT) {
        const int2 nn = m.edge_nodes[e];
        const size_t o1 = (size_t)nn.x * m.S + k, o2 = (size_t)nn.y * m.S + k;
        R ae = R(1);
        if (f >= R(0)) {
          ae = fmin2(ae, a.rp[o1]);
          ae = fmin2(ae, a.rm[o2]);
        } else {
          ae = fmin2(ae, a.rm[o1]);
          ae = fmin2(ae, a.rp[o2]);
        }
        f = ae * f;
      }
      dh = (code & 1) ? dh - f * a.dt / asv : dh + f * a.dt / asv;
    }
    const R del = R(0) + dh + dv;
    a.T_out[o] = a.T[o] + del / m.hnode_new[o];
  });
}

}  // namespace fesom
