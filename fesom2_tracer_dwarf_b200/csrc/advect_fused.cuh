// Kernels of the tracer advection step (do_oce_adv_tra,
// lib/oce_adv_tra_driver.F90:23-294, FCT of lib/oce_adv_tra_fct.F90), fused
// into four passes and batched over up to NTMAX tracers that share a mesh,
// a flow and a scheme.
//
//   k_edge  [edge cells]  volume flux of every edge level (stored once for all
//                         tracers) and, per tracer, the antidiffusive flux
//                         HO(T_AB) - LO(T) (MUSCL/MFCT/UPW1), or HO alone
//                         without FCT
//   k_col1  [node cells]  horizontal LO gather, vertical LO and HO fluxes
//                         (PPM slopes and interface values staged in shared
//                         memory, geometry coefficients shared by the tracers),
//                         LO solution
//   k_col2  [node cells]  FCT cluster bounds (a1-a3), antidiffusive in/out
//                         sums (b1) and limiter ratios (b2)
//   k_col3  [node cells]  limiting (b3), flux2dtracer, T += del / h_new
//
// Edge scatters of the reference become node-centric gathers over the
// node's incident edges in ascending edge id: every node sums its
// contributions in the order of the reference's serial edge loop, with no
// float atomics.  The FP64 build has no FMA contraction and keeps every
// operation of the reference in its order; divisions by a static geometric
// quantity use a once-per-cell reciprocal with Markstein's correction, which
// returns the correctly rounded quotient, i.e. the same bits as a division.
#pragma once
#include <cstdint>

#include "advect_ops.cuh"

namespace fesom {
FESOM_VARIANT_BEGIN

constexpr int NTMAX = 4;
constexpr int kThreads = 256;
// resident 256-thread blocks per SM each step kernel's register budget is
// cut for (4 = 64 registers, 5 = 48, 6 = 40).  Measured on the FP64 plain
// step at 1000x1000x64: more resident warps hide more gather latency than
// the extra spills cost, up to these values (k_col1's shared memory allows
// no more than 5 blocks anyway).  Build-time tuning knobs.
#ifndef FESOM_MINB_EDGE
#define FESOM_MINB_EDGE 5
#endif
#ifndef FESOM_MINB_COL1
#define FESOM_MINB_COL1 5
#endif
#ifndef FESOM_MINB_COL2
#define FESOM_MINB_COL2 6
#endif
#ifndef FESOM_MINB_COL3
#define FESOM_MINB_COL3 6
#endif
#ifndef FESOM_MINB_GRAD
#define FESOM_MINB_GRAD 5
#endif
// The same for the FP32-arithmetic kernels (FP32 and 16-bit storage), which
// need fewer registers: timed on the same workload in FP32, 4 / 5 / 6 / 7
// blocks (col2, col3: up to 8): edge best at 6 (1.98 ms), col1 at 7 (2.07),
// col2 and col3 at 7 (1.68, 1.65; 8 no better), against 1.99 / 2.38 / 1.86 /
// 1.97 ms with the FP64 budgets.
#ifndef FESOM_MINB32_EDGE
#define FESOM_MINB32_EDGE 6
#endif
#ifndef FESOM_MINB32_COL1
#define FESOM_MINB32_COL1 7
#endif
#ifndef FESOM_MINB32_COL2
#define FESOM_MINB32_COL2 7
#endif
#ifndef FESOM_MINB32_COL3
#define FESOM_MINB32_COL3 7
#endif
#ifndef FESOM_MINB32_GRAD
#define FESOM_MINB32_GRAD 5
#endif
template <typename R>
struct MinBlocks {
  static constexpr int grad = FESOM_MINB_GRAD, edge = FESOM_MINB_EDGE, col1 = FESOM_MINB_COL1, col2 = FESOM_MINB_COL2,
                       col3 = FESOM_MINB_COL3;
};
template <>
struct MinBlocks<float> {
  static constexpr int grad = FESOM_MINB32_GRAD, edge = FESOM_MINB32_EDGE, col1 = FESOM_MINB32_COL1,
                       col2 = FESOM_MINB32_COL2, col3 = FESOM_MINB32_COL3;
};
// Incidence records of each node kernel's block staged in shared memory or
// read through L1, per arithmetic type.  Measured on the 1000x1000x64 step:
// FP64 staged k_col1 3.28 ms (unstaged 3.34), k_col2 2.39 (2.50), k_col3 2.75
// (2.75); FP32 unstaged k_col1 1.81 (staged 1.84), k_col2 1.61 (1.68), k_col3
// 1.57 (1.60) -- the FP32 kernels keep more blocks resident, whose shared
// memory would otherwise crowd out the L1.
template <typename R>
struct StageIncidence {
  static constexpr bool col1 = true, col2 = true, col3 = true;
};
template <>
struct StageIncidence<float> {
  static constexpr bool col1 = false, col2 = false, col3 = false;
};
// The LO gather of k_col1 issues the loads of this many incident edges
// together before using any of them.  Every (edge, level) and (node, level)
// address of a cell's level lies inside its padded column, so the loads of
// dry edge levels, and of the clamped records past the node's last edge, are
// in bounds; their values are discarded.  The fluxes are still accumulated
// one edge at a time in ascending incidence order.  (Measured per kernel on
// the 512-cell capped schedules at 1000x1000x64: k_col1 FP64 with 1 / 2 / 3
// / 4 / 6 edges 3.24 / 2.89 / 2.76 / 3.14 / 2.98 ms, FP32 with 2 / 3 / 4 / 6
// 1.71 / 1.59 / 1.71 / 1.76 ms; the same form is slower in k_col2 and
// k_col3, whose loops stay one edge at a time.)
#ifndef FESOM_GCHUNK_COL1
#define FESOM_GCHUNK_COL1 3
#endif
constexpr int kGChunkCol1 = FESOM_GCHUNK_COL1;
constexpr int kCellsPerBlock = 512;      // schedule cap: wet cells per block (two per thread)
constexpr int kMaxCellsPerBlock = 576;   // upper bound (target + deepest column)
constexpr int kMaxItemsPerBlock = 512;

// ---------------------------------------------------------------------------
// Correctly rounded division a / b given y = RN(1/b).
//
// Markstein's theorem (P. Markstein, "Computation of elementary functions on
// the IBM RISC System/6000 processor", IBM J. Res. Dev. 34, 1990; see also
// Muller et al., Handbook of Floating-Point Arithmetic, Sec. 4.7): if y is
// within half an ulp of 1/b and q is a faithful approximation of a/b, then
// r = a - b q is exact when computed with one FMA and RN(q + r y) = RN(a/b).
// q0 = RN(a y) can be 1.5 ulp off, so one correction first makes it faithful,
// the second rounds correctly.  Zero and extreme magnitudes (where r could
// underflow or overflow) take the plain division.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double div_rcp(double a, double b, double y) {
  const double aa = fabs(a);
  if (!(aa > 0x1p-900 && aa < 0x1p900)) return a / b;
  double q = a * y;
  double r = __fma_rn(-b, q, a);
  if (r == 0.0) return q;
  q = __fma_rn(r, y, q);
  r = __fma_rn(-b, q, a);
  return __fma_rn(r, y, q);
}
__device__ __forceinline__ float div_rcp(float a, float b, float y) {
  const float aa = fabsf(a);
  if (!(aa > 0x1p-100f && aa < 0x1p100f)) return a / b;
  float q = a * y;
  float r = __fmaf_rn(-b, q, a);
  if (r == 0.0f) return q;
  q = __fmaf_rn(r, y, q);
  r = __fmaf_rn(-b, q, a);
  return __fmaf_rn(r, y, q);
}

// R: compute and geometry type; TS: tracer storage type (R itself, or a
// 16-bit float with R = float)
template <typename R, typename TS>
struct FusedArgs {
  const TS *T[NTMAX];     // values
  const TS *TAB[NTMAX];   // valuesAB (high-order fluxes)
  TS *T_out[NTMAX];
  R *adf_h[NTMAX];        // (NT, S, edge) tracer-interleaved: adf_h[t] = adf_h[0] + t, stride NT
  R *adf_v[NTMAX];        // (NT, S, node) interfaces, tracer-interleaved like adf_h
  R *lo[NTMAX];           // (NT, S, node) tracer-interleaved like adf_h
  R *rpm[NTMAX];          // (2, S, node): limiter ratios R+ and R- of each cell side by side
  R *vflux;               // (S, edge), shared by the tracers
  R *gradn[NTMAX];        // (2, S, node): ring-mean gradient (gx, gy) of valuesAB
  const R *vel;           // (2, S, elem)
  const R *W;             // (S, node) interfaces
  R dt, ph, pv;
  // learned flux (FP32 only): when feat[t] is set the edge kernel writes 16
  // BF16 features and the correction scale of every MUSCL edge cell (dense
  // edge-schedule index)
  __nv_bfloat16 *feat[NTMAX];
  float *fscale[NTMAX];
  R off[NTMAX];           // storage offsets (16-bit storage)
  uint32_t seed[NTMAX];   // per-step random stream of each tracer (stochastic rounding)
  int sround;             // 1: stochastic rounding of 16-bit stores
  // edge volume fluxes: 0 computed from the velocity (stored in vflux when the
  // limiter needs them), 1 computed and stored, 2 loaded from vflux (stored
  // by an earlier launch with the same velocity)
  int vflux_mode;
  // failure detection: count of non-finite new values (nullptr: not counted)
  unsigned long long *nonfinite;
};

// ---------------------------------------------------------------------------
// block cell maps: a block owns a range of items (nodes or edges); every wet
// cell of those items gets the local item index in shared memory
// ---------------------------------------------------------------------------
struct CellMap {
  int i0, ni, c0, nc;
};

__device__ __forceinline__ CellMap map_cells(const DSched &sc, int blk, int *s_off, int *s_item) {
  CellMap cm;
  cm.i0 = sc.blk[blk];
  cm.ni = sc.blk[blk + 1] - cm.i0;
  for (int t = threadIdx.x; t <= cm.ni; t += blockDim.x) s_off[t] = sc.cell_off[cm.i0 + t];
  __syncthreads();
  cm.c0 = s_off[0];
  cm.nc = s_off[cm.ni] - cm.c0;
  for (int j = threadIdx.x; j < cm.ni; j += blockDim.x) {
    const int a = s_off[j] - cm.c0, b = s_off[j + 1] - cm.c0;
    for (int q = a; q < b; q++) s_item[q] = j;
  }
  __syncthreads();
  return cm;
}

// A node block's incidence records (the CSR slice of its nodes) staged in
// shared memory by one cooperative load, so that every lane's walk over its
// node's edges starts from shared memory instead of a dependent global load.
// Blocks with more than kNeStage records read them from global memory.
constexpr int kNeStage = 512;
__host__ __device__ constexpr size_t smem_stage() {
  return 16 + (size_t)kNeStage * sizeof(int4) + sizeof(int) * (kMaxItemsPerBlock + 1);
}

struct Incidence {
  const int4 *ne;   // records of the block, from its first node's first record
  const int *nep;   // per local node: first record (minus sub)
  int sub;
};

// STAGE = false reads the records from global memory (through L1) and needs
// no shared memory for them.
template <bool STAGE = true, typename R>
__device__ __forceinline__ Incidence stage_incidence(const DMeshT<R> &m, const CellMap &cm, void *region) {
  int4 *s_ne = reinterpret_cast<int4 *>(((uintptr_t)region + 15) & ~(uintptr_t)15);
  int *s_nep = reinterpret_cast<int *>(s_ne + kNeStage);
  const int p0 = m.ne_ptr[cm.i0], p1 = m.ne_ptr[cm.i0 + cm.ni];
  Incidence r;
  if (STAGE && p1 - p0 <= kNeStage) {
    for (int i = threadIdx.x; i < p1 - p0; i += blockDim.x) s_ne[i] = m.ne4[p0 + i];
    for (int j = threadIdx.x; j <= cm.ni; j += blockDim.x) s_nep[j] = m.ne_ptr[cm.i0 + j] - p0;
    r.ne = s_ne;
    r.nep = s_nep;
    r.sub = 0;
  } else {
    r.ne = m.ne4 + p0;
    r.nep = m.ne_ptr + cm.i0;
    r.sub = p0;
  }
  __syncthreads();
  return r;
}

// ---------------------------------------------------------------------------
// k_grad: ring-mean gradients of valuesAB (lib/oce_muscl_adv.F90:400-450:
// the mean of tr_xy over the node's ring, weighted by element area), for the
// node-levels where some incident edge lacks a shared up/down pair
// ---------------------------------------------------------------------------
__device__ __forceinline__ void ld_pair(const double *p, double &x, double &y) {
  const double2 v = *reinterpret_cast<const double2 *>(p);
  x = v.x;
  y = v.y;
}
__device__ __forceinline__ void ld_pair(const float *p, float &x, float &y) {
  const float2 v = *reinterpret_cast<const float2 *>(p);
  x = v.x;
  y = v.y;
}
__device__ __forceinline__ void st_pair(double *p, double x, double y) {
  *reinterpret_cast<double2 *>(p) = make_double2(x, y);
}
__device__ __forceinline__ void st_pair(float *p, float x, float y) {
  *reinterpret_cast<float2 *>(p) = make_float2(x, y);
}

// Tracer-interleaved work arrays (adf_h, lo): tracer t's value of cell o is
// at X[t][o * NT] with X[t] = X[0] + t, so one vector load brings a cell's
// values of every tracer of the batch (NT = 1, 2 or 4).
template <int NT, typename R>
__device__ __forceinline__ R &il(R *const *x, int t, cix o) {
  return x[t][(size_t)o * NT];
}
template <int NT>
__device__ __forceinline__ void il_load(const double *x0, cix o, double *v) {
  const double *p = x0 + (size_t)o * NT;
  if constexpr (NT == 1) {
    v[0] = p[0];
  } else if constexpr (NT == 2) {
    const double2 a = *reinterpret_cast<const double2 *>(p);
    v[0] = a.x; v[1] = a.y;
  } else {
    static_assert(NT == 4, "batches hold 1, 2 or 4 tracers");
    const double2 a = reinterpret_cast<const double2 *>(p)[0], b = reinterpret_cast<const double2 *>(p)[1];
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
  }
}
template <int NT>
__device__ __forceinline__ void il_load(const float *x0, cix o, float *v) {
  const float *p = x0 + (size_t)o * NT;
  if constexpr (NT == 1) {
    v[0] = p[0];
  } else if constexpr (NT == 2) {
    const float2 a = *reinterpret_cast<const float2 *>(p);
    v[0] = a.x; v[1] = a.y;
  } else {
    static_assert(NT == 4, "batches hold 1, 2 or 4 tracers");
    const float4 a = *reinterpret_cast<const float4 *>(p);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
  }
}

template <typename R, typename TS, int NT>
__device__ __forceinline__ void grad_block(const DMeshT<R> &m, const FusedArgs<R, TS> &a, int blk, int *smem) {
  int *s_off = smem, *s_item = smem + kMaxItemsPerBlock + 1;
  const CellMap cm = map_cells(m.grad_sched, blk, s_off, s_item);
  for (int lc = threadIdx.x; lc < cm.nc; lc += blockDim.x) {
    const int j = s_item[lc], n = cm.i0 + j, k = m.grad_lev0[n] + lc - (s_off[j] - cm.c0);
    R gx[NTMAX], gy[NTMAX];
    ring_mean_n(m, a.TAB, a.off, NT, n, k, gx, gy);
    const cix o = (cix)n * m.S + k;
    for (int t = 0; t < NT; t++) st_pair(a.gradn[t] + 2 * o, gx[t], gy[t]);
  }
}

template <typename R, typename TS, int NT>
__global__ void __launch_bounds__(kThreads, MinBlocks<R>::grad) k_grad(DMeshT<R> m, FusedArgs<R, TS> a) {
  extern __shared__ int smem[];
  grad_block<R, TS, NT>(m, a, blockIdx.x, smem);
}

// ---------------------------------------------------------------------------
// k_edge
// ---------------------------------------------------------------------------
template <typename R, typename TS>
__device__ __forceinline__ void trxy_n(const DMeshT<R> &m, const TS *const *tab, const R *off, int NT, int elem, int k,
                                       R *gx, R *gy) {
  const int *en = m.elem_nodes + 3 * elem;
  const int a = en[0], b = en[1], c = en[2];
  const R *gs = m.grad_sca + 6 * elem;
  const R g0 = gs[0], g1 = gs[1], g2 = gs[2], g3 = gs[3], g4 = gs[4], g5 = gs[5];
  for (int t = 0; t < NT; t++) {
    const R t1 = ldT(tab[t], (cix)a * m.S + k, off[t]), t2 = ldT(tab[t], (cix)b * m.S + k, off[t]), t3 = ldT(tab[t], (cix)c * m.S + k, off[t]);
    gx[t] = (g0 * t1 + g1 * t2) + g2 * t3;
    gy[t] = (g3 * t1 + g4 * t2) + g5 * t3;
  }
}

template <typename R, typename TS>
__device__ __forceinline__ void ring_mean_n(const DMeshT<R> &m, const TS *const *tab, const R *off, int NT, int n, int k,
                                            R *gx, R *gy) {
  R tvol = R(0), tx[NTMAX], ty[NTMAX];
  for (int t = 0; t < NT; t++) { tx[t] = R(0); ty[t] = R(0); }
  const int nz = k + 1;
  for (int p = m.ring_ptr[n]; p < m.ring_ptr[n + 1]; p++) {
    const int el = m.ring_elem[p];
    if (m.nlev_elem[el] - 1 < nz) continue;
    R ax[NTMAX], ay[NTMAX];
    trxy_n(m, tab, off, NT, el, k, ax, ay);
    const R a = m.elem_area[el];
    tvol = tvol + a;
    for (int t = 0; t < NT; t++) {
      tx[t] = tx[t] + ax[t] * a;
      ty[t] = ty[t] + ay[t] * a;
    }
  }
  for (int t = 0; t < NT; t++) {
    gx[t] = tx[t] / tvol;
    gy[t] = ty[t] / tvol;
  }
}

template <typename R, typename TS, int NT, int HOR, int LIM>
__device__ __forceinline__ void edge_block(const DMeshT<R> &m, const FusedArgs<R, TS> &a, int blk, int *smem) {
  int *s_off = smem, *s_item = smem + kMaxItemsPerBlock + 1;
  const CellMap cm = map_cells(m.edge_sched, blk, s_off, s_item);
  const R re = R(kREarthD), sixth = R(1.0 / 6.0);
  for (int lc = threadIdx.x; lc < cm.nc; lc += blockDim.x) {
    const int j = s_item[lc], e = cm.i0 + j, k = lc - (s_off[j] - cm.c0);
    const cix o = (cix)e * m.S + k;
    const int2 nn = m.edge_nodes[e];
    R vflux;
    if (a.vflux_mode == 2) {
      vflux = a.vflux[o];
    } else {
      vflux = edge_vflux(m, edge_ctx(m, e), a.vel, k);
      if (LIM == LIM_FCT || a.vflux_mode == 1) a.vflux[o] = vflux;
    }
    const cix o1 = (cix)nn.x * m.S + k, o2 = (cix)nn.y * m.S + k;
    if (HOR == HOR_UPW1) {
      for (int t = 0; t < NT; t++) {
        const R flo = (LIM == LIM_FCT) ? upw1_flux(vflux, ldT(a.T[t], o1, a.off[t]), ldT(a.T[t], o2, a.off[t])) : R(0);
        il<NT>(a.adf_h, t, o) = upw1_flux(vflux, ldT(a.TAB[t], o1, a.off[t]), ldT(a.TAB[t], o2, a.off[t])) - flo;
      }
      continue;
    }
    // edge_up_dn_grad (lib/oce_muscl_adv.F90:383-527)
    R gux[NTMAX], guy[NTMAX], gdx[NTMAX], gdy[NTMAX];
    const int2 ud = m.up_dn[e];
    bool shared = false;
    if (ud.x >= 0 && ud.y >= 0) shared = (k + 1) <= min(m.nlev_node_min[nn.x], m.nlev_node_min[nn.y]) - 1;
    if (shared) {
      trxy_n(m, a.TAB, a.off, NT, ud.x, k, gux, guy);
      trxy_n(m, a.TAB, a.off, NT, ud.y, k, gdx, gdy);
    } else {
      // node ring means, computed once per node-level by k_grad
      for (int t = 0; t < NT; t++) {
        ld_pair(a.gradn[t] + 2 * o1, gux[t], guy[t]);
        ld_pair(a.gradn[t] + 2 * o2, gdx[t], gdy[t]);
      }
    }
    const R ex = m.edge_dxdy[2 * e], ey = m.edge_dxdy[2 * e + 1], aa = m.edge_a[e];
    R c_lo1 = R(1), c_lo2 = R(1);
    if (HOR == HOR_MUSCL) {
      c_lo1 = (m.nbl[nn.x] - (k + 1) >= 0) ? R(1) : R(0);
      c_lo2 = (m.nbl[nn.y] - (k + 1) >= 0) ? R(1) : R(0);
    }
    for (int t = 0; t < NT; t++) {
      const R t1 = ldT(a.TAB[t], o1, a.off[t]), t2 = ldT(a.TAB[t], o2, a.off[t]);
      R Tmean2, Tmean1;
      // lib/oce_adv_tra_hor.F90:454-469 (MUSCL), :743-753 (MFCT, no c_lo)
      const R x2 = R(2) * (t2 - t1) + ex * aa * gdx[t] + ey * re * gdy[t];
      const R x1 = R(2) * (t2 - t1) + ex * aa * gux[t] + ey * re * guy[t];
      if (HOR == HOR_MUSCL) {
        Tmean2 = t2 - div_rcp(x2, R(6), sixth) * c_lo2;
        Tmean1 = t1 + div_rcp(x1, R(6), sixth) * c_lo1;
      } else {
        Tmean2 = t2 - div_rcp(x2, R(6), sixth);
        Tmean1 = t1 + div_rcp(x1, R(6), sixth);
      }
      const R cHO = (vflux + fabs(vflux)) * Tmean1 + (vflux - fabs(vflux)) * Tmean2;
      const R ho = -(R(0.5) * (R(1) - a.ph) * cHO) - vflux * a.ph * R(0.5) * (Tmean1 + Tmean2);
      const R flo = (LIM == LIM_FCT) ? upw1_flux(vflux, ldT(a.T[t], o1, a.off[t]), ldT(a.T[t], o2, a.off[t])) : R(0);
      il<NT>(a.adf_h, t, o) = ho - flo;
      if constexpr (sizeof(R) == 4 && HOR == HOR_MUSCL) {
        if (a.feat[t]) {
          // features in the flow's frame, in units of the local variation sig
          const bool fwd = vflux >= R(0);
          const R tu = fwd ? t1 : t2, td = fwd ? t2 : t1;
          const R xu = fwd ? x1 : -x2, xd = fwd ? x2 : -x1;
          const R face = R(0.5) * (Tmean1 + Tmean2);
          const R sig = fabs(td - tu) + (fabs(xu) + fabs(xd)) * sixth + R(1e-6) * (fabs(tu) + fabs(td)) + R(1e-20);
          const R inv = R(1) / sig;
          const cix ou = fwd ? o1 : o2;
          const R cour = fmin(fabs(vflux) * a.dt / (m.areasvol[ou] * m.hnode_new[ou]), R(4));
          const R gx = fwd ? gux[t] : gdx[t], gy = fwd ? guy[t] : gdy[t];
          const R trans = (-ey * re * gx + ex * aa * gy) * inv;
          float f[16];
          f[0] = (float)((td - tu) * inv);
          f[1] = (float)(xu * sixth * inv);
          f[2] = (float)(xd * sixth * inv);
          f[3] = (float)((face - tu) * inv);
          f[4] = (float)cour;
          f[5] = (float)(cour * cour);
          f[6] = (float)(fwd ? c_lo1 : c_lo2);
          f[7] = (float)(fwd ? c_lo2 : c_lo1);
          f[8] = (float)k / (float)max(1, m.nl - 2);
          f[9] = shared ? 1.0f : 0.0f;
          f[10] = fabsf(f[0]);
          f[11] = f[1] - f[2];
          f[12] = (xu * xd > R(0)) ? 1.0f : -1.0f;
          f[13] = fminf(fabsf(f[1]), fabsf(f[2]));
          f[14] = fmaxf(-8.0f, fminf(8.0f, (float)trans));
          f[15] = 1.0f;
          const int cell = cm.c0 + lc;
          __align__(16) __nv_bfloat16 h[16];
          for (int q = 0; q < 16; q++) h[q] = __float2bfloat16_rn(f[q]);
          uint4 *dst = reinterpret_cast<uint4 *>(a.feat[t] + (size_t)cell * 16);
          dst[0] = reinterpret_cast<const uint4 *>(h)[0];
          dst[1] = reinterpret_cast<const uint4 *>(h)[1];
          a.fscale[t][cell] = (float)(-vflux * sig);
        }
      }
    }
  }
}

template <typename R, typename TS, int NT, int HOR, int LIM>
__global__ void __launch_bounds__(kThreads, MinBlocks<R>::edge) k_edge(DMeshT<R> m, FusedArgs<R, TS> a) {
  extern __shared__ int smem[];
  edge_block<R, TS, NT, HOR, LIM>(m, a, blockIdx.x, smem);
}

// ---------------------------------------------------------------------------
// k_col1: LO solution and vertical fluxes
// ---------------------------------------------------------------------------
// PPM slope of layer j (1-based) with the limiter of lib/oce_adv_tra_ver.F90:
// 525-540; c1, c2, c3 are the geometric factors of that layer.
template <typename R>
__device__ __forceinline__ R ppm_slope(R Tm1, R T0, R Tp1, R c1, R c2, R c3) {
  R d = c1 * (c2 * (Tp1 - T0) + c3 * (T0 - Tm1));
  if ((Tp1 - T0) * (T0 - Tm1) > R(0))
    d = fmin3(fabs(d), R(2) * fabs(Tp1 - T0), R(2) * fabs(T0 - Tm1)) * sgn1(d);
  else
    d = R(0);
  return d;
}

template <typename R, typename TS, int NT, int VER, int LIM>
__device__ __forceinline__ void col1_block(const DMeshT<R> &m, const FusedArgs<R, TS> &a, int blk, int *smem) {
  int *s_off = smem, *s_item = smem + kMaxItemsPerBlock + 1;
  R *s_slope = (R *)(smem + kMaxItemsPerBlock + 1 + kMaxCellsPerBlock + 1);  // 16-byte aligned below
  s_slope = (R *)(((uintptr_t)s_slope + 15) & ~(uintptr_t)15);
  R *s_tv = s_slope + NT * kMaxCellsPerBlock;
  // the vertical LO fluxes of stage C reuse the slopes' storage, dead after
  // stage B: two arrays of shared memory instead of three leave more of the
  // SM's unified L1 to the column and neighbour re-reads
  R *s_fv = s_slope;
  const CellMap cm = map_cells(m.node_sched, blk, s_off, s_item);
  const Incidence inc = stage_incidence<StageIncidence<R>::col1>(m, cm, s_tv + NT * kMaxCellsPerBlock);
  const int S = m.S;

  // stage A: PPM slopes
  for (int lc = threadIdx.x; lc < cm.nc; lc += blockDim.x) {
    const int j = s_item[lc], n = cm.i0 + j, k = lc - (s_off[j] - cm.c0), nz = k + 1;
    if (VER == VER_PPM) {
      const int nlev = m.nlev_node[n];
      if (nz >= 2 && nz <= nlev - 2) {
        const R *HN = m.hnode_new + (cix)n * S;
        const R dzjm1 = HN[k - 1], dzj = HN[k], dzjp1 = HN[k + 1];
        const R c1 = dzj / (dzjm1 + dzj + dzjp1);
        const R c2 = (R(2) * dzjm1 + dzj) / (dzjp1 + dzj);
        const R c3 = (dzj + R(2) * dzjp1) / (dzjm1 + dzj);
        for (int t = 0; t < NT; t++) {
          const TS *Tc = a.TAB[t] + (cix)n * S;
          s_slope[t * kMaxCellsPerBlock + lc] = ppm_slope(ldT(Tc, k - 1, a.off[t]), ldT(Tc, k, a.off[t]), ldT(Tc, k + 1, a.off[t]), c1, c2, c3);
        }
      }
    }
  }
  __syncthreads();

  // stage B: PPM interface values tv(i), interface i = nz (top of layer nz)
  if (VER == VER_PPM) {
    for (int lc = threadIdx.x; lc < cm.nc; lc += blockDim.x) {
      const int j = s_item[lc], n = cm.i0 + j, k = lc - (s_off[j] - cm.c0), i = k + 1;
      const int nlev = m.nlev_node[n];
      const R *HN = m.hnode_new + (cix)n * S;
      const R *Wc = a.W + (cix)n * S;
      if (i == 1) {
        for (int t = 0; t < NT; t++) s_tv[t * kMaxCellsPerBlock + lc] = ldT(a.TAB[t], (cix)n * S, a.off[t]);
      } else if (i == nlev - 1) {
        const R s = sgn1(Wc[nlev - 2]);
        for (int t = 0; t < NT; t++) {
          const TS *Tc = a.TAB[t] + (cix)n * S;
          s_tv[t * kMaxCellsPerBlock + lc] = -ldT(Tc, nlev - 3, a.off[t]) * fmin2(s, R(0)) + ldT(Tc, nlev - 2, a.off[t]) * fmax2(s, R(0));
        }
      } else if (i == 2) {
        for (int t = 0; t < NT; t++) {
          const TS *Tc = a.TAB[t] + (cix)n * S;
          s_tv[t * kMaxCellsPerBlock + lc] = R(0.5) * (ldT(Tc, 0, a.off[t]) + ldT(Tc, 1, a.off[t]));
        }
      } else {
        // lib/oce_adv_tra_ver.F90:545-553 with nz = i - 1
        const int nzz = i - 1;  // 1-based layer above the interface
        const R dzjm1 = HN[nzz - 2], dzj = HN[nzz - 1], dzjp1 = HN[nzz], dzjp2 = HN[nzz + 1];
        const R A = dzj / (dzj + dzjp1);
        const R B = R(1) / (dzjm1 + dzj + dzjp1 + dzjp2);
        const R C = (R(2) * dzjp1 * dzj) / (dzj + dzjp1) *
                    ((dzjm1 + dzj) / (R(2) * dzj + dzjp1) - (dzjp2 + dzjp1) / (R(2) * dzjp1 + dzj));
        const R D = dzj * (dzjm1 + dzj) / (R(2) * dzj + dzjp1);
        const R E = dzjp1 * (dzjp1 + dzjp2) / (dzj + R(2) * dzjp1);
        for (int t = 0; t < NT; t++) {
          const TS *Tc = a.TAB[t] + (cix)n * S;
          const R T0 = ldT(Tc, nzz - 1, a.off[t]), T1 = ldT(Tc, nzz, a.off[t]);
          const R dj = s_slope[t * kMaxCellsPerBlock + lc - 1];   // layer nzz
          const R djp1 = s_slope[t * kMaxCellsPerBlock + lc];     // layer nzz + 1
          s_tv[t * kMaxCellsPerBlock + lc] = T0 + A * (T1 - T0) + B * (C * (T1 - T0) - D * djp1 + E * dj);
        }
      }
    }
    __syncthreads();
  }

  // stage C: fluxes at interface i = nz (and the bottom one for the deepest layer)
  for (int lc = threadIdx.x; lc < cm.nc; lc += blockDim.x) {
    const int j = s_item[lc], n = cm.i0 + j, k = lc - (s_off[j] - cm.c0);
    const cix col = (cix)n * S;
    const int nlev = m.nlev_node[n];
    const R *Wc = a.W + col, *Ac = m.area + col;
    const int i_last = (k + 2 == nlev) ? k + 2 : k + 1;
    for (int i = k + 1; i <= i_last; i++) {
      R lov[NTMAX], hov[NTMAX];
      for (int t = 0; t < NT; t++) lov[t] = R(0);
      if (LIM == LIM_FCT) {
        for (int t = 0; t < NT; t++) {
          Col<R, TS> cT;
          cT.T = a.T[t] + col; cT.W = Wc; cT.A = Ac; cT.nlev = nlev; cT.off = a.off[t];
          lov[t] = ver_upw1(cT, i);
        }
      }
      if (VER == VER_PPM) {
        // lib/oce_adv_tra_ver.F90:597-639
        if (i == nlev) {
          for (int t = 0; t < NT; t++) hov[t] = R(0) - lov[t];
        } else if (i == 1) {
          for (int t = 0; t < NT; t++) hov[t] = -(s_tv[t * kMaxCellsPerBlock + lc] * Wc[0] * Ac[0]) - lov[t];
        } else {
          const R w = Wc[i - 1];
          if (!(w > R(0)) && !(w < R(0))) {
            for (int t = 0; t < NT; t++) hov[t] = R(0) - lov[t];
          } else {
            const int jl = (w > R(0)) ? i : i - 1;              // supplying layer (1-based)
            const int sl = lc + (jl - i);                        // its cell slot
            const R dzj = m.hnode[col + jl - 1];
            const R x = (w > R(0)) ? fmin2(w * a.dt / dzj, R(1)) : fmin2(-(w * a.dt / dzj), R(1));
            const R two3 = R(2.0 / 3.0), sixth = R(1.0 / 6.0);
            for (int t = 0; t < NT; t++) {
              const R Tc = ldT(a.TAB[t], col + jl - 1, a.off[t]);
              R aL = s_tv[t * kMaxCellsPerBlock + sl];
              R aR = (jl + 1 == nlev) ? ldT(a.TAB[t], col + nlev - 2, a.off[t]) : s_tv[t * kMaxCellsPerBlock + sl + 1];
              if ((aR - Tc) * (Tc - aL) <= R(0)) { aL = Tc; aR = Tc; }
              // x / 6 by the corrected reciprocal (correctly rounded, as in the MUSCL fluxes)
              if ((aR - aL) * (Tc - R(0.5) * (aL + aR)) > div_rcp((aR - aL) * (aR - aL), R(6), sixth)) aL = R(3) * Tc - R(2) * aR;
              if ((aR - aL) * (Tc - R(0.5) * (aR + aL)) < -div_rcp((aR - aL) * (aR - aL), R(6), sixth)) aR = R(3) * Tc - R(2) * aL;
              const R aj = R(6) * (Tc - R(0.5) * (aL + aR));
              R tt;
              if (w > R(0)) tt = (-aL - R(0.5) * x * (aR - aL + (R(1) - two3 * x) * aj));
              else tt = (-aR + R(0.5) * x * (aR - aL - (R(1) - two3 * x) * aj));
              hov[t] = tt * Ac[i - 1] * w - lov[t];
            }
          }
        }
      } else {
        for (int t = 0; t < NT; t++) {
          Col<R, TS> cA;
          cA.T = a.TAB[t] + col; cA.W = Wc; cA.A = Ac; cA.nlev = nlev; cA.off = a.off[t];
          if (VER == VER_QR4C) hov[t] = ver_qr4c(cA, m.zbar, m.Z, i, a.pv, lov[t]);
          else if (VER == VER_CDIFF) hov[t] = ver_cdiff(cA, i, lov[t]);
          else hov[t] = ver_upw1(cA, i) - lov[t];
        }
      }
      for (int t = 0; t < NT; t++) {
        il<NT>(a.adf_v, t, col + i - 1) = hov[t];
        if (LIM == LIM_FCT && i == k + 1) s_fv[t * kMaxCellsPerBlock + lc] = lov[t];
      }
    }
  }
  if (LIM != LIM_FCT) return;
  __syncthreads();

  // stage D: horizontal LO gather and the LO solution
  // (lib/oce_adv_tra_driver.F90:122-181, :202-211)
  for (int lc = threadIdx.x; lc < cm.nc; lc += blockDim.x) {
    const int j = s_item[lc], n = cm.i0 + j, k = lc - (s_off[j] - cm.c0), nz = k + 1;
    const cix o = (cix)n * S + k;
    const int nlev = m.nlev_node[n];
    R acc[NTMAX], tself[NTMAX];
    for (int t = 0; t < NT; t++) {
      acc[t] = R(0);
      tself[t] = ldT(a.T[t], o, a.off[t]);
    }
    for (int p = inc.nep[j] - inc.sub, pe = inc.nep[j + 1] - inc.sub; p < pe; p += kGChunkCol1) {
      int4 qs[kGChunkCol1];
      R vfs[kGChunkCol1], tos[kGChunkCol1][NT];
#pragma unroll
      for (int u = 0; u < kGChunkCol1; u++) {
        qs[u] = inc.ne[min(p + u, pe - 1)];
        vfs[u] = a.vflux[(cix)(qs[u].x >> 1) * S + k];
        const cix oo = (cix)qs[u].w + k;  // the edge's other node (column base in .w)
        for (int t = 0; t < NT; t++) tos[u][t] = ldT(a.T[t], oo, a.off[t]);
      }
#pragma unroll
      for (int u = 0; u < kGChunkCol1; u++) {
        if (p + u >= pe || nz > qs[u].z) continue;
        const bool second = qs[u].x & 1;
        for (int t = 0; t < NT; t++) {
          // upw1_flux(vf, T(first node), T(second node))
          const R F = second ? upw1_flux(vfs[u], tos[u][t], tself[t]) : upw1_flux(vfs[u], tself[t], tos[u][t]);
          acc[t] = second ? acc[t] - F : acc[t] + F;
        }
      }
    }
    const R asv = m.areasvol[o], hn = m.hnode_new[o], h = m.hnode[o];
    const R yasv = m.rcp[o], yhn = m.rcp[m.rcp_plane + o];  // reciprocal planes (k_rcp_planes)
    for (int t = 0; t < NT; t++) {
      const R fk = s_fv[t * kMaxCellsPerBlock + lc];
      const R fk1 = (k + 2 == nlev) ? R(0) : s_fv[t * kMaxCellsPerBlock + lc + 1];
      const R num = tself[t] * h + div_rcp((acc[t] + (fk - fk1)) * a.dt, asv, yasv);
      il<NT>(a.lo, t, o) = div_rcp(num, hn, yhn);
    }
  }
}

template <typename R, typename TS, int NT, int VER, int LIM>
__global__ void __launch_bounds__(kThreads, MinBlocks<R>::col1) k_col1(DMeshT<R> m, FusedArgs<R, TS> a) {
  extern __shared__ int smem[];
  col1_block<R, TS, NT, VER, LIM>(m, a, blockIdx.x, smem);
}

// ---------------------------------------------------------------------------
// k_col2: bounds, in/out sums, ratios (lib/oce_adv_tra_fct.F90:105-374)
// ---------------------------------------------------------------------------
template <typename R, typename TS, int NT>
__device__ __forceinline__ void col2_block(const DMeshT<R> &m, const FusedArgs<R, TS> &a, int blk, int *smem) {
  int *s_off = smem, *s_item = smem + kMaxItemsPerBlock + 1;
  R *s_mx = (R *)(smem + kMaxItemsPerBlock + 1 + kMaxCellsPerBlock + 1);
  s_mx = (R *)(((uintptr_t)s_mx + 15) & ~(uintptr_t)15);
  R *s_mn = s_mx + NT * kMaxCellsPerBlock;
  const CellMap cm = map_cells(m.node_sched, blk, s_off, s_item);
  const Incidence inc = stage_incidence<StageIncidence<R>::col2>(m, cm, s_mn + NT * kMaxCellsPerBlock);
  const int S = m.S;
  const R big = R(1e3);

  for (int lc = threadIdx.x; lc < cm.nc; lc += blockDim.x) {
    const int j = s_item[lc], n = cm.i0 + j, k = lc - (s_off[j] - cm.c0), nz = k + 1;
    R tmx[NTMAX], tmn[NTMAX];
    if (m.ring_full[n]) {
      // With a complete ring, the nodes of the ring elements wet at this level
      // are the node itself and the far ends of its edges wet at this level
      // (each such edge has a wet triangle holding both ends); max and min
      // are exact, so the bounds equal the per-element ones below.
      const cix on = (cix)n * S + k;
      R lv[NTMAX];
      il_load<NT>(a.lo[0], on, lv);
      for (int t = 0; t < NT; t++) {
        const R l = lv[t], tt = ldT(a.T[t], on, a.off[t]);
        tmx[t] = fmax2(l, tt);
        tmn[t] = fmin2(l, tt);
      }
#pragma unroll 4
    for (int p = inc.nep[j] - inc.sub, pe = inc.nep[j + 1] - inc.sub; p < pe; p++) {
        const int4 q = inc.ne[p];
        if (nz > q.z) continue;
        const cix o = (cix)q.w + k;
        il_load<NT>(a.lo[0], o, lv);
        for (int t = 0; t < NT; t++) {
          const R l = lv[t], tt = ldT(a.T[t], o, a.off[t]);
          tmx[t] = fmax2(tmx[t], fmax2(l, tt));
          tmn[t] = fmin2(tmn[t], fmin2(l, tt));
        }
      }
      if (nz > m.nlev_node_min[n] - 1) {  // a ring element is dry here: +-big enter the bounds
        for (int t = 0; t < NT; t++) {
          tmx[t] = fmax2(tmx[t], -big);
          tmn[t] = fmin2(tmn[t], big);
        }
      }
      for (int t = 0; t < NT; t++) {
        s_mx[t * kMaxCellsPerBlock + lc] = tmx[t];
        s_mn[t * kMaxCellsPerBlock + lc] = tmn[t];
      }
      continue;
    }
    for (int p = m.ring_ptr[n]; p < m.ring_ptr[n + 1]; p++) {
      const int el = m.ring_elem[p];
      const bool wet = nz <= m.nlev_elem[el] - 1;
      int e0 = 0, e1 = 0, e2 = 0;
      if (wet) {
        const int *en = m.elem_nodes + 3 * el;
        e0 = en[0]; e1 = en[1]; e2 = en[2];
      }
      for (int t = 0; t < NT; t++) {
        R amx, amn;
        if (wet) {
          const cix o0 = (cix)e0 * S + k, o1 = (cix)e1 * S + k, o2 = (cix)e2 * S + k;
          const R l0 = il<NT>(a.lo, t, o0), l1 = il<NT>(a.lo, t, o1), l2 = il<NT>(a.lo, t, o2);
          const R t0 = ldT(a.T[t], o0, a.off[t]), t1 = ldT(a.T[t], o1, a.off[t]), t2 = ldT(a.T[t], o2, a.off[t]);
          amx = fmax3(fmax2(l0, t0), fmax2(l1, t1), fmax2(l2, t2));
          amn = fmin3(fmin2(l0, t0), fmin2(l1, t1), fmin2(l2, t2));
        } else {
          amx = -big;
          amn = big;
        }
        if (p == m.ring_ptr[n]) { tmx[t] = amx; tmn[t] = amn; }
        else { tmx[t] = fmax2(tmx[t], amx); tmn[t] = fmin2(tmn[t], amn); }
      }
    }
    for (int t = 0; t < NT; t++) {
      s_mx[t * kMaxCellsPerBlock + lc] = tmx[t];
      s_mn[t * kMaxCellsPerBlock + lc] = tmn[t];
    }
  }
  __syncthreads();

  const R eps = R((double)1e-16f);  // real(MP) :: flux_eps = 1e-16 (default-real literal)
  for (int lc = threadIdx.x; lc < cm.nc; lc += blockDim.x) {
    const int j = s_item[lc], n = cm.i0 + j, k = lc - (s_off[j] - cm.c0), nz = k + 1;
    const cix col = (cix)n * S, o = col + k;
    const int nl1 = m.nlev_node[n];
    const bool edge_lev = (nz == 1 || nz == nl1 - 1);
    R fp[NTMAX], fm[NTMAX];
    {
      R v0[NTMAX], v1[NTMAX];  // interfaces k and k + 1 of every tracer
      il_load<NT>(a.adf_v[0], o, v0);
      il_load<NT>(a.adf_v[0], o + 1, v1);
      for (int t = 0; t < NT; t++) {
        fp[t] = R(0) + (fmax2(R(0), v0[t]) + fmax2(R(0), -v1[t]));
        fm[t] = R(0) + (fmin2(R(0), v0[t]) + fmin2(R(0), -v1[t]));
      }
    }
#pragma unroll 4
    for (int p = inc.nep[j] - inc.sub, pe = inc.nep[j + 1] - inc.sub; p < pe; p++) {
      const int4 q = inc.ne[p];
      if (nz > q.z) continue;
      R fv[NTMAX];
      il_load<NT>(a.adf_h[0], (cix)(q.x >> 1) * S + k, fv);
      for (int t = 0; t < NT; t++) {
        const R f = fv[t];
        if (q.x & 1) {
          fp[t] = fp[t] + fmax2(R(0), -f);
          fm[t] = fm[t] + fmin2(R(0), -f);
        } else {
          fp[t] = fp[t] + fmax2(R(0), f);
          fm[t] = fm[t] + fmin2(R(0), f);
        }
      }
    }
    const R asv = m.areasvol[o];
    const R yasv = m.rcp[o];  // 1/areasvol plane (k_rcp_planes)
    for (int t = 0; t < NT; t++) {
      const int b = t * kMaxCellsPerBlock + lc;
      const R LO = il<NT>(a.lo, t, o);
      R bmax, bmin;
      if (edge_lev) {
        bmax = s_mx[b] - LO;
        bmin = s_mn[b] - LO;
      } else {
        bmax = fmax3(s_mx[b - 1], s_mx[b], s_mx[b + 1]) - LO;
        bmin = fmin3(s_mn[b - 1], s_mn[b], s_mn[b + 1]) - LO;
      }
      if constexpr (sizeof(R) == 8) {
        // two scalar stores into the pair: R+ leaves the registers before R- is formed
        R flux = div_rcp(fp[t] * a.dt, asv, yasv) + eps;
        a.rpm[t][2 * o] = fmin2(R(1), bmax / flux);
        flux = div_rcp(fm[t] * a.dt, asv, yasv) - eps;
        a.rpm[t][2 * o + 1] = fmin2(R(1), bmin / flux);
      } else {
        // FP32 arithmetic: the ratio denominators, where cancellation with
        // flux_eps matters, are formed and divided in FP64
        const double e64 = (double)1e-16f, dt64 = (double)a.dt, asv64 = (double)asv;
        double flux = (double)fp[t] * dt64 / asv64 + e64;
        a.rpm[t][2 * o] = (R)fmin2(1.0, (double)bmax / flux);
        flux = (double)fm[t] * dt64 / asv64 - e64;
        a.rpm[t][2 * o + 1] = (R)fmin2(1.0, (double)bmin / flux);
      }
    }
  }
}

template <typename R, typename TS, int NT>
__global__ void __launch_bounds__(kThreads, MinBlocks<R>::col2) k_col2(DMeshT<R> m, FusedArgs<R, TS> a) {
  extern __shared__ int smem[];
  col2_block<R, TS, NT>(m, a, blockIdx.x, smem);
}

// limited vertical flux at interface i (lib/oce_adv_tra_fct.F90:396-427);
// av: the tracer's slot of the column's interleaved interface fluxes (stride
// NT); rpm: the column's (R+, R-) pairs
template <int NT, typename R>
__device__ __forceinline__ R limit_v(const R *av, const R *rpm, int i, int nlev) {
  const R f = av[(i - 1) * NT];
  if (i == nlev) return f;
  R ae = R(1);
  if (i == 1) {
    ae = (f >= R(0)) ? fmin2(ae, rpm[0]) : fmin2(ae, rpm[1]);
  } else if (f >= R(0)) {
    ae = fmin2(ae, rpm[2 * (i - 2) + 1]);
    ae = fmin2(ae, rpm[2 * (i - 1)]);
  } else {
    ae = fmin2(ae, rpm[2 * (i - 2)]);
    ae = fmin2(ae, rpm[2 * (i - 1) + 1]);
  }
  return ae * f;
}

// ---------------------------------------------------------------------------
// k_col3: limiting + flux2dtracer + update
// ---------------------------------------------------------------------------
// Reciprocals of the static cell geometry, 1/areasvol and 1/hnode_new, for
// the Markstein divisions of k_col1's LO solution, k_col2's ratio
// denominators and k_col3's update (computed per step they cost an IEEE
// division each; measured in k_col3: loading them is 2-3 % faster, while
// the same for k_col1's ten PPM weights was slower).
template <typename R>
__global__ void k_rcp_planes(DMeshT<R> m, R *rcp) {
  const size_t plane = (size_t)m.S * m.N;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < plane; q += (size_t)gridDim.x * blockDim.x) {
    const int n = (int)(q / m.S), k = (int)(q - (size_t)n * m.S);
    if (k >= m.nlev_node[n] - 1) continue;  // dry cells stay zero
    rcp[q] = R(1) / m.areasvol[q];
    rcp[plane + q] = R(1) / m.hnode_new[q];
  }
}

template <typename R, typename TS, int NT, int LIM>
__device__ __forceinline__ void col3_block(const DMeshT<R> &m, const FusedArgs<R, TS> &a, int blk, int *smem) {
  int *s_off = smem, *s_item = smem + kMaxItemsPerBlock + 1;
  const CellMap cm = map_cells(m.node_sched, blk, s_off, s_item);
  const Incidence inc = stage_incidence<StageIncidence<R>::col3>(m, cm, smem + kMaxItemsPerBlock + 1 + kMaxCellsPerBlock + 1);
  const int S = m.S;
  for (int lc = threadIdx.x; lc < cm.nc; lc += blockDim.x) {
    const int j = s_item[lc], n = cm.i0 + j, k = lc - (s_off[j] - cm.c0), nz = k + 1;
    const cix col = (cix)n * S, o = col + k;
    const int nlev = m.nlev_node[n];
    const R asv = m.areasvol[o], hn = m.hnode_new[o];
    const R yasv = m.rcp[o], yhn = m.rcp[m.rcp_plane + o];
    R dv[NTMAX], dh[NTMAX];
    for (int t = 0; t < NT; t++) {
      const R *av = a.adf_v[t] + (size_t)col * NT;
      dv[t] = R(0);
      if (LIM == LIM_FCT) {
        dv[t] = dv[t] - ldT(a.T[t], o, a.off[t]) * m.hnode[o] + il<NT>(a.lo, t, o) * hn;
        const R fk = limit_v<NT>(av, a.rpm[t] + 2 * col, nz, nlev);
        const R fk1 = limit_v<NT>(av, a.rpm[t] + 2 * col, nz + 1, nlev);
        dv[t] = dv[t] + div_rcp((fk - fk1) * a.dt, asv, yasv);
      } else {
        dv[t] = dv[t] + div_rcp((av[k * NT] - av[(k + 1) * NT]) * a.dt, asv, yasv);
      }
      dh[t] = R(0);
    }
    R rps[NTMAX], rms[NTMAX];
    if (LIM == LIM_FCT)
      for (int t = 0; t < NT; t++) {
        ld_pair(a.rpm[t] + 2 * o, rps[t], rms[t]);
      }
#pragma unroll 4
    for (int p = inc.nep[j] - inc.sub, pe = inc.nep[j + 1] - inc.sub; p < pe; p++) {
      const int4 q = inc.ne[p];
      if (nz > q.z) continue;
      const bool second = q.x & 1;
      const cix oo = (cix)q.w + k;  // the edge's other node (column base in .w)
      R fv[NTMAX];
      il_load<NT>(a.adf_h[0], (cix)(q.x >> 1) * S + k, fv);
      for (int t = 0; t < NT; t++) {
        R f = fv[t];
        if (LIM == LIM_FCT) {
          // r+/- at the edge's first (o1) and second (o2) node
          R rpo, rmo;
          ld_pair(a.rpm[t] + 2 * oo, rpo, rmo);
          const R rp1 = second ? rpo : rps[t], rm1 = second ? rmo : rms[t];
          const R rp2 = second ? rps[t] : rpo, rm2 = second ? rms[t] : rmo;
          R ae = R(1);
          if (f >= R(0)) {
            ae = fmin2(ae, rp1);
            ae = fmin2(ae, rm2);
          } else {
            ae = fmin2(ae, rm1);
            ae = fmin2(ae, rp2);
          }
          f = ae * f;
        }
        const R term = div_rcp(f * a.dt, asv, yasv);
        dh[t] = second ? dh[t] - term : dh[t] + term;
      }
    }
    for (int t = 0; t < NT; t++) {
      const R del = R(0) + dh[t] + dv[t];
      const R tnew = ldT(a.T[t], o, a.off[t]) + div_rcp(del, hn, yhn);
      a.T_out[t][o] = stT<R, TS>(tnew, a.off[t], a.sround != 0, a.sround ? mix32(a.seed[t] ^ mix32((uint32_t)o)) : 0u);
      if (a.nonfinite && !isfinite(tnew)) atomicAdd(a.nonfinite, 1ull);
    }
  }
}

template <typename R, typename TS, int NT, int LIM>
__global__ void __launch_bounds__(kThreads, MinBlocks<R>::col3) k_col3(DMeshT<R> m, FusedArgs<R, TS> a) {
  extern __shared__ int smem[];
  col3_block<R, TS, NT, LIM>(m, a, blockIdx.x, smem);
}

// dynamic shared memory of each kernel
constexpr size_t smem_edge() { return sizeof(int) * (kMaxItemsPerBlock + 1 + kMaxCellsPerBlock + 1); }
template <typename R>
constexpr size_t smem_col(int nt, int arrays) {
  return sizeof(int) * (kMaxItemsPerBlock + 1 + kMaxCellsPerBlock + 1) + 16 + sizeof(R) * (size_t)arrays * nt * kMaxCellsPerBlock;
}
// k_col2 / k_col3: their arrays plus the staged incidence records
template <typename R>
constexpr size_t smem_col_staged(int nt, int arrays) {
  return smem_col<R>(nt, arrays) + smem_stage();
}

FESOM_VARIANT_END
}  // namespace fesom
