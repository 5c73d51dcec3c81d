// Fused tracer step: one thread block advances the owned nodes of one patch
// (tile.hpp) through the whole of do_oce_adv_tra (lib/oce_adv_tra_driver.F90:
// 23-294 with the FCT limiter of lib/oce_adv_tra_fct.F90:53-483) and writes
// only the owned new values.  Every intermediate -- element gradients, edge
// volume and antidiffusive fluxes, the low-order solution, the FCT bounds and
// ratios -- lives in registers or shared memory; the halo's intermediates are
// recomputed by the block itself.
//
// The block walks the levels from the surface down, level j per iteration,
// as a software pipeline whose stages lag behind the level being loaded by
// the reach of the vertical stencils:
//
//   P1  level j of T, T_AB (own columns: registers; ring 3: cp.async into
//       shared memory) and of the edge volume fluxes (cp.async, one level
//       ahead)
//   P2  element gradients tr_xy at level j            (MUSCL / MFCT)
//   P3  per edge at level j: low-order flux, antidiffusive flux HO - LO
//   P4  per N2 node: LO solution at level j (horizontal gather + vertical
//       upwind); per N1 node: vertical high-order flux at interface j (PPM
//       reads T_AB two levels below, held in the thread's column window)
//   P5  per N1 node: FCT bounds at level j, ratios R+/- at level j-1
//   P6  per owned node: limiting, flux2dtracer and the new value at level j-2
//
// Each thread owns one N2 column for the whole walk and keeps that column's
// vertical windows (values, PPM slopes and interface values, vertical fluxes,
// LO solutions, bounds) in registers; neighbours' values of the current
// level come from shared memory.  Every formula, its operand order and the
// order of every sum (incident edges in ascending edge id) are those of the
// five-kernel path (advect_fused.cuh), so the FP64 results are bit-identical
// to it and to the CPU oracle.
#pragma once
#include <cstdint>

#include "advect_fused.cuh"
#include "tile.hpp"

namespace fesom {
FESOM_VARIANT_BEGIN

template <typename R>
struct TileArgs {
  const R *T;      // values (S, node)
  const R *TAB;    // valuesAB (the same array when AB)
  R *T_out;
  const R *vflux;  // (S, edge slot): edge volume fluxes of the current velocity
  const R *W;      // (S, node) interfaces
  R dt, ph;
  int hor;         // HOR_UPW1 / HOR_MUSCL / HOR_MFCT
  int ver;         // VER_UPW1 / VER_PPM
  unsigned long long *nonfinite;  // count of non-finite new values (nullptr: not counted)
};

// asynchronous global -> shared copies of one element (4 or 8 bytes)
template <typename R>
__device__ __forceinline__ void cp_async_el(R *dst, const R *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  if constexpr (sizeof(R) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// FCT ratio R = min(1, b / (f dt / asv +- eps)) (lib/oce_adv_tra_fct.F90:363-374); FP32 arithmetic
// forms the denominator in FP64
template <typename R>
__device__ __forceinline__ R fct_ratio(R b, R f, R dt, R asv, R yasv, bool plus) {
  const R eps = R((double)1e-16f);  // real(MP) :: flux_eps = 1e-16 (default-real literal)
  if constexpr (sizeof(R) == 8) {
    const R flux = plus ? div_rcp(f * dt, asv, yasv) + eps : div_rcp(f * dt, asv, yasv) - eps;
    return fmin2(R(1), b / flux);
  } else {
    const double e64 = (double)1e-16f, dt64 = (double)dt, asv64 = (double)asv;
    const double flux = plus ? (double)f * dt64 / asv64 + e64 : (double)f * dt64 / asv64 - e64;
    return (R)fmin2(1.0, (double)b / flux);
  }
}

template <typename R, int LIM, bool AB>
__global__ void __launch_bounds__(kTileThreads, 1) k_tile(DMeshT<R> m, TileArgs<R> a, DTiles pl, TileLayout L) {
  extern __shared__ __align__(16) unsigned char tsmem[];
  constexpr int NTH = kTileThreads;
  const TileCounts c = pl.cnt[blockIdx.x];
  const int tid = threadIdx.x;
  const int S = m.S;
  const bool grad = a.hor != HOR_UPW1;
  const bool muscl = a.hor == HOR_MUSCL;
  const bool ppm = a.ver == VER_PPM;

  uint32_t *s_info = (uint32_t *)(tsmem + L.info);
  int *s_incp = (int *)(tsmem + L.incp);
  uint32_t *s_inc = (uint32_t *)(tsmem + L.inc);
  int *s_eslot = (int *)(tsmem + L.eslot);
  uint32_t *s_enn = (uint32_t *)(tsmem + L.enn);
  uint32_t *s_eud = (uint32_t *)(tsmem + L.eud);
  uint32_t *s_elnn = (uint32_t *)(tsmem + L.elnn);
  int *s_elg = (int *)(tsmem + L.elg);
  unsigned char *s_elv = tsmem + L.elv;
  R *sT = (R *)(tsmem + L.sT);                       // [2][max_n3]
  R *sA = AB ? sT : (R *)(tsmem + L.sA);             // [2][max_n3]
  R *sG = (R *)(tsmem + L.sG);                       // [max_el][2]
  R *sVF = (R *)(tsmem + L.sVF);                     // [2][max_e2]
  R *sLF = (R *)(tsmem + L.sLF);                     // [max_e2]
  R *sAH = (R *)(tsmem + L.sAH);                     // [kTileAH][max_e1]
  R *sLO = (R *)(tsmem + L.sLO);                     // [max_n2]
  R *sRp = (R *)(tsmem + L.sRp), *sRm = (R *)(tsmem + L.sRm);  // [kTileR][max_n1]
  const int n3s = L.n3s, e2s = L.e2s, e1s = L.e1s, n1s = L.n1s;

  // ---- stage the patch's tables ------------------------------------------
  for (int i = tid; i < c.n3; i += NTH) s_info[i] = pl.node_info[c.node_off + i];
  for (int i = tid; i <= c.n2; i += NTH) s_incp[i] = pl.inc_ptr[c.ptr_off + i];
  const int ninc = pl.inc_ptr[c.ptr_off + c.n2];
  for (int i = tid; i < ninc; i += NTH) s_inc[i] = pl.inc[c.inc_off + i];
  for (int i = tid; i < c.e2; i += NTH) {
    s_eslot[i] = pl.edge_slot[c.edge_off + i];
    s_enn[i] = pl.edge_nn[c.edge_off + i];
  }
  if (grad) {
    for (int i = tid; i < c.e1; i += NTH) s_eud[i] = pl.edge_ud[c.edge_off + i];
    for (int i = tid; i < c.nel; i += NTH) {
      const int g = pl.elem_gid[c.elem_off + i];
      s_elnn[i] = pl.elem_nn[c.elem_off + i];
      s_elg[i] = g;
      s_elv[i] = (unsigned char)m.nlev_elem[g];
    }
  }

  // ---- the thread's own column (an N2 node) and its ring-3 node --------
  const bool own = tid < c.n2;
  const bool in1 = tid < c.n1, in0 = tid < c.n0;
  int nw = 0;  // wet layers of the own column
  size_t col = 0;
  uint32_t info = 0;
  if (own) {
    col = (size_t)pl.node_gid[c.node_off + tid] * S;
    info = pl.node_info[c.node_off + tid];
    nw = (int)(info & 255u) - 1;
  }
  const int nlmin = (int)((info >> 8) & 255u);
  const bool ring_full = (info >> 24) & 1u;
  const int i3 = c.n2 + tid;
  const bool r3 = i3 < c.n3;
  int nw3 = 0;
  size_t col3 = 0;
  if (r3) {
    col3 = (size_t)pl.node_gid[c.node_off + i3] * S;
    nw3 = (int)(pl.node_info[c.node_off + i3] & 255u) - 1;
  }
  const R *Tg = a.T, *Ag = a.TAB;
  const R *HNg = m.hnode_new + col, *Hg = m.hnode + col, *Wg = a.W + col, *ARg = m.area + col;
  const R *ASg = m.areasvol + col, *YAg = m.rcp + col, *YHg = m.rcp + m.rcp_plane + col;
  const R dt = a.dt;
  const R big = R(1e3);
  const R re = R(kREarthD), sixth = R(1.0 / 6.0), two3 = R(2.0 / 3.0);

  // column windows (index = level relative to j, after the P1 shift of
  // iteration j): T(j-2..j+1) [+ T(j+2) with AB], T_AB(j-1..j+2)
  R T_m2 = 0, T_m1 = 0, T_0 = 0, T_p1 = 0, T_p2 = 0;
  R A_m1 = 0, A_0 = 0, A_p1 = 0, A_p2 = 0;
  R HN_m1 = 0, HN_0 = 0, HN_p1 = 0, HN_p2 = 0;  // hnode_new(j-1..j+2)
  R H_m1 = 0, H_0 = 0;                          // hnode(j-1..j)
  R W_0 = 0, W_p1 = 0, AR_0 = 0, AR_p1 = 0;     // W, area at interfaces j, j+1
  R AS_0 = 0, YA_0 = 0, YH_0 = 0;               // areasvol, 1/areasvol, 1/hnode_new at j
  R sl_0 = 0, sl_p1 = 0;                        // PPM slopes of layers j, j+1
  R tv_m1 = 0, tv_0 = 0, tv_p1 = 0;             // PPM interface values j-1..j+1
  R lov_0 = 0;                                  // vertical LO flux at interface j
  R av_m2 = 0, av_m1 = 0, av_0 = 0;             // vertical antidiffusive (or HO) flux at interfaces j-2..j
  R lo_m2 = 0, lo_m1 = 0, lo_0 = 0;             // LO solution at j-2..j
  R mx_m1 = 0, mx_0 = 0, mn_m1 = 0, mn_0 = 0;   // FCT bounds at j-1, j
  R mx_m2 = 0, mn_m2 = 0;

  // prime the windows: T(0), T(1) [T(2) with AB]; T_AB(0), T_AB(1); interface 0
  if (own) {
    if constexpr (AB) {
      T_p1 = nw > 0 ? Tg[col] : R(0);
      T_p2 = nw > 1 ? Tg[col + 1] : R(0);
    } else {
      T_p1 = nw > 0 ? Tg[col] : R(0);
      A_p1 = nw > 0 ? Ag[col] : R(0);
      A_p2 = nw > 1 ? Ag[col + 1] : R(0);
    }
    HN_p1 = nw > 0 ? HNg[0] : R(0);
    HN_p2 = nw > 1 ? HNg[1] : R(0);
    H_0 = nw > 0 ? Hg[0] : R(0);
    W_p1 = Wg[0];
    AR_p1 = ARg[0];
  }
  // ring-3 node and edge volume fluxes of level 0
  if (r3 && nw3 > 0) {
    cp_async_el(sT + i3, Tg + col3);
    if constexpr (!AB) cp_async_el(sA + i3, Ag + col3);
  }
  for (int e = tid; e < c.e2; e += NTH) {
    const int lev = (int)(pl.edge_nn[c.edge_off + e] >> 20);
    if (lev > 0) cp_async_el(sVF + e, a.vflux + (size_t)pl.edge_slot[c.edge_off + e] * S);
  }
  cp_async_commit();

  const int jend = c.jmax + 2;
  for (int j = 0; j < jend; j++) {
    const int cur = j & 1, nxt = cur ^ 1;
    // ---------------- P1: level j in, level j+1 requested -----------------
    // window shift
    T_m2 = T_m1; T_m1 = T_0; T_0 = T_p1;
    if constexpr (AB) {
      T_p1 = T_p2;
    } else {
      A_m1 = A_0; A_0 = A_p1; A_p1 = A_p2;
    }
    HN_m1 = HN_0; HN_0 = HN_p1; HN_p1 = HN_p2;
    H_m1 = H_0;
    W_0 = W_p1; AR_0 = AR_p1;
    if (own) {
      // level j of the own column into shared memory
      if (j < nw) {
        sT[cur * n3s + tid] = T_0;
        if constexpr (!AB) sA[cur * n3s + tid] = A_0;
      }
      // loads consumed in P4 of this iteration
      if constexpr (AB) {
        T_p2 = (j + 2 < nw) ? Tg[col + j + 2] : R(0);
      } else {
        T_p1 = (j + 1 < nw) ? Tg[col + j + 1] : R(0);
        A_p2 = (j + 2 < nw) ? Ag[col + j + 2] : R(0);
      }
      HN_p2 = (j + 2 < nw) ? HNg[j + 2] : R(0);
      H_0 = (j < nw) ? Hg[j] : R(0);
      if (j + 1 <= nw) {
        W_p1 = Wg[j + 1];
        AR_p1 = ARg[j + 1];
      }
      if (j < nw) {
        AS_0 = ASg[j];
        YA_0 = YAg[j];
        YH_0 = YHg[j];
      }
    }
    if constexpr (AB) {
      (void)A_m1; (void)A_0; (void)A_p1; (void)A_p2;
    }
    // ring-3 node and edge volume fluxes of level j+1 (cp.async into the
    // other buffer, which iteration j-1 finished reading)
    if (r3 && j + 1 < nw3) {
      cp_async_el(sT + nxt * n3s + i3, Tg + col3 + j + 1);
      if constexpr (!AB) cp_async_el(sA + nxt * n3s + i3, Ag + col3 + j + 1);
    }
    for (int e = tid; e < c.e2; e += NTH) {
      const int lev = (int)(s_enn[e] >> 20);
      if (j + 1 < lev) cp_async_el(sVF + nxt * e2s + e, a.vflux + (size_t)s_eslot[e] * S + j + 1);
    }
    cp_async_commit();
    // wait for level j's copies (issued one iteration ago)
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");
    __syncthreads();

    const R *sTc = sT + cur * n3s;
    const R *sAc = sA + cur * n3s;
    const R *sVFc = sVF + cur * e2s;
    // ---------------- P2: element gradients at level j --------------------
    if (grad) {
      for (int el = tid; el < c.nel; el += NTH) {
        if (j + 1 > (int)s_elv[el] - 1) continue;
        const uint32_t nn = s_elnn[el];
        const int na = nn & 1023u, nb = (nn >> 10) & 1023u, nc = nn >> 20;
        const R *gs = m.grad_sca + 6 * (size_t)s_elg[el];
        const R t1 = sAc[na], t2 = sAc[nb], t3 = sAc[nc];
        sG[2 * el] = (gs[0] * t1 + gs[1] * t2) + gs[2] * t3;
        sG[2 * el + 1] = (gs[3] * t1 + gs[4] * t2) + gs[5] * t3;
      }
      __syncthreads();
    }

    // ---------------- P3: edge fluxes at level j --------------------------
    R *sAHj = sAH + (j % kTileAH) * e1s;
    for (int e = tid; e < c.e2; e += NTH) {
      const uint32_t enn = s_enn[e];
      const int lev = (int)(enn >> 20);
      if (j >= lev) continue;
      const int n1 = enn & 1023u, n2 = (enn >> 10) & 1023u;
      const R vflux = sVFc[e];
      R flo = R(0);
      if (LIM == LIM_FCT) {
        flo = upw1_flux(vflux, sTc[n1], sTc[n2]);
        sLF[e] = flo;
      }
      if (e >= c.e1) continue;
      const R t1 = sAc[n1], t2 = sAc[n2];
      if (!grad) {
        sAHj[e] = upw1_flux(vflux, t1, t2) - flo;
        continue;
      }
      // edge_up_dn_grad (lib/oce_muscl_adv.F90:383-527)
      const uint32_t ud = s_eud[e];
      const int up = ud & 0xffffu, dn = ud >> 16;
      R gux, guy, gdx, gdy;
      bool shared = false;
      if (up != 0xffff && dn != 0xffff) {
        const int mn1 = (int)((s_info[n1] >> 8) & 255u), mn2 = (int)((s_info[n2] >> 8) & 255u);
        shared = (j + 1) <= min(mn1, mn2) - 1;
      }
      if (shared) {
        gux = sG[2 * up]; guy = sG[2 * up + 1];
        gdx = sG[2 * dn]; gdy = sG[2 * dn + 1];
      } else {
        // area-weighted ring means of tr_xy at both nodes (k_grad's sums)
        for (int side = 0; side < 2; side++) {
          const int nd = side ? n2 : n1;
          R tvol = R(0), tx = R(0), ty = R(0);
          const int p0 = pl.ring_ptr[c.ptr_off + nd], p1 = pl.ring_ptr[c.ptr_off + nd + 1];
          for (int p = p0; p < p1; p++) {
            const int el = pl.ring[c.ring_off + p];
            if ((int)s_elv[el] - 1 < j + 1) continue;
            const R ar = m.elem_area[s_elg[el]];
            tvol = tvol + ar;
            tx = tx + sG[2 * el] * ar;
            ty = ty + sG[2 * el + 1] * ar;
          }
          if (side) { gdx = tx / tvol; gdy = ty / tvol; }
          else { gux = tx / tvol; guy = ty / tvol; }
        }
      }
      const int slot = s_eslot[e];
      const R ex = m.edge_dxdy[2 * (size_t)slot], ey = m.edge_dxdy[2 * (size_t)slot + 1], aa = m.edge_a[slot];
      R c_lo1 = R(1), c_lo2 = R(1);
      if (muscl) {
        c_lo1 = ((int)((s_info[n1] >> 16) & 255u) - (j + 1) >= 0) ? R(1) : R(0);
        c_lo2 = ((int)((s_info[n2] >> 16) & 255u) - (j + 1) >= 0) ? R(1) : R(0);
      }
      // lib/oce_adv_tra_hor.F90:454-469 (MUSCL), :743-753 (MFCT, no c_lo)
      const R x2 = R(2) * (t2 - t1) + ex * aa * gdx + ey * re * gdy;
      const R x1 = R(2) * (t2 - t1) + ex * aa * gux + ey * re * guy;
      R Tmean2, Tmean1;
      if (muscl) {
        Tmean2 = t2 - div_rcp(x2, R(6), sixth) * c_lo2;
        Tmean1 = t1 + div_rcp(x1, R(6), sixth) * c_lo1;
      } else {
        Tmean2 = t2 - div_rcp(x2, R(6), sixth);
        Tmean1 = t1 + div_rcp(x1, R(6), sixth);
      }
      const R cHO = (vflux + fabs(vflux)) * Tmean1 + (vflux - fabs(vflux)) * Tmean2;
      const R ho = -(R(0.5) * (R(1) - a.ph) * cHO) - vflux * a.ph * R(0.5) * (Tmean1 + Tmean2);
      sAHj[e] = ho - flo;
    }
    __syncthreads();

    // ---------------- P4: LO solution (N2), vertical HO flux (N1) ---------
    if (own) {
      // vertical LO flux at interface j+1 (bottom of layer j); interface 0
      // is primed here (lib/oce_adv_tra_ver.F90:300-327)
      R lov_p1 = R(0), lo_new = R(0), hov = R(0);
      if (LIM == LIM_FCT) {
        if (j == 0 && nw > 0) lov_0 = -(W_0 * T_0 * AR_0);
        if (j + 1 < nw) {
          const R w = W_p1;
          lov_p1 = -(R(0.5) * (T_p1 * (w + fabs(w)) + T_0 * (w - fabs(w))) * AR_p1);
        }
        if (j < nw) {
          // lib/oce_adv_tra_driver.F90:122-181 (gather in ascending edge id), :202-211
          R acc = R(0);
          for (int p = s_incp[tid], pe = s_incp[tid + 1]; p < pe; p++) {
            const uint32_t q = s_inc[p];
            if (j + 1 > (int)(q >> 22)) continue;
            const R F = sLF[q & 2047u];
            acc = ((q >> 11) & 1u) ? acc - F : acc + F;
          }
          const R num = T_0 * H_0 + div_rcp((acc + (lov_0 - lov_p1)) * dt, AS_0, YA_0);
          lo_new = div_rcp(num, HN_0, YH_0);
          sLO[tid] = lo_new;
        }
      }
      lo_m2 = lo_m1; lo_m1 = lo_0; lo_0 = lo_new;
      if (in1 && j <= nw) {
        // interface j (1-based i = j + 1); with AB the T_AB window is the T one
        const R Am1 = AB ? T_m1 : A_m1, A0 = AB ? T_0 : A_0, Ap1 = AB ? T_p1 : A_p1, Ap2 = AB ? T_p2 : A_p2;
        const int nlev = nw + 1;
        if (ppm) {
          // slope of layer j+1 (lib/oce_adv_tra_ver.F90:525-540) and the
          // interface value below it (:545-594)
          const R sl_new = (j + 1 >= 1 && j + 1 <= nw - 2)
                               ? ppm_slope(A0, Ap1, Ap2, HN_p1 / (HN_0 + HN_p1 + HN_p2),
                                           (R(2) * HN_0 + HN_p1) / (HN_p2 + HN_p1), (HN_p1 + R(2) * HN_p2) / (HN_0 + HN_p1))
                               : R(0);
          R tv_new = R(0);
          const int i = j + 2;  // interface of the new value
          if (j + 1 <= nw - 1) {
            if (i == nlev - 1) {
              const R s = sgn1(W_p1);
              tv_new = -A0 * fmin2(s, R(0)) + Ap1 * fmax2(s, R(0));
            } else if (i == 2) {
              tv_new = R(0.5) * (A0 + Ap1);
            } else {
              const R dzjm1 = HN_m1, dzj = HN_0, dzjp1 = HN_p1, dzjp2 = HN_p2;
              const R Ac = dzj / (dzj + dzjp1);
              const R Bc = R(1) / (dzjm1 + dzj + dzjp1 + dzjp2);
              const R Cc = (R(2) * dzjp1 * dzj) / (dzj + dzjp1) *
                           ((dzjm1 + dzj) / (R(2) * dzj + dzjp1) - (dzjp2 + dzjp1) / (R(2) * dzjp1 + dzj));
              const R Dc = dzj * (dzjm1 + dzj) / (R(2) * dzj + dzjp1);
              const R Ec = dzjp1 * (dzjp1 + dzjp2) / (dzj + R(2) * dzjp1);
              tv_new = A0 + Ac * (Ap1 - A0) + Bc * (Cc * (Ap1 - A0) - Dc * sl_new + Ec * sl_p1);
            }
          }
          sl_0 = sl_p1;
          sl_p1 = sl_new;
          if (j == 0) tv_0 = A0;  // interface 1 takes T_AB(1) itself
          tv_m1 = tv_0;           // shift: tv(j-1), tv(j), tv(j+1)
          tv_0 = (j == 0) ? A0 : tv_p1;
          tv_p1 = tv_new;
          // flux at interface j (lib/oce_adv_tra_ver.F90:597-639)
          if (j == nw) {
            hov = R(0) - lov_0;
          } else if (j == 0) {
            hov = -(tv_0 * W_0 * AR_0) - lov_0;
          } else {
            const R w = W_0;
            if (!(w > R(0)) && !(w < R(0))) {
              hov = R(0) - lov_0;
            } else {
              const bool upw = w > R(0);      // supplying layer j (w > 0) or j-1
              const R dzj = upw ? H_0 : H_m1;
              const R x = upw ? fmin2(w * dt / dzj, R(1)) : fmin2(-(w * dt / dzj), R(1));
              const R Tc = upw ? A0 : Am1;
              R aL = upw ? tv_0 : tv_m1;
              const bool last = upw ? (j == nw - 1) : (j - 1 == nw - 1);
              R aR = last ? Tc : (upw ? tv_p1 : tv_0);
              if ((aR - Tc) * (Tc - aL) <= R(0)) { aL = Tc; aR = Tc; }
              if ((aR - aL) * (Tc - R(0.5) * (aL + aR)) > div_rcp((aR - aL) * (aR - aL), R(6), sixth)) aL = R(3) * Tc - R(2) * aR;
              if ((aR - aL) * (Tc - R(0.5) * (aR + aL)) < -div_rcp((aR - aL) * (aR - aL), R(6), sixth)) aR = R(3) * Tc - R(2) * aL;
              const R aj = R(6) * (Tc - R(0.5) * (aL + aR));
              R tt;
              if (upw) tt = (-aL - R(0.5) * x * (aR - aL + (R(1) - two3 * x) * aj));
              else tt = (-aR + R(0.5) * x * (aR - aL - (R(1) - two3 * x) * aj));
              hov = tt * AR_0 * w - lov_0;
            }
          }
        } else {
          // adv_tra_ver_upw1 of T_AB (lib/oce_adv_tra_ver.F90:300-327)
          R up;
          if (j == 0) up = -(W_0 * A0 * AR_0);
          else if (j == nw) up = R(0);
          else {
            const R w = W_0;
            up = -(R(0.5) * (A0 * (w + fabs(w)) + Am1 * (w - fabs(w))) * AR_0);
          }
          hov = up - lov_0;
        }
      }
      av_m2 = av_m1; av_m1 = av_0; av_0 = hov;
      lov_0 = lov_p1;
    }
    __syncthreads();

    // ---------------- P5: FCT bounds at j, ratios at j-1 (N1) --------------
    if (LIM == LIM_FCT && own && in1) {
      R tmx = R(0), tmn = R(0);
      if (j < nw) {
        if (ring_full) {
          // complete ring: the node and the far ends of its edges wet here
          tmx = fmax2(lo_0, T_0);
          tmn = fmin2(lo_0, T_0);
          for (int p = s_incp[tid], pe = s_incp[tid + 1]; p < pe; p++) {
            const uint32_t q = s_inc[p];
            if (j + 1 > (int)(q >> 22)) continue;
            const int o = (q >> 12) & 1023u;
            const R l = sLO[o], tt = sTc[o];
            tmx = fmax2(tmx, fmax2(l, tt));
            tmn = fmin2(tmn, fmin2(l, tt));
          }
          if (j + 1 > nlmin - 1) {
            tmx = fmax2(tmx, -big);
            tmn = fmin2(tmn, big);
          }
        } else {
          const int p0 = pl.ring_ptr[c.ptr_off + tid], p1 = pl.ring_ptr[c.ptr_off + tid + 1];
          for (int p = p0; p < p1; p++) {
            const int el = pl.ring[c.ring_off + p];
            // ring elements of an N1 node are in EL (every element with a node in N2)
            const int g = pl.elem_gid[c.elem_off + el];
            const bool wet = j + 1 <= m.nlev_elem[g] - 1;
            R amx, amn;
            if (wet) {
              const uint32_t nn = pl.elem_nn[c.elem_off + el];
              const int q0 = nn & 1023u, q1 = (nn >> 10) & 1023u, q2 = nn >> 20;
              const R l0 = sLO[q0], l1 = sLO[q1], l2 = sLO[q2];
              const R t0 = sTc[q0], t1 = sTc[q1], t2 = sTc[q2];
              amx = fmax3(fmax2(l0, t0), fmax2(l1, t1), fmax2(l2, t2));
              amn = fmin3(fmin2(l0, t0), fmin2(l1, t1), fmin2(l2, t2));
            } else {
              amx = -big;
              amn = big;
            }
            if (p == p0) { tmx = amx; tmn = amn; }
            else { tmx = fmax2(tmx, amx); tmn = fmin2(tmn, amn); }
          }
        }
      }
      mx_m2 = mx_m1; mx_m1 = mx_0; mx_0 = tmx;
      mn_m2 = mn_m1; mn_m1 = mn_0; mn_0 = tmn;
      const int k = j - 1;
      if (k >= 0 && k < nw) {
        const bool edge_lev = (k == 0 || k == nw - 1);
        const R bmax = (edge_lev ? mx_m1 : fmax3(mx_m2, mx_m1, mx_0)) - lo_m1;
        const R bmin = (edge_lev ? mn_m1 : fmin3(mn_m2, mn_m1, mn_0)) - lo_m1;
        // av_m2 / av_m1 / av_0 are interfaces j-2, j-1, j: layer k has k = j-1 and k+1 = j
        R fp = R(0) + (fmax2(R(0), av_m1) + fmax2(R(0), -av_0));
        R fm = R(0) + (fmin2(R(0), av_m1) + fmin2(R(0), -av_0));
        const R *sAHk = sAH + (k % kTileAH) * e1s;
        for (int p = s_incp[tid], pe = s_incp[tid + 1]; p < pe; p++) {
          const uint32_t q = s_inc[p];
          if (k + 1 > (int)(q >> 22)) continue;
          const R f = sAHk[q & 2047u];
          if ((q >> 11) & 1u) {
            fp = fp + fmax2(R(0), -f);
            fm = fm + fmin2(R(0), -f);
          } else {
            fp = fp + fmax2(R(0), f);
            fm = fm + fmin2(R(0), f);
          }
        }
        const R asv = ASg[k], yasv = YAg[k];
        sRp[(k % kTileR) * n1s + tid] = fct_ratio(bmax, fp, dt, asv, yasv, true);
        sRm[(k % kTileR) * n1s + tid] = fct_ratio(bmin, fm, dt, asv, yasv, false);
      }
    }
    __syncthreads();

    // ---------------- P6: new values at j-2 (owned nodes) -----------------
    if (own && in0) {
      const int k = j - 2;
      if (k >= 0 && k < nw) {
        const size_t o = col + k;
        const R asv = ASg[k], yasv = YAg[k], hn = HNg[k], yhn = YHg[k];
        // av_m2 = interface k, av_m1 = interface k+1
        R dv = R(0);
        R rps = R(0), rms = R(0);
        if (LIM == LIM_FCT) {
          const R *rp_k = sRp + (k % kTileR) * n1s, *rm_k = sRm + (k % kTileR) * n1s;
          rps = rp_k[tid];
          rms = rm_k[tid];
          dv = dv - T_m2 * Hg[k] + lo_m2 * hn;
          // limited vertical fluxes at interfaces k and k+1 (lib/oce_adv_tra_fct.F90:396-427)
          R fk = av_m2;
          {
            R ae = R(1);
            if (k == 0) {
              ae = (fk >= R(0)) ? fmin2(ae, rps) : fmin2(ae, rms);
            } else {
              const R rpu = sRp[((k - 1) % kTileR) * n1s + tid], rmu = sRm[((k - 1) % kTileR) * n1s + tid];
              if (fk >= R(0)) { ae = fmin2(ae, rmu); ae = fmin2(ae, rps); }
              else { ae = fmin2(ae, rpu); ae = fmin2(ae, rms); }
            }
            fk = ae * fk;
          }
          R fk1 = av_m1;
          if (k + 1 != nw) {
            const R rpd = sRp[((k + 1) % kTileR) * n1s + tid], rmd = sRm[((k + 1) % kTileR) * n1s + tid];
            R ae = R(1);
            if (fk1 >= R(0)) { ae = fmin2(ae, rms); ae = fmin2(ae, rpd); }
            else { ae = fmin2(ae, rps); ae = fmin2(ae, rmd); }
            fk1 = ae * fk1;
          }
          dv = dv + div_rcp((fk - fk1) * dt, asv, yasv);
        } else {
          dv = dv + div_rcp((av_m2 - av_m1) * dt, asv, yasv);
        }
        R dh = R(0);
        const R *sAHk = sAH + (k % kTileAH) * e1s;
        const R *rp_k = sRp + (k % kTileR) * n1s, *rm_k = sRm + (k % kTileR) * n1s;
        for (int p = s_incp[tid], pe = s_incp[tid + 1]; p < pe; p++) {
          const uint32_t q = s_inc[p];
          if (k + 1 > (int)(q >> 22)) continue;
          const bool second = (q >> 11) & 1u;
          R f = sAHk[q & 2047u];
          if (LIM == LIM_FCT) {
            const int oth = (q >> 12) & 1023u;
            const R rpo = rp_k[oth], rmo = rm_k[oth];
            const R rp1 = second ? rpo : rps, rm1 = second ? rmo : rms;
            const R rp2 = second ? rps : rpo, rm2 = second ? rms : rmo;
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
          const R term = div_rcp(f * dt, asv, yasv);
          dh = second ? dh - term : dh + term;
        }
        const R del = R(0) + dh + dv;
        const R tnew = T_m2 + div_rcp(del, hn, yhn);
        a.T_out[o] = tnew;
        if (a.nonfinite && !isfinite(tnew)) atomicAdd(a.nonfinite, 1ull);
      }
    }
    (void)AS_0; (void)YA_0; (void)YH_0; (void)HN_m1; (void)sl_0; (void)mn_m2;
  }
  cp_async_wait_all();
}

FESOM_VARIANT_END
}  // namespace fesom
