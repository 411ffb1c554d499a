// mbm_stage.cuh -- the Heun stage kernel (Update, src/Main.c:297-396), compiled once per
// arithmetic mode: mbm_kernels.cu instantiates it in namespace mbm::bitwise (with
// -fmad=false), mbm_stage_fast.cu in mbm::fastmath (MBM_FAST_ARITH, -fmad=true).
//
// One warp owns a strip of 28 output columns plus a 2-column halo on each side
// (lane l <-> column I0 - 2 + l) and a segment of rows, and marches up the segment.
// Iteration r loads the moments of row r, forms its projected primitives (raw
// Primitive on the outermost ring, relaxed otherwise) into a three-row window in
// shared memory, the y slopes of row r-1 and the y-face flux between rows r-2 and
// r-1, then the x slopes and x-face states of row r-2 (the left neighbour from the
// window, the right-hand difference and face state through warp shuffles), its
// x-face fluxes and its update.  Warps are independent (no barrier); a persistent
// grid takes work items (block, strip, segment) from an atomic counter.  Every
// cell's update keeps the reference's accumulation order
//   New = ((((R + dtdx*F[i-1/2]) + dtdy*G[j-1/2]) - dtdy*G[j+1/2]) - dtdx*F[i+1/2])
// (its x-outer / y-inner face loop, src/Main.c:353-384), then *0.5 in stage 2.
// The CFL maxima cover ghost faces and cells exactly as the reference's loops do.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <type_traits>

#include "mbm_internal.h"
#include "mbm_math.cuh"

namespace mbm {
namespace MBM_ARITH {

// moments of a state at rest with rho = theta = 1: fed to lanes and rows that fall
// outside the padded grid, whose results are never used
__device__ __forceinline__ void benign(double (&U)[NV]) {
  U[0] = 1.0; U[1] = 0.0; U[2] = 0.0; U[3] = 1.5; U[4] = 1.0;
  U[5] = 0.0; U[6] = 1.0; U[7] = 0.0; U[8] = 0.0;
}

__device__ __forceinline__ void load_cell(const double* __restrict__ base, long long plane,
                                          long long idx, double (&U)[NV]) {
#pragma unroll
  for (int n = 0; n < NV; n++) U[n] = __ldg(base + n * plane + idx);
}

// Rolling state of one warp, lane fastest (conflict-free 8-byte accesses): the
// projected primitives of three consecutive rows, the lower state of the next
// y face and the y flux of the face below the row being finished.  Stage 2 adds two
// slots its asynchronous copies land in (stage 1 prefetches into registers).  Measured
// and dropped: stage 1 keeping its relaxation terms in a window ring instead of reading
// them back from global memory (neutral to 5 % slower), and stage 2 copying the update
// row's moments into a third slot (per-lane copies: 20 % slower than loading them).
struct WarpWindow1 {
  double P[3][NV][32];
  double lo[NV][32];
  double G[NV][32];
};
struct WarpWindow2 : WarpWindow1 {
  double Ua[NV][32];      // the moments of the next row
  double D0a[NV][32];     // Data0 (or its stored relaxation term) of the next update row
  // completion barriers of the bulk tensor copies into Ua and into D0a; the padding
  // keeps every slot of every warp's window on a 128-byte boundary
  unsigned long long bar[2];
  unsigned long long pad_[14];
};
static_assert(sizeof(WarpWindow2) % 128 == 0, "window slots must stay 128-byte aligned");
template <int HEUN>
using WarpWindow = typename std::conditional<HEUN == 1, WarpWindow2, WarpWindow1>::type;

// Bulk tensor copies (TMA) of the fast stage 2: one elected lane copies the nine moment
// planes of 32 columns of one row (a 32 x 1 x 9 box of a 3-D tensor map over a layer of
// one block: column, row, plane) into a window slot, completing on an mbarrier of the
// warp; each copy lands in the issuing CTA only, and the maps cover only this device's
// layers.  Every wait is bounded.
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
// one test of the phase; the thread may be suspended up to 20 us while it is incomplete
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity), "r"(20000u)
      : "memory");
  return done != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}
// false when the phase did not complete within 0.25 s of device time (a copy that never
// lands); at most 65,536 tests of at most 20 us each, should the timer not advance
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (int i = 0; i < (1 << 16); i++) {
    if (mbar_try_wait(bar, parity)) return true;
    if (global_ns() - t0 > 250000000ull) return false;
  }
  return false;
}
__device__ __forceinline__ void tma_rows(void* dst, const void* map, int x, int y, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];\n" ::"r"(smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(0), "r"(smem_u32(bar))
      : "memory");
}
// this thread's earlier shared-memory accesses ordered before later bulk copies
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
constexpr unsigned ROW_BOX_BYTES = NV * 32 * sizeof(double);   // one 32 x 1 x 9 box

// per-thread asynchronous 8-byte copy global -> shared (cp.async), and its groups
__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
#ifndef STAGE_CTA_WARPS
#define STAGE_CTA_WARPS CTA_WARPS   // warps per CTA of this instantiation
#endif
constexpr int STAGE_WARPS = STAGE_CTA_WARPS;
#ifndef STAGE_MIN_CTAS
#define STAGE_MIN_CTAS 3   // CTAs per SM the register budget is sized for (168 registers)
#endif

// One work item.  TMA (the fast stage 2 only): the instantiation that can fill its window
// slots by bulk tensor copies; tma: whether it does (warp-uniform; ph holds the phase
// bits of the warp's two window barriers across items).  The instantiation without it
// carries only the per-lane copies: the unused branches alone cost 4 % of stage 2.
// SetBoundary (src/Boundary.c:173-193) fused into the stage: once a work item's cells
// are stored, its warp writes the ghost cells whose owners the item wrote, one entry per
// lane -- the owner's value read back from the output layer, or the Dirichlet row --
// sign-flipped on the wall components as the gather does
__device__ __forceinline__ void scatter_item(const StageArgs& a, int wi, int lane, double* base,
                                             const double* out, long long plane) {
  const int2 r = a.gs_item[wi];
  if (r.y <= 0) return;
  __syncwarp();     // every lane's stores of this item are visible to the warp
  for (int e = r.x + lane; e < r.x + r.y; e += 32) {
    const GhostScatter g = a.gs[e];
    const bool fx = g.flags & 1, fy = (g.flags >> 1) & 1;
#pragma unroll
    for (int m = 0; m < NV; m++) {
      const double v = g.drow < 0 ? out[m * plane + g.src] : __ldg(a.dirichlet + (size_t)g.drow * NV + m);
      const bool flip = (fx && (m == 1 || m == 5 || m == 7)) != (fy && (m == 2 || m == 5 || m == 8));
      base[g.dst + m * g.plane] = flip ? -v : v;
    }
  }
}

// Returns false when a bounded wait on a copy ran out: the case is flagged (the
// controller stops it with a timeout status) and the warp stops taking items.
template <int HEUN, int LIM, bool TMA>
__device__ __forceinline__ bool stage_item(const StageArgs& a, const Work w, const int wi, const int lane,
                                           WarpWindow<HEUN>& win, const bool tma_on, unsigned& ph,
                                           bool& drop) {
  const bool tma = TMA && tma_on;
  const BlockDev B = a.blk[w.blk];
  const CaseDev& cs = a.cases[B.case_id];
  if (cs.done) return true;
  const int cur = cs.cur;
  const double dt = cs.dt, Fx = cs.F;
  const Recip Kn(cs.Kn);
  const double* __restrict__ in = layer_ptr(a.buf, phys_layer(a.sel_in, cur)) + B.off;
  const double* __restrict__ d0 = layer_ptr(a.buf, phys_layer(a.sel_d0, cur)) + B.off;
  double* __restrict__ out = layer_ptr(a.buf, phys_layer(a.sel_out, cur)) + B.off;
  // the relaxation term of the stage-1 input (flag -1): written by stage 1 at its row r
  // (fast arithmetic: read back, with plain loads, by the update of that row two
  // iterations later); stage 2 reads it with rlx_read in place of forming it from
  // Data0.  Null (bitwise only): not stored.
  double* __restrict__ rlx = a.rlx ? a.rlx + B.off : nullptr;
  const bool rlx_rd = HEUN == 1 && a.rlx_read;
  const double* __restrict__ d0src = rlx_rd ? rlx : d0;
  const int nxp = B.nxp, nyp = B.nyp, pitch = B.pitch;
  const long long plane = B.plane;
  const int C = w.I0 - 2 + lane;
  const bool col_in = C >= 0 && C < nxp;
  const bool col_ring = C == 0 || C == nxp - 1;
  const bool col_face = C >= 1 && C <= nxp - 3;      // face loop range (src/Main.c:353-354)
  const bool col_cell = C >= 1 && C <= nxp - 2;      // relaxation range (src/Main.c:320-321)
  const bool col_out = lane >= 2 && lane <= 29 && C >= NG && C <= nxp - 1 - NG;
  const bool ylane = lane >= 2 && lane <= 29;        // owners of this strip's y faces
  const double dtdx = dt / B.dx, dtdy = dt / B.dy;
#if !MBM_FAST_ARITH
  const Recip rdx(B.dx), rdy(B.dy);   // dx, dy in the safe range (checked at creation)
  const double hdx = 0.5 * B.dx, hdy = 0.5 * B.dy;
#endif
  double lamx = 0.0, lamy = 0.0, prod = 0.0;
  int expmax = 0;     // largest exponent field (high word & 0x7ff00000) written: all ones = NaN or inf

  // The march: iteration r forms the primitives of row r, the y slope of row r-1
  // and the y face (r-2 | r-1), then finishes row J = r-2 (x face, update).
  const int rs = w.J0 >= 2 ? w.J0 - 2 : w.J0 - 1;
  int s0 = rs % 3;                 // window slot of row r
  // Stage 1 loads the moments of row r+1 while it works on row r (nine registers,
  // which stage 2, holding Data0 as well, cannot spare without spilling).
  constexpr bool PREFETCH = HEUN == 0;
  // Stage 2 copies, without registers, the moments of row r+1 into shared memory while
  // it works on row r, and Data0 (or its relaxation term) of update row J+1 while it
  // finishes row J (= r-2):
  // one group per fetch, committed even when empty, so that the groups alternate
  // U(r), D0(r-2), U(r+1), D0(r-1), ... and each wait leaves only the newest in flight
  // bulk tensor copies: lane 0 issues each fetch after every lane has read the slot
  // (__syncwarp, then the proxy fence); a fetch of a row outside the block completes
  // its barrier phase with a plain arrive, so every fetch is matched by one wait
  const char* maps = tma ? (const char*)a.tmap + (size_t)w.blk * 2 * TMAP_BYTES : nullptr;
  const int tx0 = w.I0 - 1;        // tensor column of lane 0 (C + 1): 28 k, a multiple of 2 doubles
  bool aborted = false;
  int abort_k = -1;                // the barrier whose wait ran out
  auto bar_wait = [&](int k) {     // wait for the phase of barrier k; false: ran out
    if constexpr (HEUN == 1) {
      const bool okw = __all_sync(0xffffffffu, mbar_wait(&win.bar[k], (ph >> k) & 1u));
      ph ^= 1u << k;
      if (!okw) abort_k = k;
      return okw;
    }
    return true;
  };
  auto u_fetch = [&](int rr) {
    if constexpr (HEUN == 1) {
      if (tma) {
        __syncwarp();
        if (lane == 0) {
          fence_proxy_async();
          if (drop) {
            // failure-detection test: neither copy nor arrive, the phase never completes
          } else if (rr >= 0 && rr < nyp) {
            mbar_expect_tx(&win.bar[0], ROW_BOX_BYTES);
            tma_rows(win.Ua, maps, tx0, rr, &win.bar[0]);
          } else {
            mbar_arrive(&win.bar[0]);
          }
        }
        drop = false;
        return;
      }
      if (col_in && rr >= 0 && rr < nyp) {
        const long long idx = (long long)rr * pitch + C + 1;
#pragma unroll
        for (int n = 0; n < NV; n++) cp_async8(&win.Ua[n][lane], in + n * plane + idx);
      }
      cp_async_commit();
    }
  };
  auto d0_fetch = [&](int Jn) {
    if constexpr (HEUN == 1) {
      if (tma) {
        __syncwarp();
        if (lane == 0) {
          fence_proxy_async();
          if (Jn >= NG && Jn <= nyp - 1 - NG && Jn >= w.J0 && Jn < w.J1) {
            mbar_expect_tx(&win.bar[1], ROW_BOX_BYTES);
            tma_rows(win.D0a, maps + TMAP_BYTES, tx0, Jn, &win.bar[1]);
          } else {
            mbar_arrive(&win.bar[1]);
          }
        }
        return;
      }
      if (col_out && Jn >= NG && Jn <= nyp - 1 - NG && Jn >= w.J0 && Jn < w.J1) {
        const long long idx = (long long)Jn * pitch + C + 1;
#pragma unroll
        for (int n = 0; n < NV; n++) cp_async8(&win.D0a[n][lane], d0src + n * plane + idx);
      }
      cp_async_commit();
    }
  };
  u_fetch(rs);
  d0_fetch(rs - 2);
  double Un[NV];
  if (PREFETCH) {
    const bool ok = col_in && rs >= 0 && rs < nyp;
    if (ok) load_cell(in, plane, (long long)rs * pitch + C + 1, Un);
    else benign(Un);
  }
  for (int r = rs; r <= w.J1 + 1; r++) {
    const int sm1 = s0 == 0 ? 2 : s0 - 1, sm2 = sm1 == 0 ? 2 : sm1 - 1;
    // (a) projected primitives of row r: Aux.Prim (src/Main.c:314-336)
    {
      double U[NV], Q[NV];
      const bool ok = col_in && r >= 0 && r < nyp;
      if (PREFETCH) {
#pragma unroll
        for (int n = 0; n < NV; n++) U[n] = Un[n];
        const bool okn = col_in && r + 1 >= 0 && r + 1 < nyp;
        if (okn) load_cell(in, plane, (long long)(r + 1) * pitch + C + 1, Un);
        else benign(Un);
      } else if constexpr (HEUN == 1) {
        if (tma) {
          if (!bar_wait(0)) { aborted = true; break; }
        } else {
          cp_async_wait_one();               // this row's moments have landed
        }
        if (ok) {
#pragma unroll
          for (int n = 0; n < NV; n++) U[n] = win.Ua[n][lane];
        } else {
          benign(U);
        }
        u_fetch(r + 1);                      // into the slot just read
      }
      primitive(U, Q);
#if MBM_FAST_ARITH
      if (HEUN == 0) {
        // stage 1: one collision number and one reciprocal per damping argument serve
        // the CFL share (flag 0), the relaxation term of the update (flag -1, stored for
        // the update of this row and for stage 2) and the projection (flag 1)
        const Damp01 dm(Q[0] * fsqrt(Q[3]) * Kn.r * dt);
        if (ok && col_cell && r >= 1 && r <= nyp - 2) {
          const double c = 0.5 * (1 - dm.d2_0);
          if (c > prod) prod = c;
        }
        if (ok && col_out && r >= NG && r <= nyp - 1 - NG && r >= w.J0 && r < w.J1) {
          double R0[NV];
          relaxed_moments(Q, dm.d1_0, dm.d2_0, R0);
          const long long idx = (long long)r * pitch + C + 1;
#pragma unroll
          for (int n = 0; n < NV; n++) {
            rlx[n * plane + idx] = R0[n];
          }
        }
        if (!(col_ring || r == 0 || r == nyp - 1)) {
          const double th = Q[3];
          Q[4] = fma(dm.d1_1, Q[4] - th, th);
          Q[5] = dm.d1_1 * Q[5];
          Q[6] = fma(dm.d1_1, Q[6] - th, th);
          Q[7] = dm.d2_1 * Q[7];
          Q[8] = dm.d2_1 * Q[8];
        }
      }
#endif
#if !MBM_FAST_ARITH
      // one collision number serves every ProductionsDirect of this cell in this stage,
      // each flag's damping factors formed from it with the reference's expressions:
      // the CFL share and the update's relaxation term (flag 2 HEUN, parked in the
      // output layer until the update of this row two iterations later), stage 1's
      // relaxation of Data0 for stage 2 (flag -1: flag 0 without the force) and the
      // projection (flag 2 HEUN + 1)
      const double z = coll_of(Q, dt, Kn);
      const double d2u = rdamp<2 * HEUN>(2.0 / 3 * z);
      if (ok && col_cell && r >= 1 && r <= nyp - 2) {
        const double c = 0.5 * (1 - d2u);
        if (c > prod) prod = c;
      }
      if (ok && col_out && r >= NG && r <= nyp - 1 - NG && r >= w.J0 && r < w.J1) {
        const double d1u = rdamp<2 * HEUN>(z);
        const long long idx = (long long)r * pitch + C + 1;
        double R[NV];
        relax_d<2 * HEUN>(Q, R, dt, Fx, d1u, d2u);
#pragma unroll
        for (int n = 0; n < NV; n++) out[n * plane + idx] = R[n];
        if (HEUN == 0 && rlx) {
          relax_d<-1>(Q, R, dt, Fx, d1u, d2u);
#pragma unroll
          for (int n = 0; n < NV; n++) rlx[n * plane + idx] = R[n];
        }
      }
#endif
      if (!(col_ring || r == 0 || r == nyp - 1)) {
#if MBM_FAST_ARITH
        if (HEUN == 1) {   // stage 2 (flag 3): no CFL share (flag 2 is the identity)
          double V[NV];
          relax_prim<3>(Q, V, dt, Kn, Fx);
#pragma unroll
          for (int n = 0; n < NV; n++) Q[n] = V[n];
        }
#else
        double V[NV];
        relax_d<2 * HEUN + 1>(Q, V, dt, Fx, rdamp<2 * HEUN + 1>(z), rdamp<2 * HEUN + 1>(2.0 / 3 * z));
        primitive(V, Q);
#endif
      }
#pragma unroll
      for (int n = 0; n < NV; n++) win.P[s0][n][lane] = Q[n];
    }
    // (b) y slope of row r-1 (src/Main.c:348-349) and the y face (r-2 | r-1)
    double G[NV];
    const bool face_now = r >= rs + 3;
    if (r >= rs + 2) {
      double hi[NV], S[NV];
#if MBM_FAST_ARITH
      // the face states P -+ (dy/2) (L/dy) are P -+ L/2: dy cancels
#pragma unroll
      for (int n = 0; n < NV; n++) {
        const double pm = win.P[sm2][n][lane], p0 = win.P[sm1][n][lane], pp = win.P[s0][n][lane];
        S[n] = limit<LIM>(p0 - pm, pp - p0);
      }
#pragma unroll
      for (int n = 0; n < NV; n++) {
        const double p0 = win.P[sm1][n][lane];
        hi[n] = fma(-0.5, S[n], p0);
        G[n] = fma(0.5, S[n], p0);            // lower state of the next face, parked in G
      }
#else
      bool sbad = false;
#pragma unroll
      for (int n = 0; n < NV; n++) {
        const double pm = win.P[sm2][n][lane], p0 = win.P[sm1][n][lane], pp = win.P[s0][n][lane];
        const double L = limit<LIM>(p0 - pm, pp - p0);
        sbad |= !mk_in(L);
        S[n] = mk_div(L, rdy.y, rdy.r);
      }
      if (__builtin_expect(sbad, 0)) {
#pragma unroll
        for (int n = 0; n < NV; n++) {
          const double pm = win.P[sm2][n][lane], p0 = win.P[sm1][n][lane], pp = win.P[s0][n][lane];
          S[n] = div_ieee(limit<LIM>(p0 - pm, pp - p0), rdy.y);
        }
      }
#pragma unroll
      for (int n = 0; n < NV; n++) {
        const double p0 = win.P[sm1][n][lane];
        hi[n] = p0 - hdy * S[n];
        G[n] = p0 + hdy * S[n];               // lower state of the next face, parked in G
      }
#endif
      if (face_now && ylane) {
        double lo[NV];
#pragma unroll
        for (int n = 0; n < NV; n++) {
          lo[n] = win.lo[n][lane];
          win.lo[n][lane] = G[n];
        }
        const double lam = hll<2>(lo, hi, G);
        const int J = r - 2;
        if (col_face && J >= 1 && J <= nyp - 3 && lam > lamy) lamy = lam;
      } else {
#pragma unroll
        for (int n = 0; n < NV; n++) win.lo[n][lane] = G[n];
      }
    }
    // (c) row J = r-2: x slope, x face C | C+1 (src/Main.c:346-347, 372-378), update
    const int J = r - 2;
    if (HEUN == 1) {                        // this row's Data0 and moments have landed
      if (tma) {
        if (!bar_wait(1)) { aborted = true; break; }
      } else {
        cp_async_wait_one();
      }
    }
    if (J >= w.J0 && J < w.J1) {
      double P0[NV], Sx[NV], lo[NV], hi[NV], F[NV];
      __syncwarp();   // the window row is read across lanes below (other lanes wrote it)
      // the right-hand difference of a lane is its right neighbour's left-hand one (the
      // same subtraction of the same operands), passed down instead of recomputed
#if MBM_FAST_ARITH
#pragma unroll
      for (int n = 0; n < NV; n++) {
        P0[n] = win.P[sm2][n][lane];
        const double d1 = P0[n] - win.P[sm2][n][(lane + 31) & 31];   // left neighbour (lane 0: unused)
        Sx[n] = limit<LIM>(d1, __shfl_down_sync(0xffffffffu, d1, 1));
      }
#pragma unroll
      for (int n = 0; n < NV; n++) {        // P -+ L/2, as for the y faces
        lo[n] = fma(0.5, Sx[n], P0[n]);
        hi[n] = __shfl_down_sync(0xffffffffu, fma(-0.5, Sx[n], P0[n]), 1);
      }
#else
      bool xbad = false;
#pragma unroll
      for (int n = 0; n < NV; n++) {
        P0[n] = win.P[sm2][n][lane];
        const double d1 = P0[n] - win.P[sm2][n][(lane + 31) & 31];   // left neighbour (lane 0: unused)
        const double L = limit<LIM>(d1, __shfl_down_sync(0xffffffffu, d1, 1));
        xbad |= !mk_in(L);
        Sx[n] = mk_div(L, rdx.y, rdx.r);
      }
      if (__builtin_expect(__any_sync(0xffffffffu, xbad), 0)) {   // warp-uniform cold path
#pragma unroll
        for (int n = 0; n < NV; n++) {
          const double pl = __shfl_up_sync(0xffffffffu, P0[n], 1);
          const double pr = __shfl_down_sync(0xffffffffu, P0[n], 1);
          Sx[n] = div_ieee(limit<LIM>(P0[n] - pl, pr - P0[n]), rdx.y);
        }
      }
#pragma unroll
      for (int n = 0; n < NV; n++) {
        lo[n] = P0[n] + hdx * Sx[n];
        hi[n] = __shfl_down_sync(0xffffffffu, P0[n] - hdx * Sx[n], 1);
      }
#endif
#pragma unroll
      for (int n = 0; n < NV; n++) F[n] = 0.0;
      if (lane >= 1 && lane <= 29) {
        const double lam = hll<1>(lo, hi, F);
        if (col_face && J >= 1 && J <= nyp - 3 && lam > lamx) lamx = lam;
      }
      double Fm[NV];
#pragma unroll
      for (int n = 0; n < NV; n++) Fm[n] = __shfl_up_sync(0xffffffffu, F[n], 1);
      // cell update of row J (src/Main.c:323-331, 367-393)
      if (col_out && J >= NG && J <= nyp - 1 - NG) {
        const long long idx = (long long)J * pitch + C + 1;
        double U[NV], Q[NV], R[NV];
#if MBM_FAST_ARITH
        const double g = dt * Fx;
        if constexpr (HEUN == 1) {
          load_cell(in, plane, idx, U);
        } else {
#pragma unroll
          for (int n = 0; n < NV; n++) U[n] = rlx[n * plane + idx];   // relax<-1> of this cell
        }
        // stage 1: relax<0> = the force push of relax<-1>; stage 2: relax<2> = the force
        // push of the moments (both the identity without a force)
        if (g != 0.0) {
          push_moments(U, g, R);
        } else {
#pragma unroll
          for (int n = 0; n < NV; n++) R[n] = U[n];
        }
#else
        // relax<2 HEUN> of this cell, parked here by the window pass (plain loads)
#pragma unroll
        for (int n = 0; n < NV; n++) R[n] = out[n * plane + idx];
#endif
        if constexpr (HEUN == 1) {
          double R0[NV];
#pragma unroll
          for (int n = 0; n < NV; n++) U[n] = win.D0a[n][lane];
          if (rlx_rd) {                       // relax<-1>(Data0), stored by stage 1
#pragma unroll
            for (int n = 0; n < NV; n++) R0[n] = U[n];
          } else {
            primitive(U, Q);
            relax<-1>(Q, R0, dt, Kn, Fx);
          }
#pragma unroll
          for (int n = 0; n < NV; n++) R[n] += R0[n];
        }
#pragma unroll
        for (int n = 0; n < NV; n++) {
          double v = R[n];
          v += dtdx * Fm[n];
          v += dtdy * win.G[n][lane];
          v -= dtdy * G[n];
          v -= dtdx * F[n];
          if (HEUN == 1) v = 0.5 * v;
          out[n * plane + idx] = v;
          expmax = max(expmax, __double2hiint(v) & 0x7ff00000);
        }
      }
    }
    if (face_now && ylane) {
#pragma unroll
      for (int n = 0; n < NV; n++) win.G[n][lane] = G[n];
    }
    d0_fetch(r - 1);                        // the next update row, into the slot row J has left
    s0 = s0 == 2 ? 0 : s0 + 1;
  }
  if constexpr (HEUN == 1) {                // nothing in flight past the work item
    if (tma) {
      if (aborted) {
        // a copy did not land within the bound: flag the case, give the copies still in
        // flight one more bounded wait (the phase that ran out, and the one fetch
        // pending on the other barrier), and stop taking items
        if (lane == 0) atomicOr(&a.cases[B.case_id].nonfinite, 2);
        for (int k = 0; k < 2; k++) {
          const unsigned par = (ph >> k) & 1u;
          mbar_wait(&win.bar[k], k == abort_k ? par ^ 1u : par);
        }
        return false;
      }
      if (!bar_wait(0) || !bar_wait(1)) {
        if (lane == 0) atomicOr(&a.cases[B.case_id].nonfinite, 2);
        return false;
      }
    } else {
      cp_async_wait_all();
    }
  }
  if (a.gs_item) scatter_item(a, wi, lane, out - B.off, out, plane);

  // per-block maxima; the values are >= 0 (or NaN, which never passes a '>' test
  // above), so their bit patterns order like the values
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lamx = fmax(lamx, __shfl_xor_sync(0xffffffffu, lamx, o));
    lamy = fmax(lamy, __shfl_xor_sync(0xffffffffu, lamy, o));
    prod = fmax(prod, __shfl_xor_sync(0xffffffffu, prod, o));
  }
  // failure detection: a NaN or infinity in a written cell marks the case
  if (__any_sync(0xffffffffu, expmax == 0x7ff00000) && lane == 0) atomicOr(&a.cases[B.case_id].nonfinite, 1);
  if (lane == 0) {
    unsigned long long* slot = a.lam + ((size_t)w.blk * 2 + HEUN) * 3;
    if (lamx > 0.0) atomicMax(slot + 0, (unsigned long long)__double_as_longlong(lamx));
    if (lamy > 0.0) atomicMax(slot + 1, (unsigned long long)__double_as_longlong(lamy));
    if (prod > 0.0) atomicMax(slot + 2, (unsigned long long)__double_as_longlong(prod));
  }
  return true;
}

// Persistent grid (as many CTAs as fit on the SMs); every warp takes the next work
// item from a counter until the table is exhausted, so uneven blocks and the last
// wave balance themselves.
// the windows live in dynamic shared memory (stage_smem<HEUN> bytes, above the 48 KB a
// static allocation may take)
template <int HEUN>
constexpr int stage_smem() { return (int)sizeof(WarpWindow<HEUN>) * STAGE_WARPS; }

// register budget: STAGE_MAXNREG caps the registers per thread directly (for CTAs of
// one warp, whose residency the minimum-CTA form of the bound describes poorly);
// otherwise the launch bound asks for STAGE_MIN_CTAS resident CTAs
#ifdef STAGE_MAXNREG
#define STAGE_BOUNDS __maxnreg__(STAGE_MAXNREG)
#else
#define STAGE_BOUNDS __launch_bounds__(32 * STAGE_WARPS, STAGE_MIN_CTAS)
#endif
template <int HEUN, int LIM, bool TMA>
__global__ void STAGE_BOUNDS stage_kernel(const StageArgs a) {
  pdl_enter();
  extern __shared__ __align__(128) unsigned char stage_shared[];
  WarpWindow<HEUN>* win = reinterpret_cast<WarpWindow<HEUN>*>(stage_shared);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  bool tma = false, drop = false;
  unsigned ph = 0;
#if MBM_FAST_ARITH
  if constexpr (HEUN == 1 && TMA) {
    // bulk tensor copies need 128-byte aligned slots (the window layout keeps them so
    // from an aligned base; otherwise the per-lane copies serve)
    tma = a.tmap != nullptr && (smem_u32(&win[warp]) & 127u) == 0;
    if (tma && a.tma_drop && blockIdx.x == 0 && warp == 0) {
      int d = 0;
      if (lane == 0) d = atomicExch(a.tma_drop, 0);
      drop = __shfl_sync(0xffffffffu, d, 0) != 0;
    }
    if (tma) {
      if (lane == 0) {
        mbar_init(&win[warp].bar[0]);
        mbar_init(&win[warp].bar[1]);
        fence_mbar_init();
      }
      __syncwarp();
    }
  }
#endif
  for (;;) {
    int w = 0;
    if (lane == 0) w = atomicAdd(a.queue, 1);
    w = __shfl_sync(0xffffffffu, w, 0);
    if (w >= a.nwork) break;
    if (!stage_item<HEUN, LIM, TMA>(a, a.work[w], w, lane, win[warp], tma, ph, drop)) break;
  }
}

template <int HEUN, int LIM>
static void smem_attr() {
  cudaFuncSetAttribute(stage_kernel<HEUN, LIM, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       stage_smem<HEUN>());
  if constexpr (HEUN == 1 && MBM_FAST_ARITH != 0)
    cudaFuncSetAttribute(stage_kernel<HEUN, LIM, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         stage_smem<HEUN>());
}

// called at context creation (the device current), before any launch or graph capture:
// allows the dynamic shared memory for every instantiation on this device, then asks
// how many CTAs of Heun stage `heun` fit per SM
int stage_ctas_per_sm(int heun) {
  static std::mutex mu;
  static unsigned long long done = 0;     // one bit per device ordinal < 64
  int dev = 0;
  cudaGetDevice(&dev);
  {
    std::lock_guard<std::mutex> g(mu);
    const unsigned long long bit = dev < 64 ? (1ull << dev) : 0ull;
    if (!bit || !(done & bit)) {
      smem_attr<0, 0>(); smem_attr<0, 1>(); smem_attr<0, 2>(); smem_attr<0, 3>(); smem_attr<0, 4>();
      smem_attr<1, 0>(); smem_attr<1, 1>(); smem_attr<1, 2>(); smem_attr<1, 3>(); smem_attr<1, 4>();
      done |= bit;
    }
  }
  int n = 0;
  if (heun)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, stage_kernel<1, 4, false>, 32 * STAGE_WARPS, stage_smem<1>());
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, stage_kernel<0, 4, false>, 32 * STAGE_WARPS, stage_smem<0>());
  return n > 0 ? n : 1;
}

int stage_cta_warps() { return STAGE_WARPS; }

template <int HEUN, bool TMA>
static cudaError_t launch_stage_lim(int lim, const StageArgs& a, int grid, cudaStream_t s) {
  switch (lim) {
    case 0: return launch_k(stage_kernel<HEUN, 0, TMA>, dim3(grid), dim3(32 * STAGE_WARPS), stage_smem<HEUN>(), s, a);
    case 1: return launch_k(stage_kernel<HEUN, 1, TMA>, dim3(grid), dim3(32 * STAGE_WARPS), stage_smem<HEUN>(), s, a);
    case 2: return launch_k(stage_kernel<HEUN, 2, TMA>, dim3(grid), dim3(32 * STAGE_WARPS), stage_smem<HEUN>(), s, a);
    case 3: return launch_k(stage_kernel<HEUN, 3, TMA>, dim3(grid), dim3(32 * STAGE_WARPS), stage_smem<HEUN>(), s, a);
    default: return launch_k(stage_kernel<HEUN, 4, TMA>, dim3(grid), dim3(32 * STAGE_WARPS), stage_smem<HEUN>(), s, a);
  }
}

cudaError_t launch_stage(int lim, const StageArgs& a, int grid, cudaStream_t s) {
  if (!a.heun) return launch_stage_lim<0, false>(lim, a, grid, s);
#if MBM_FAST_ARITH
  if (a.tmap) return launch_stage_lim<1, true>(lim, a, grid, s);
#endif
  return launch_stage_lim<1, false>(lim, a, grid, s);
}

}  // namespace MBM_ARITH
}  // namespace mbm
