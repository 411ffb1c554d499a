// mbm_kernels.cu -- the Heun stage kernel, the ghost-cell gather, the step
// controller and the layout transposes.
//
// Stage kernel (Update, src/Main.c:297-396).  One warp owns a strip of 28 output
// columns plus a 2-column halo on each side (lane l <-> column I0 - 2 + l) and
// marches up the block row by row.  Per row it loads the moments of row J+2,
// forms the projected primitives (raw Primitive on the outermost ring, relaxed
// otherwise), the y slopes from three rows held in registers, the x slopes and
// x-face states through warp shuffles, the two HLL fluxes, and finishes the
// update of row J.  Nothing is staged through shared memory and no barrier is
// taken: warps are independent, so latency hides across warps.  Every cell's
// update keeps the reference's accumulation order
//   New = ((((R + dtdx*F[i-1/2]) + dtdy*G[j-1/2]) - dtdy*G[j+1/2]) - dtdx*F[i+1/2])
// (its x-outer / y-inner face loop, src/Main.c:353-384), then *0.5 in stage 2.
// The CFL maxima cover ghost faces and cells exactly as the reference's loops do.
#include <cuda_runtime.h>
#include <stdint.h>

#include "mbm_internal.h"
#include "mbm_math.cuh"

namespace mbm {

__device__ __forceinline__ void shfl_up9(const double (&a)[NV], double (&b)[NV]) {
#pragma unroll
  for (int n = 0; n < NV; n++) b[n] = __shfl_up_sync(0xffffffffu, a[n], 1);
}
__device__ __forceinline__ void shfl_down9(const double (&a)[NV], double (&b)[NV]) {
#pragma unroll
  for (int n = 0; n < NV; n++) b[n] = __shfl_down_sync(0xffffffffu, a[n], 1);
}
__device__ __forceinline__ void copy9(const double (&a)[NV], double (&b)[NV]) {
#pragma unroll
  for (int n = 0; n < NV; n++) b[n] = a[n];
}

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

template <int HEUN, int LIM>
__device__ __forceinline__ void stage_item(const StageArgs& a, const Work w, const int lane) {
  const BlockDev B = a.blk[w.blk];
  const CaseDev& cs = a.cases[B.case_id];
  if (cs.done) return;
  const int cur = cs.cur;
  const double dt = cs.dt, Fx = cs.F;
  const Recip Kn(cs.Kn);
  const double* __restrict__ in = a.buf[phys_layer(a.sel_in, cur)] + B.off;
  const double* __restrict__ d0 = a.buf[phys_layer(a.sel_d0, cur)] + B.off;
  double* __restrict__ out = a.buf[phys_layer(a.sel_out, cur)] + B.off;
  const int nxp = B.nxp, nyp = B.nyp, pitch = B.pitch;
  const long long plane = B.plane;
  const int C = w.I0 - 2 + lane;
  const bool col_in = C >= 0 && C < nxp;
  const bool col_ring = C == 0 || C == nxp - 1;
  const bool col_face = C >= 1 && C <= nxp - 3;      // face loop range (src/Main.c:353-354)
  const bool col_cell = C >= 1 && C <= nxp - 2;      // relaxation range (src/Main.c:320-321)
  const bool col_out = lane >= 2 && lane <= 29 && C >= NG && C <= nxp - 1 - NG;
  const double dx = B.dx, dy = B.dy;
  const double dtdx = dt / dx, dtdy = dt / dy;
  const Recip rdx(dx), rdy(dy);
  const double hdx = 0.5 * dx, hdy = 0.5 * dy;
  double lamx = 0.0, lamy = 0.0, prod = 0.0;

  // projected primitives of cell (C, J): Aux.Prim after src/Main.c:314-336
  auto prim_at = [&](int J, double (&P)[NV]) {
    double U[NV], Q[NV];
    const bool ok = col_in && J >= 0 && J < nyp;
    if (ok) load_cell(in, plane, (long long)J * pitch + C + 1, U);
    else benign(U);
    primitive(U, Q);
    const bool ring = col_ring || J == 0 || J == nyp - 1;
    if (ok && col_cell && J >= 1 && J <= nyp - 2) {
      const double c = relax_cfl<2 * HEUN>(Q, dt, Kn);
      if (c > prod) prod = c;
    }
    if (ring) {
      copy9(Q, P);
    } else {
      double V[NV];
      relax<2 * HEUN + 1>(Q, V, dt, Kn, Fx);
      primitive(V, P);
    }
  };
  // y slope from three consecutive rows (src/Main.c:348-349)
  auto slope = [&](const double (&Pm)[NV], const double (&P0)[NV], const double (&Pp)[NV],
                   const Recip& h, double (&S)[NV]) {
#pragma unroll
    for (int n = 0; n < NV; n++) S[n] = h.div(limit<LIM>(P0[n] - Pm[n], Pp[n] - P0[n]));
  };
  // y face between rows J and J+1 (src/Main.c:359-365)
  auto yface = [&](const double (&Pb)[NV], const double (&Sb)[NV], const double (&Pt)[NV],
                   const double (&St)[NV], int J, double (&G)[NV]) {
    double lo[NV], hi[NV];
#pragma unroll
    for (int n = 0; n < NV; n++) {
      lo[n] = Pb[n] + hdy * Sb[n];
      hi[n] = Pt[n] - hdy * St[n];
    }
    const double lam = hll<2>(lo, hi, G);
    if (col_face && J >= 1 && J <= nyp - 3 && lam > lamy) lamy = lam;
  };

  double P0[NV], P1[NV], P2[NV], S0[NV], S1[NV], Gm[NV];
  const int J0 = w.J0;
  {
    double Pm[NV];
    if (J0 >= 2) {
      double Pmm[NV], Sm[NV];
      prim_at(J0 - 2, Pmm);
      prim_at(J0 - 1, Pm);
      prim_at(J0, P0);
      prim_at(J0 + 1, P1);
      slope(Pmm, Pm, P0, rdy, Sm);
      slope(Pm, P0, P1, rdy, S0);
      if (lane >= 2 && lane <= 29) yface(Pm, Sm, P0, S0, J0 - 1, Gm);
    } else {
      prim_at(J0 - 1, Pm);
      prim_at(J0, P0);
      prim_at(J0 + 1, P1);
      slope(Pm, P0, P1, rdy, S0);
#pragma unroll
      for (int n = 0; n < NV; n++) Gm[n] = 0.0;
    }
  }

  for (int J = J0; J < w.J1; J++) {
    prim_at(J + 2, P2);
    slope(P0, P1, P2, rdy, S1);
    double G[NV];
    if (lane >= 2 && lane <= 29) yface(P0, S0, P1, S1, J, G);

    // x slope and x face C | C+1 of row J (src/Main.c:346-347, 372-378)
    double Pl[NV], Pr[NV], Sx[NV], lo[NV], hi[NV], F[NV], Fm[NV];
    shfl_up9(P0, Pl);
    shfl_down9(P0, Pr);
#pragma unroll
    for (int n = 0; n < NV; n++) {
      Sx[n] = rdx.div(limit<LIM>(P0[n] - Pl[n], Pr[n] - P0[n]));
      lo[n] = P0[n] + hdx * Sx[n];
      Pl[n] = P0[n] - hdx * Sx[n];
    }
    shfl_down9(Pl, hi);
    if (lane >= 1 && lane <= 29) {
      const double lam = hll<1>(lo, hi, F);
      if (col_face && J >= 1 && J <= nyp - 3 && lam > lamx) lamx = lam;
    }
    shfl_up9(F, Fm);

    // cell update of row J (src/Main.c:323-331, 367-393)
    if (col_out && J >= NG && J <= nyp - 1 - NG) {
      const long long idx = (long long)J * pitch + C + 1;
      double U[NV], Q[NV], R[NV];
      load_cell(in, plane, idx, U);
      primitive(U, Q);
      relax<2 * HEUN>(Q, R, dt, Kn, Fx);
      if (HEUN == 1) {
        double R0[NV];
        load_cell(d0, plane, idx, U);
        primitive(U, Q);
        relax<-1>(Q, R0, dt, Kn, Fx);
#pragma unroll
        for (int n = 0; n < NV; n++) R[n] += R0[n];
      }
#pragma unroll
      for (int n = 0; n < NV; n++) {
        double v = R[n];
        v += dtdx * Fm[n];
        v += dtdy * Gm[n];
        v -= dtdy * G[n];
        v -= dtdx * F[n];
        if (HEUN == 1) v = 0.5 * v;
        out[n * plane + idx] = v;
      }
    }
    copy9(P1, P0);
    copy9(P2, P1);
    copy9(S1, S0);
    copy9(G, Gm);
  }

  // per-block maxima; the values are >= 0 (or NaN, which never passes a '>' test
  // above), so their bit patterns order like the values
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lamx = fmax(lamx, __shfl_xor_sync(0xffffffffu, lamx, o));
    lamy = fmax(lamy, __shfl_xor_sync(0xffffffffu, lamy, o));
    prod = fmax(prod, __shfl_xor_sync(0xffffffffu, prod, o));
  }
  if (lane == 0) {
    unsigned long long* slot = a.lam + ((size_t)w.blk * 2 + HEUN) * 3;
    if (lamx > 0.0) atomicMax(slot + 0, (unsigned long long)__double_as_longlong(lamx));
    if (lamy > 0.0) atomicMax(slot + 1, (unsigned long long)__double_as_longlong(lamy));
    if (prod > 0.0) atomicMax(slot + 2, (unsigned long long)__double_as_longlong(prod));
  }
}

template <int HEUN, int LIM>
__global__ void __launch_bounds__(128) stage_kernel(const StageArgs a) {
  const int lane = threadIdx.x & 31;
  const int warps = blockDim.x >> 5;
  for (int w = blockIdx.x * warps + (threadIdx.x >> 5); w < a.nwork; w += gridDim.x * warps)
    stage_item<HEUN, LIM>(a, a.work[w], lane);
}

// ---------------------------------------------------------------- ghost fill --
// SetBoundary (src/Boundary.c:173-193) as a gather: the host resolved the two
// sweeps into the final source of every ghost cell (an interior cell of some
// block, with the composed wall signs of src/Scenario.c:57-63, or a Dirichlet row).
__global__ void ghost_kernel(const BlockDev* __restrict__ blk, const CaseDev* __restrict__ cases,
                             const GhostEntry* __restrict__ map, int n, double* buf0,
                             double* buf1, double* buf2, const double* __restrict__ dirichlet,
                             int sel) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const GhostEntry e = map[i];
  const BlockDev D = blk[e.dst_blk];
  const CaseDev& cs = cases[D.case_id];
  if (cs.done) return;
  double* bufs[3] = {buf0, buf1, buf2};
  double* layer = bufs[phys_layer(sel, cs.cur)];
  double* dst = layer + D.off + e.dst;
  const int sblk = e.src_blk_flags & 0xffff;
  const bool fx = (e.src_blk_flags >> 16) & 1, fy = (e.src_blk_flags >> 17) & 1;
#pragma unroll
  for (int m = 0; m < NV; m++) {
    double v;
    if (e.src >= 0) {
      const BlockDev S = blk[sblk];
      v = layer[S.off + m * S.plane + e.src];
    } else {
      v = dirichlet[(size_t)(-(e.src + 1)) * NV + m];
    }
    const bool flip = (fx && (m == 1 || m == 5 || m == 7)) != (fy && (m == 2 || m == 5 || m == 8));
    dst[m * D.plane] = flip ? -v : v;
  }
}

// ---------------------------------------------------------------- controller --
// One Steps iteration's bookkeeping for every case (src/Main.c:196-216, 253-283):
// CFL = max over stages and blocks of dt*lx/dx + dt*ly/dy + prod; reject if
// CFL > CFLmax, else accept, swap DATA/NEW and advance t; next dt = dt*CFLreg/CFL.
__global__ void control_kernel(CaseDev* cases, int ncases, const BlockDev* __restrict__ blk,
                               unsigned long long* lam, double* trace, cudaGraphConditionalHandle h,
                               int use_handle) {
  int live = 0;
  for (int c = threadIdx.x; c < ncases; c += blockDim.x) {
    CaseDev& cs = cases[c];
    if (cs.done) continue;
    const double dt = cs.dt;
    double cfl1 = 0.0, cfl2 = 0.0;
    for (int b = cs.blk0; b < cs.blk0 + cs.nblk; b++) {
      unsigned long long* s = lam + (size_t)b * 6;
      const double dx = blk[b].dx, dy = blk[b].dy;
      const double v1 = dt * __longlong_as_double(s[0]) / dx + dt * __longlong_as_double(s[1]) / dy +
                        __longlong_as_double(s[2]);
      const double v2 = dt * __longlong_as_double(s[3]) / dx + dt * __longlong_as_double(s[4]) / dy +
                        __longlong_as_double(s[5]);
      if (v1 > cfl1) cfl1 = v1;
      if (v2 > cfl2) cfl2 = v2;
      for (int k = 0; k < 6; k++) s[k] = 0ull;
    }
    const double cfl = rmax(cfl1, rmax(cfl2, 0.0));
    cs.cfl_last = cfl;
    cs.attempts++;
    if (cfl > cs.CFLmax) {
      cs.dt = dt * cs.CFLreg / cfl;
      cs.nrej++;
    } else {
      cs.t += dt;
      double nd = dt * cs.CFLreg / cfl;
      if (cs.t + nd > cs.tend) nd = cs.tend - cs.t;
      cs.dt = nd;
      cs.nstep++;
      cs.cur = 1 - cs.cur;
      if (cs.show_every > 0 && cs.nstep % cs.show_every == 0 && cs.trace_n < MAX_TRACE) {
        double* r = trace + ((size_t)c * MAX_TRACE + cs.trace_n) * 4;
        r[0] = cs.nstep; r[1] = cfl; r[2] = cs.t; r[3] = cs.dt;
        cs.trace_n++;
      }
      if (!(cs.t < cs.tend) || (cs.step_cap > 0 && cs.nstep >= cs.step_cap)) cs.done = 1;
    }
    if (!cs.done) {
      if (!isfinite(cfl) || !isfinite(cs.dt) || !(cs.dt > 0.0)) {
        cs.status = 2;  // MBM_ENONFINITE
        cs.done = 1;
      } else if (cs.attempts >= cs.max_attempts) {
        cs.status = 5;  // MBM_ESTEPLIMIT
        cs.done = 1;
      }
    }
    if (!cs.done) live = 1;
  }
  live = __syncthreads_or(live);
  if (use_handle && threadIdx.x == 0) cudaGraphSetConditional(h, live ? 1u : 0u);
}

// CFL of one stage per block, for the single-stage entry points
__global__ void stage_cfl_kernel(const BlockDev* __restrict__ blk, int nblk, const CaseDev* cases,
                                 unsigned long long* lam, int stage, double* out) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nblk) return;
  unsigned long long* s = lam + ((size_t)b * 2 + stage) * 3;
  const double dt = cases[blk[b].case_id].dt;
  out[b] = dt * __longlong_as_double(s[0]) / blk[b].dx + dt * __longlong_as_double(s[1]) / blk[b].dy +
           __longlong_as_double(s[2]);
  s[0] = s[1] = s[2] = 0ull;
}

// ------------------------------------------------------------------ transposes --
// host layout (cells x 9, x fastest, ghosts included) <-> device planes
__global__ void aos_to_planes(const double* __restrict__ aos, double* __restrict__ dst, int nxp,
                              int nyp, int pitch, long long plane) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long ncell = (long long)nxp * nyp;
  if (k >= ncell * NV) return;
  const long long cell = k / NV;
  const int m = (int)(k - cell * NV);
  const int J = (int)(cell / nxp), I = (int)(cell - (long long)J * nxp);
  dst[m * plane + (long long)J * pitch + I + 1] = aos[k];
}

__global__ void planes_to_aos(const double* __restrict__ src, double* __restrict__ aos, int nxp,
                              int nyp, int pitch, long long plane) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long ncell = (long long)nxp * nyp;
  if (k >= ncell * NV) return;
  const long long cell = k / NV;
  const int m = (int)(k - cell * NV);
  const int J = (int)(cell / nxp), I = (int)(cell - (long long)J * nxp);
  aos[k] = src[m * plane + (long long)J * pitch + I + 1];
}

// ------------------------------------------------------------------ launchers --
template <int HEUN>
static cudaError_t launch_stage_lim(int lim, const StageArgs& a, int grid, cudaStream_t s) {
  switch (lim) {
    case 0: stage_kernel<HEUN, 0><<<grid, 128, 0, s>>>(a); break;
    case 1: stage_kernel<HEUN, 1><<<grid, 128, 0, s>>>(a); break;
    case 2: stage_kernel<HEUN, 2><<<grid, 128, 0, s>>>(a); break;
    case 3: stage_kernel<HEUN, 3><<<grid, 128, 0, s>>>(a); break;
    default: stage_kernel<HEUN, 4><<<grid, 128, 0, s>>>(a); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_stage(int lim, const StageArgs& a, int grid, cudaStream_t s) {
  return a.heun ? launch_stage_lim<1>(lim, a, grid, s) : launch_stage_lim<0>(lim, a, grid, s);
}

cudaError_t launch_ghost(const BlockDev* blk, const CaseDev* cases, const GhostEntry* map, int n,
                         double* const buf[3], const double* dirichlet, int sel, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  ghost_kernel<<<(n + 127) / 128, 128, 0, s>>>(blk, cases, map, n, buf[0], buf[1], buf[2],
                                               dirichlet, sel);
  return cudaGetLastError();
}

cudaError_t launch_control(CaseDev* cases, int ncases, const BlockDev* blk, unsigned long long* lam,
                           double* trace, cudaGraphConditionalHandle h, int use_handle,
                           cudaStream_t s) {
  control_kernel<<<1, 256, 0, s>>>(cases, ncases, blk, lam, trace, h, use_handle);
  return cudaGetLastError();
}

cudaError_t launch_stage_cfl(const BlockDev* blk, int nblk, const CaseDev* cases,
                             unsigned long long* lam, int stage, double* out, cudaStream_t s) {
  stage_cfl_kernel<<<(nblk + 127) / 128, 128, 0, s>>>(blk, nblk, cases, lam, stage, out);
  return cudaGetLastError();
}

cudaError_t launch_aos_to_planes(const double* aos, double* dst, int nxp, int nyp, int pitch,
                                 long long plane, cudaStream_t s) {
  const long long n = (long long)nxp * nyp * NV;
  aos_to_planes<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(aos, dst, nxp, nyp, pitch, plane);
  return cudaGetLastError();
}

cudaError_t launch_planes_to_aos(const double* src, double* aos, int nxp, int nyp, int pitch,
                                 long long plane, cudaStream_t s) {
  const long long n = (long long)nxp * nyp * NV;
  planes_to_aos<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(src, aos, nxp, nyp, pitch, plane);
  return cudaGetLastError();
}

}  // namespace mbm
