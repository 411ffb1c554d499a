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
// y face and the y flux of the face below the row being finished.
struct WarpWindow {
  double P[3][NV][32];
  double lo[NV][32];
  double G[NV][32];
};
constexpr int STAGE_WARPS = 4;
#ifndef STAGE_MIN_CTAS
#define STAGE_MIN_CTAS 3   // CTAs per SM the register budget is sized for (168 registers)
#endif

template <int HEUN, int LIM>
__device__ __forceinline__ void stage_item(const StageArgs& a, const Work w, const int lane,
                                           WarpWindow& win) {
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
  const bool ylane = lane >= 2 && lane <= 29;        // owners of this strip's y faces
  const double dtdx = dt / B.dx, dtdy = dt / B.dy;
  const Recip rdx(B.dx), rdy(B.dy);   // dx, dy in the safe range (checked at creation)
  const double hdx = 0.5 * B.dx, hdy = 0.5 * B.dy;
  double lamx = 0.0, lamy = 0.0, prod = 0.0;
  bool nonfinite = false;

  // The march: iteration r forms the primitives of row r, the y slope of row r-1
  // and the y face (r-2 | r-1), then finishes row J = r-2 (x face, update).
  const int rs = w.J0 >= 2 ? w.J0 - 2 : w.J0 - 1;
  int s0 = rs % 3;                 // window slot of row r
  for (int r = rs; r <= w.J1 + 1; r++) {
    const int sm1 = s0 == 0 ? 2 : s0 - 1, sm2 = sm1 == 0 ? 2 : sm1 - 1;
    // (a) projected primitives of row r: Aux.Prim (src/Main.c:314-336)
    {
      double U[NV], Q[NV];
      const bool ok = col_in && r >= 0 && r < nyp;
      if (ok) load_cell(in, plane, (long long)r * pitch + C + 1, U);
      else benign(U);
      primitive(U, Q);
      if (ok && col_cell && r >= 1 && r <= nyp - 2) {
        const double c = relax_cfl<2 * HEUN>(Q, dt, Kn);
        if (c > prod) prod = c;
      }
      if (!(col_ring || r == 0 || r == nyp - 1)) {
        double V[NV];
        relax<2 * HEUN + 1>(Q, V, dt, Kn, Fx);
        primitive(V, Q);
      }
#pragma unroll
      for (int n = 0; n < NV; n++) win.P[s0][n][lane] = Q[n];
    }
    // (b) y slope of row r-1 (src/Main.c:348-349) and the y face (r-2 | r-1)
    double G[NV];
    const bool face_now = r >= rs + 3;
    if (r >= rs + 2) {
      double hi[NV], S[NV];
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
    if (J >= w.J0 && J < w.J1) {
      double P0[NV], Sx[NV], lo[NV], hi[NV], F[NV];
      bool xbad = false;
#pragma unroll
      for (int n = 0; n < NV; n++) {
        P0[n] = win.P[sm2][n][lane];
        const double pl = __shfl_up_sync(0xffffffffu, P0[n], 1);
        const double pr = __shfl_down_sync(0xffffffffu, P0[n], 1);
        const double L = limit<LIM>(P0[n] - pl, pr - P0[n]);
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
          v += dtdy * win.G[n][lane];
          v -= dtdy * G[n];
          v -= dtdx * F[n];
          if (HEUN == 1) v = 0.5 * v;
          out[n * plane + idx] = v;
          nonfinite |= (__double2hiint(v) & 0x7ff00000) == 0x7ff00000;
        }
      }
    }
    if (face_now && ylane) {
#pragma unroll
      for (int n = 0; n < NV; n++) win.G[n][lane] = G[n];
    }
    s0 = s0 == 2 ? 0 : s0 + 1;
  }

  // per-block maxima; the values are >= 0 (or NaN, which never passes a '>' test
  // above), so their bit patterns order like the values
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lamx = fmax(lamx, __shfl_xor_sync(0xffffffffu, lamx, o));
    lamy = fmax(lamy, __shfl_xor_sync(0xffffffffu, lamy, o));
    prod = fmax(prod, __shfl_xor_sync(0xffffffffu, prod, o));
  }
  // failure detection: a NaN or infinity in a written cell marks the case
  if (__any_sync(0xffffffffu, nonfinite) && lane == 0) atomicOr(&a.cases[B.case_id].nonfinite, 1);
  if (lane == 0) {
    unsigned long long* slot = a.lam + ((size_t)w.blk * 2 + HEUN) * 3;
    if (lamx > 0.0) atomicMax(slot + 0, (unsigned long long)__double_as_longlong(lamx));
    if (lamy > 0.0) atomicMax(slot + 1, (unsigned long long)__double_as_longlong(lamy));
    if (prod > 0.0) atomicMax(slot + 2, (unsigned long long)__double_as_longlong(prod));
  }
}

// Persistent grid (as many CTAs as fit on the SMs); every warp takes the next work
// item from a counter until the table is exhausted, so uneven blocks and the last
// wave balance themselves.
template <int HEUN, int LIM>
__global__ void __launch_bounds__(32 * STAGE_WARPS, STAGE_MIN_CTAS) stage_kernel(const StageArgs a) {
  __shared__ WarpWindow win[STAGE_WARPS];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (;;) {
    int w = 0;
    if (lane == 0) w = atomicAdd(a.queue, 1);
    w = __shfl_sync(0xffffffffu, w, 0);
    if (w >= a.nwork) break;
    stage_item<HEUN, LIM>(a, a.work[w], lane, win[warp]);
  }
}

int stage_ctas_per_sm() {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, stage_kernel<1, 4>, 32 * STAGE_WARPS, 0);
  return n > 0 ? n : 1;
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
                               unsigned long long* lam, double* trace, int* queues,
                               cudaGraphConditionalHandle h, int use_handle) {
  if (threadIdx.x < 10) queues[threadIdx.x] = 0;  // work counters [stage][limiter]
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
    if (cs.nonfinite) {       // a stage wrote a NaN or infinity: stop before accepting it
      cs.status = 2;          // MBM_ENONFINITE
      cs.done = 1;
    } else if (cfl > cs.CFLmax) {
      cs.dt = dt * cs.CFLreg / cfl;
      cs.nrej++;
    } else {
      cs.t += dt;
      double nd = dt * cs.CFLreg / cfl;
      if (cs.t + nd > cs.tend) nd = cs.tend - cs.t;
      cs.dt = nd;
      cs.nstep++;
      cs.cur = 1 - cs.cur;
      if (cs.dtlog && cs.nstep <= cs.dtlog_cap) cs.dtlog[cs.nstep - 1] = dt;   // frozen for the adjoint
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

// checkpoint of DATA after every ckpt_every-th accepted step (adjoint runs); a
// rejected attempt copies the same DATA again
__global__ void ckpt_kernel(const CaseDev* __restrict__ cases, const double* buf0, const double* buf1,
                            long long layer_elems) {
  const CaseDev& cs = cases[0];
  if (!cs.ckpt || cs.ckpt_every <= 0 || cs.nstep == 0 || cs.nstep % cs.ckpt_every) return;
  const double* src = cs.cur ? buf1 : buf0;
  double* dst = cs.ckpt + (size_t)(cs.nstep / cs.ckpt_every) * layer_elems;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < layer_elems;
       k += (long long)gridDim.x * blockDim.x)
    dst[k] = src[k];
}

cudaError_t launch_ckpt(const CaseDev* cases, const double* buf0, const double* buf1, long long layer_elems,
                        int grid, cudaStream_t s) {
  ckpt_kernel<<<grid, 256, 0, s>>>(cases, buf0, buf1, layer_elems);
  return cudaGetLastError();
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

// uniform state at rest (rho = theta = 1) in every cell of a block, for tuning runs
__global__ void fill_block_uniform(double* __restrict__ base, long long plane) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= plane) return;
  const double v[NV] = {1.0, 0.0, 0.0, 1.5, 1.0, 0.0, 1.0, 0.0, 0.0};
#pragma unroll
  for (int m = 0; m < NV; m++) base[m * plane + k] = v[m];
}

cudaError_t launch_fill_uniform(double* base, long long plane, cudaStream_t s) {
  fill_block_uniform<<<(unsigned)((plane + 255) / 256), 256, 0, s>>>(base, plane);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- output fields --
// Output's payload on the device (src/Output.c:195-243): for the interior plus one
// ghost ring, x outer / y inner, the fields rho vx vy T p Pxx Pxy Pyy qx qy of
// Primitive(U), variables fastest, as float (rounded like the reference's cast) or
// double.
__global__ void output_fields(const double* __restrict__ src, int nxp, int nyp, int pitch, long long plane,
                              int single, void* __restrict__ dst) {
  const int ni = nyp - 4, nj = nxp - 4;          // points per column (y), columns (x)
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= (long long)ni * nj) return;
  const int i = (int)(p / ni), j = (int)(p - (long long)i * ni);   // x index outer, y inner
  const int I = 2 + i, J = 2 + j;
  double U[NV], P[NV];
#pragma unroll
  for (int m = 0; m < NV; m++) U[m] = src[m * plane + (long long)J * pitch + I + 1];
  primitive(U, P);
  const double v[10] = {P[0], P[1], P[2], P[3], P[0] * P[3], P[0] * P[4],
                        P[0] * P[5], P[0] * P[6], P[7], P[8]};
  if (single) {
    float* o = (float*)dst + p * 10;
#pragma unroll
    for (int m = 0; m < 10; m++) o[m] = (float)v[m];
  } else {
    double* o = (double*)dst + p * 10;
#pragma unroll
    for (int m = 0; m < 10; m++) o[m] = v[m];
  }
}

cudaError_t launch_output_fields(const double* src, int nxp, int nyp, int pitch, long long plane, int single,
                                 void* dst, cudaStream_t s) {
  const long long n = (long long)(nyp - 4) * (nxp - 4);
  output_fields<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(src, nxp, nyp, pitch, plane, single, dst);
  return cudaGetLastError();
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
    case 0: stage_kernel<HEUN, 0><<<grid, 32 * STAGE_WARPS, 0, s>>>(a); break;
    case 1: stage_kernel<HEUN, 1><<<grid, 32 * STAGE_WARPS, 0, s>>>(a); break;
    case 2: stage_kernel<HEUN, 2><<<grid, 32 * STAGE_WARPS, 0, s>>>(a); break;
    case 3: stage_kernel<HEUN, 3><<<grid, 32 * STAGE_WARPS, 0, s>>>(a); break;
    default: stage_kernel<HEUN, 4><<<grid, 32 * STAGE_WARPS, 0, s>>>(a); break;
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
                           double* trace, int* queues, cudaGraphConditionalHandle h, int use_handle,
                           cudaStream_t s) {
  control_kernel<<<1, 256, 0, s>>>(cases, ncases, blk, lam, trace, queues, h, use_handle);
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
