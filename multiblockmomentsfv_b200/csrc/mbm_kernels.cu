// mbm_kernels.cu -- the ghost-cell gather, the step controller, checkpoints,
// output staging and the layout transposes, and the bitwise instantiation of the
// Heun stage kernel (mbm_stage.cuh).
#include <cuda_runtime.h>
#include <stdint.h>

#include "mbm_internal.h"
// the bitwise kernel's unfused arithmetic needs more registers than the fast one: two
// CTAs per SM (255 registers, no spills) run it 2 % faster than three (168, spilling)
#define STAGE_MIN_CTAS 2
#include "mbm_stage.cuh"   // the stage kernel in namespace mbm::bitwise

namespace mbm {

thread_local bool tl_pdl = false;

using namespace bitwise;    // the output conversion uses the bitwise Primitive

// ---------------------------------------------------------------- ghost fill --
// SetBoundary (src/Boundary.c:173-193) as a gather: the host resolved the two
// sweeps into the final source of every ghost cell (an interior cell of some
// block, with the composed wall signs of src/Scenario.c:57-63, or a Dirichlet row).
__global__ void ghost_kernel(const BlockDev* __restrict__ blk, const CaseDev* __restrict__ cases,
                             const GhostEntry* __restrict__ map, int n, double* buf0,
                             double* buf1, double* buf2, const double* __restrict__ dirichlet,
                             const double* __restrict__ recv, int sel) {
  pdl_enter();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const GhostEntry e = map[i];
  const BlockDev D = blk[e.dst_blk];
  const CaseDev& cs = cases[D.case_id];
  if (cs.done) return;
  const int l = phys_layer(sel, cs.cur);
  double* layer = l == 0 ? buf0 : (l == 1 ? buf1 : buf2);
  double* dst = layer + D.off + e.dst;
  const int sblk = e.src_blk_flags & 0xffff;
  const bool fx = (e.src_blk_flags >> 16) & 1, fy = (e.src_blk_flags >> 17) & 1;
#pragma unroll
  for (int m = 0; m < NV; m++) {
    double v;
    if (e.src_blk_flags & GHOST_REMOTE) {          // a source cell on another rank
      v = recv[(size_t)e.src * NV + m];
    } else if (e.src >= 0) {
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
                               cudaGraphConditionalHandle h, int use_handle, const double* cfl_ext) {
  pdl_enter();
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
    // a case split over ranks brings the max over all ranks (single-case contexts)
    const double cfl = cfl_ext ? *cfl_ext : rmax(cfl1, rmax(cfl2, 0.0));
    cs.cfl_last = cfl;
    cs.attempts++;
    cs.accepted = 0;
    if (cs.nonfinite) {       // a stage wrote a NaN or infinity: stop before accepting it
      // bit 2: a bounded wait for a bulk copy ran out (MBM_ETIMEOUT), else MBM_ENONFINITE
      cs.status = (cs.nonfinite & 2) ? 3 : 2;
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
      cs.accepted = 1;
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

// a frozen-dt step's set-up (the adjoint's recomputation, mbm_replay): the step's dt
// from the device log into the case record, the work counters zeroed -- a kernel, so
// that the step's launches follow one another as kernels
__global__ void frozen_prep_kernel(CaseDev* cases, const double* __restrict__ ddt, int* queues) {
  pdl_enter();
  if (threadIdx.x == 0) cases[0].dt = *ddt;
  if (threadIdx.x < 10) queues[threadIdx.x] = 0;
}

cudaError_t launch_frozen_prep(CaseDev* cases, const double* ddt, int* queues, cudaStream_t s) {
  return launch_k(frozen_prep_kernel, dim3(1), dim3(32), 0, s, cases, ddt, queues);
}

// checkpoint of DATA after every ckpt_every-th accepted step (adjoint runs); a
// rejected attempt copies the same DATA again.  After an accepted step m inside the last
// segment [a, b) it also keeps that step's stage-1 state (TMP, still the accepted
// attempt's) and the new state D_m, so that the reverse sweep need not recompute the
// segment.
__global__ void ckpt_kernel(const CaseDev* __restrict__ cases, const double* buf0, const double* buf1,
                            const double* buf2, long long layer_elems) {
  pdl_enter();
  const CaseDev& cs = cases[0];
  const long long k0 = (long long)blockIdx.x * blockDim.x + threadIdx.x, ks = (long long)gridDim.x * blockDim.x;
  const double* data = cs.cur ? buf1 : buf0;
  if (cs.tail_d && cs.accepted) {
    const int m = cs.nstep;   // step m-1 was just accepted: T_{m-1} in TMP, D_m in DATA
    if (m - 1 >= cs.tail_a && m - 1 < cs.tail_b) {
      double* dst = cs.tail_t + (size_t)(m - 1 - cs.tail_a) * layer_elems;
      for (long long k = k0; k < layer_elems; k += ks) dst[k] = buf2[k];
    }
    if (m >= cs.tail_a && m < cs.tail_b) {
      double* dst = cs.tail_d + (size_t)(m - cs.tail_a) * layer_elems;
      for (long long k = k0; k < layer_elems; k += ks) dst[k] = data[k];
    }
  }
  if (!cs.ckpt || cs.ckpt_every <= 0 || cs.nstep == 0 || cs.nstep % cs.ckpt_every) return;
  double* dst = cs.ckpt + (size_t)(cs.nstep / cs.ckpt_every) * layer_elems;
  for (long long k = k0; k < layer_elems; k += ks) dst[k] = data[k];
}

cudaError_t launch_ckpt(const CaseDev* cases, const double* buf0, const double* buf1, const double* buf2,
                        long long layer_elems, int grid, cudaStream_t s) {
  return launch_k(ckpt_kernel, dim3(grid), dim3(256), 0, s, cases, buf0, buf1, buf2, layer_elems);
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

// ------------------------------------------------------------------ restart load --
// LoadData on the device (src/Mesh.c:198-283): one block's zone of a result file, as
// stored (the interior plus one ghost ring, x outer / y inner, the 10 fields rho vx vy T
// p Pxx Pxy Pyy qx qy fastest; float widened to double, as the reference reads a
// Float32 file), becomes the moments of L_DATA; every other cell of the block is zero, as
// the reference's main leaves it before SetBoundary.  The reference's mapping (faithful =
// 0) puts the stored p where theta belongs and P_ij where T_ij belongs (src/Mesh.c:
// 263-273); faithful = 1 maps the fields to the state they were written from
// (theta = T, T_ij = P_ij / rho).  Conservative keeps the reference's expression order
// (bitwise instantiation), so the moments equal the reference's LoadData bit for bit.
__global__ void fields_to_planes(const void* __restrict__ src, int single, int faithful, int nxp, int nyp,
                                 int pitch, long long plane, double* __restrict__ dst) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (long long)nxp * nyp) return;
  const int J = (int)(k / nxp), I = (int)(k - (long long)J * nxp);
  double U[NV];
  if (I >= 2 && I <= nxp - 3 && J >= 2 && J <= nyp - 3) {
    const long long p = (long long)(I - 2) * (nyp - 4) + (J - 2);
    double v[10];
    if (single) {
#pragma unroll
      for (int m = 0; m < 10; m++) v[m] = (double)((const float*)src)[p * 10 + m];
    } else {
#pragma unroll
      for (int m = 0; m < 10; m++) v[m] = ((const double*)src)[p * 10 + m];
    }
    double P[NV];
    P[0] = v[0];
    P[1] = v[1];
    P[2] = v[2];
    if (faithful) {
      P[3] = v[3];
      P[4] = v[5] / v[0];
      P[5] = v[6] / v[0];
      P[6] = v[7] / v[0];
    } else {
      P[3] = v[4];
      P[4] = v[5];
      P[5] = v[6];
      P[6] = v[7];
    }
    P[7] = v[8];
    P[8] = v[9];
    conservative(P, U);
  } else {
#pragma unroll
    for (int m = 0; m < NV; m++) U[m] = 0.0;
  }
#pragma unroll
  for (int m = 0; m < NV; m++) dst[m * plane + (long long)J * pitch + I + 1] = U[m];
}

cudaError_t launch_fields_to_planes(const void* src, int single, int faithful, int nxp, int nyp, int pitch,
                                    long long plane, double* dst, cudaStream_t s) {
  const long long n = (long long)nxp * nyp;
  fields_to_planes<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(src, single, faithful, nxp, nyp, pitch, plane, dst);
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

// ------------------------------------------------------------------ sharding --
// A case split over ranks by block.  pack: the cells other ranks' ghost cells copy,
// gathered from the selected layer into the send buffer (9 values per cell, in the
// plan's order); the ghost kernel reads them back from the receive buffer.
__global__ void shard_pack_kernel(const BlockDev* __restrict__ blk, const CaseDev* __restrict__ cases,
                                  const int2* __restrict__ list, int n, const double* buf0,
                                  const double* buf1, const double* buf2, int sel, double* __restrict__ send) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * NV) return;
  const int i = (int)(t / NV), m = (int)(t - (long long)i * NV);
  const int2 e = list[i];
  const BlockDev B = blk[e.x];
  const int l = phys_layer(sel, cases[0].cur);
  const double* layer = l == 0 ? buf0 : (l == 1 ? buf1 : buf2);
  send[t] = layer[B.off + m * B.plane + e.y];
}

// this rank's share of the CFL of one attempt (case 0, all local blocks), into *out;
// the per-block maxima are cleared as the controller would
__global__ void shard_cfl_kernel(const CaseDev* __restrict__ cases, const BlockDev* __restrict__ blk, int nblk,
                                 unsigned long long* lam, double* out) {
  if (threadIdx.x != 0) return;
  const double dt = cases[0].dt;
  double cfl1 = 0.0, cfl2 = 0.0;
  for (int b = 0; b < nblk; b++) {
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
  // a non-finite write on this rank makes every rank reject the attempt and stop
  *out = cases[0].nonfinite ? __longlong_as_double(0x7ff0000000000000LL) : rmax(cfl1, rmax(cfl2, 0.0));
}

cudaError_t launch_shard_pack(const BlockDev* blk, const CaseDev* cases, const int2* list, int n,
                              double* const buf[3], int sel, double* send, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  shard_pack_kernel<<<(unsigned)(((long long)n * NV + 255) / 256), 256, 0, s>>>(blk, cases, list, n, buf[0], buf[1],
                                                                                buf[2], sel, send);
  return cudaGetLastError();
}

cudaError_t launch_shard_cfl(const CaseDev* cases, const BlockDev* blk, int nblk, unsigned long long* lam,
                             double* out, cudaStream_t s) {
  shard_cfl_kernel<<<1, 32, 0, s>>>(cases, blk, nblk, lam, out);
  return cudaGetLastError();
}

cudaError_t launch_control_ext(CaseDev* cases, const BlockDev* blk, unsigned long long* lam, double* trace,
                               int* queues, const double* cfl_ext, cudaStream_t s) {
  control_kernel<<<1, 256, 0, s>>>(cases, 1, blk, lam, trace, queues, cudaGraphConditionalHandle{}, 0, cfl_ext);
  return cudaGetLastError();
}

// ------------------------------------------------------------------ launchers --
cudaError_t launch_ghost(const BlockDev* blk, const CaseDev* cases, const GhostEntry* map, int n,
                         double* const buf[3], const double* dirichlet, int sel, cudaStream_t s,
                         const double* recv) {
  if (n <= 0) return cudaSuccess;
  return launch_k(ghost_kernel, dim3((n + 127) / 128), dim3(128), 0, s, blk, (const CaseDev*)cases, map, n, buf[0],
                  buf[1], buf[2], dirichlet, recv, sel);
}

cudaError_t launch_control(CaseDev* cases, int ncases, const BlockDev* blk, unsigned long long* lam,
                           double* trace, int* queues, cudaGraphConditionalHandle h, int use_handle,
                           cudaStream_t s) {
  return launch_k(control_kernel, dim3(1), dim3(256), 0, s, cases, ncases, blk, lam, trace, queues, h, use_handle,
                  (const double*)nullptr);
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
