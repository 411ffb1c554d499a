// mbm_adjoint.cu -- discrete adjoint of the Heun step (the reverse of Update and
// SetBoundary), by hand, in three passes per stage over the blocks of a context:
//
//   A  projected primitives P of every cell of the stage input (as the forward
//      stage computes them: Primitive, relaxed with flag 2H+1 off the outermost ring);
//   B  per face next to an output cell: the flux adjoint
//         lambda_F = s * dt/h * (lambda_out(right) - lambda_out(left)),  s = 1 or 1/2,
//      through the HLL flux to the two reconstructed states (PL, PR);
//   C  per cell: the state adjoints of its faces, through the reconstructions
//      P +- h/2 S and the limited slopes S = Limit1(d1, d2)/h of itself and its two
//      neighbours (one-sided derivatives at the limiter's kinks), then through the
//      relaxation and Primitive to the stage input; the relaxation term R of the
//      update adds Cons/relax/Primitive adjoints to the input (and to Data0 in
//      stage 2); the Kn derivative is summed.
//
// The ghost fill is linear: its adjoint adds each ghost cell's adjoint, with the
// wall signs, into the interior cell it was copied from (Dirichlet ghosts have no
// source and contribute nothing).  dt is frozen from the forward run.
#include <cuda_runtime.h>

#include "mbm_internal.h"
#define MBM_HD __host__ __device__ __forceinline__
#include "mbm_adjoint_math.cuh"

namespace mbm {

__device__ __forceinline__ long long cidx(const BlockDev& B, int I, int J) {
  return B.off + (long long)J * B.pitch + I + 1;
}

// Thread mapping: every 128-thread CTA covers a tile of 32 x 4 cells of one block
// (x fastest), so the y neighbours a cell reads were mostly loaded by the same CTA.
// Tiles are numbered block by block; k is the flat thread index.
constexpr int TILE_X = 32, TILE_Y = 4, TILE_T = TILE_X * TILE_Y;

__device__ __forceinline__ bool locate(const BlockDev* blk, int nblk, long long k, int& b, int& I, int& J) {
  long long tile = k / TILE_T;
  const int t = (int)(k - tile * TILE_T);
  for (b = 0; b < nblk; b++) {
    const int tx = (blk[b].nxp + TILE_X - 1) / TILE_X, ty = (blk[b].nyp + TILE_Y - 1) / TILE_Y;
    const long long n = (long long)tx * ty;
    if (tile < n) {
      const int jt = (int)(tile / tx), it = (int)(tile - (long long)jt * tx);
      I = it * TILE_X + (t % TILE_X);
      J = jt * TILE_Y + (t / TILE_X);
      return I < blk[b].nxp && J < blk[b].nyp;
    }
    tile -= n;
  }
  return false;
}

__device__ __forceinline__ void load9(const double* base, const BlockDev& B, int I, int J, double* v) {
  const long long i = cidx(B, I, J);
#pragma unroll
  for (int m = 0; m < NV; m++) v[m] = base[i + m * B.plane];
}

// pass A: the forward stage's projected primitives (Aux.Prim, src/Main.c:314-336)
__global__ void adj_prims(AdjArgs a, long long nthr) {
  pdl_enter();
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int b, I, J;
  if (k >= nthr || !locate(a.blk, a.nblk, k, b, I, J)) return;
  const BlockDev B = a.blk[b];
  double U[NV], P[NV];
  load9(a.x, B, I, J, U);
  mbm_adj::prim(U, P);
  const bool ring = I == 0 || J == 0 || I == B.nxp - 1 || J == B.nyp - 1;
  if (!ring) {
    double Q[NV];
    mbm_adj::relax_p(P, Q, a.dt, a.Kn, a.F, 2 * a.heun + 1);
#pragma unroll
    for (int m = 0; m < NV; m++) P[m] = Q[m];
  }
  const long long i = cidx(B, I, J);
#pragma unroll
  for (int m = 0; m < NV; m++) a.P[i + m * B.plane] = P[m];
}

__device__ __forceinline__ bool inner(const BlockDev& B, int I, int J) {
  return I >= NG && I <= B.nxp - 1 - NG && J >= NG && J <= B.nyp - 1 - NG;
}

// limited slope of cell (I,J) along dir from the primitives (src/Main.c:346-349).  The
// face and cell passes are specialised per Heun stage and limiter (HEUN, LIM), as the
// forward stage kernel is: the limiter's branches and the stage's relaxation flags fold
// away at compile time.
template <int LIM>
__device__ __forceinline__ double slope_at(const AdjArgs& a, const BlockDev& B, int I, int J, int dir, int m,
                                          double h) {
  const long long i = cidx(B, I, J) + m * B.plane;
  const long long s = dir == 1 ? 1 : B.pitch;
  const double d1 = a.P[i] - a.P[i - s], d2 = a.P[i + s] - a.P[i];
  return mbm_adj::limit_val(LIM, d1, d2) * mbm_adj::rcp(h);
}

// pass B: faces (I,J)|(I+1,J) (dir 1) or (I,J)|(I,J+1) (dir 2) next to an output cell
// 128 registers: four 128-thread CTAs per SM hide the neighbour loads better than
// the spill-free allocation at half the occupancy
template <int HEUN, int LIM>
__device__ __forceinline__ void face_adj(const AdjArgs& a, const BlockDev& B, int I, int J, int dir,
                                         double* __restrict__ FL, double* __restrict__ FR) {
  const int I2 = dir == 1 ? I + 1 : I, J2 = dir == 1 ? J : J + 1;
  const bool face = I2 < B.nxp && J2 < B.nyp;
  const bool inL = inner(B, I, J), inR = face && inner(B, I2, J2);
  if (!inL && !inR) {            // no output cell next to this face: zero adjoint
    const long long i = cidx(B, I, J);
#pragma unroll
    for (int m = 0; m < NV; m++) {
      FL[i + m * B.plane] = 0.0;
      FR[i + m * B.plane] = 0.0;
    }
    return;
  }
  const double h = dir == 1 ? B.dx : B.dy, rh = mbm_adj::rcp(h);
  const double s = HEUN ? 0.5 : 1.0;
  double PL[NV], PR[NV], fb[NV], gl[NV] = {0}, gr[NV] = {0};
  bool any = false;
  for (int m = 0; m < NV; m++) {
    const double lo = inL ? a.lout[cidx(B, I, J) + m * B.plane] : 0.0;
    const double hi = inR ? a.lout[cidx(B, I2, J2) + m * B.plane] : 0.0;
    fb[m] = s * a.dt * rh * (hi - lo);
    any = any || fb[m] != 0.0;
    PL[m] = a.P[cidx(B, I, J) + m * B.plane] + 0.5 * h * slope_at<LIM>(a, B, I, J, dir, m, h);
    PR[m] = a.P[cidx(B, I2, J2) + m * B.plane] - 0.5 * h * slope_at<LIM>(a, B, I2, J2, dir, m, h);
  }
  if (any) mbm_adj::hll_p_adj(PL, PR, fb, gl, gr, dir);
  const long long i = cidx(B, I, J);
#pragma unroll
  for (int m = 0; m < NV; m++) {
    FL[i + m * B.plane] = gl[m];
    FR[i + m * B.plane] = gr[m];
  }
}

// both faces of a cell that lie on its high side: (I,J)|(I+1,J) and (I,J)|(I,J+1)
#ifndef ADJ_FACE_CTAS
#define ADJ_FACE_CTAS 4     // resident 128-thread CTAs per SM the face pass is compiled for
#endif
#ifndef ADJ_CELL_CTAS
#define ADJ_CELL_CTAS 8     // the same for the cell pass
#endif
template <int HEUN, int LIM>
__global__ void __launch_bounds__(128, ADJ_FACE_CTAS) adj_faces(AdjArgs a, long long nthr, double* FLx, double* FRx,
                                                    double* FLy, double* FRy) {
  pdl_enter();
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int b, I, J;
  if (k >= nthr || !locate(a.blk, a.nblk, k, b, I, J)) return;
  const BlockDev B = a.blk[b];
  face_adj<HEUN, LIM>(a, B, I, J, 1, FLx, FRx);
  face_adj<HEUN, LIM>(a, B, I, J, 2, FLy, FRy);
}

// adjoint of the reconstruction and slopes along one direction, accumulated into Pb;
// called for cells off the outermost ring (1 <= c <= n-2).  All loads of one
// component are issued before any arithmetic; the slope terms of a neighbour are
// skipped when its slope adjoint is zero (cells no output depends on may hold no
// state, and 0 * NaN would leak into the sum)
// one component m of it (the element index i of that component's plane)
template <int LIM>
__device__ __forceinline__ double gather_comp(const AdjArgs& a, const BlockDev& B, int I, int J, int dir,
                                              const double* FL, const double* FR, long long i) {
  const long long s = dir == 1 ? 1 : B.pitch;
  const int n = dir == 1 ? B.nxp : B.nyp, c = dir == 1 ? I : J;
  const double h = dir == 1 ? B.dx : B.dy, rh = mbm_adj::rcp(h);
  const bool lft = c >= 2, rgt = c <= n - 3;      // slopes of c-1 and c+1 exist (off the ring)
  {
    // face (q | q+1) adjoints: FL = its left state, FR = its right state
    const double flm = FL[i - s], fl0 = FL[i], flp = FL[i + s];
    const double frm2 = lft ? FR[i - 2 * s] : 0.0, frm = FR[i - s], fr0 = FR[i];
    const double pm2 = lft ? a.P[i - 2 * s] : 0.0, pm = a.P[i - s], p0 = a.P[i], pp = a.P[i + s];
    const double pp2 = rgt ? a.P[i + 2 * s] : 0.0;
    // direct: left state of face c|c+1, right state of face c-1|c
    double g = fl0 + frm;
    // S(q) = L(P(q)-P(q-1), P(q+1)-P(q)) / h, its adjoint h/2 (FL(q) - FR(q-1))
    const double l0 = 0.5 * h * (fl0 - frm);
    if (l0 != 0.0) {
      double g1, g2;
      mbm_adj::limit_grad(LIM, p0 - pm, pp - p0, &g1, &g2);
      g += l0 * (g1 - g2) * rh;
    }
    const double lm = lft ? 0.5 * h * (flm - frm2) : 0.0;
    if (lm != 0.0) {
      double g1, g2;
      mbm_adj::limit_grad(LIM, pm - pm2, p0 - pm, &g1, &g2);
      g += lm * g2 * rh;
    }
    const double lp = rgt ? 0.5 * h * (flp - fr0) : 0.0;
    if (lp != 0.0) {
      double g1, g2;
      mbm_adj::limit_grad(LIM, pp - p0, pp2 - pp, &g1, &g2);
      g -= lp * g1 * rh;
    }
    return g;
  }
}

template <int LIM>
__device__ __forceinline__ void gather_dir(const AdjArgs& a, const BlockDev& B, int I, int J, int dir,
                                           const double* FL, const double* FR, double* Pb) {
  const long long i0 = cidx(B, I, J);
#pragma unroll 1
  for (int m = 0; m < NV; m++) Pb[m] += gather_comp<LIM>(a, B, I, J, dir, FL, FR, i0 + m * B.plane);
}

// pass C: per cell, back to the stage input (and Data0)
// one cell's share; returns its contribution to dJ/dKn
// the adjoint of Data0's relaxation term in the stage-2 update, Conservative(relax(
// Primitive(D0), -1)) with weight 1/2: adds to *knb, returns the Data0 adjoint in Vb
__device__ __forceinline__ void data0_adj(const AdjArgs& a, const BlockDev& B, int I, int J, double (&Vb)[NV],
                                          double* knb) {
  double Rb[NV], V[NV], W[NV], Q2[NV], C2[NV] = {0}, Pd[NV] = {0};
#pragma unroll
  for (int m = 0; m < NV; m++) Rb[m] = 0.5 * a.lout[cidx(B, I, J) + m * B.plane];
  load9(a.d0, B, I, J, V);
  mbm_adj::prim(V, W);
  mbm_adj::relax_p(W, Q2, a.dt, a.Kn, a.F, -1);
  mbm_adj::cons_adj(Q2, Rb, C2);
  mbm_adj::relax_p_adj(W, C2, Pd, knb, a.dt, a.Kn, -1);
  mbm_adj::prim_adj(V, Pd, Vb);
}

// the rest of a cell's share once its reconstruction and slope adjoints Pb are gathered;
// D0: the Data0 term here too (stage 2 of the fused cell pass)
template <int HEUN, bool D0>
__device__ __forceinline__ double cell_rest(const AdjArgs& a, const BlockDev& B, int I, int J,
                                            const double (&Pb)[NV]) {
  double Ub[NV] = {0}, U[NV], P0[NV];
  double knb = 0.0;
  load9(a.x, B, I, J, U);
  mbm_adj::prim(U, P0);
  double Qb[NV] = {0};
  bool anyP = false;
#pragma unroll
  for (int m = 0; m < NV; m++) anyP = anyP || Pb[m] != 0.0;
  if (anyP) {     // Aux = relax(Primitive(U), 2H+1) off the ring (ring cells never reach a face)
    mbm_adj::relax_p_adj(P0, Pb, Qb, &knb, a.dt, a.Kn, 2 * HEUN + 1);
  }
  const long long ic = cidx(B, I, J);
  double Vb[NV] = {0};
  if (inner(B, I, J)) {
    // update term R: Conservative(relax(Primitive(X), 2H)) [+ Conservative(relax(Primitive(D0), -1))]
    const double s = HEUN ? 0.5 : 1.0;
    double Rb[NV], Q[NV], Cb[NV] = {0};
#pragma unroll
    for (int m = 0; m < NV; m++) Rb[m] = s * a.lout[cidx(B, I, J) + m * B.plane];
    mbm_adj::relax_p(P0, Q, a.dt, a.Kn, a.F, 2 * HEUN);
    mbm_adj::cons_adj(Q, Rb, Cb);
    mbm_adj::relax_p_adj(P0, Cb, Qb, &knb, a.dt, a.Kn, 2 * HEUN);
    if (HEUN && D0) data0_adj(a, B, I, J, Vb, &knb);
  }
  bool anyQ = false;
#pragma unroll
  for (int m = 0; m < NV; m++) anyQ = anyQ || Qb[m] != 0.0;
  if (anyQ) mbm_adj::prim_adj(U, Qb, Ub);   // cells no stage output depends on may hold no state
  // stage 2 starts both adjoint layers (every cell written: no clearing pass), stage 1
  // adds to the layer stage 2 started
  if (HEUN) {
#pragma unroll
    for (int m = 0; m < NV; m++) {
      a.lx[ic + m * B.plane] = Ub[m];
      if (D0) a.ld0[ic + m * B.plane] = Vb[m];
    }
  } else if (anyQ) {
#pragma unroll
    for (int m = 0; m < NV; m++) a.lx[ic + m * B.plane] += Ub[m];
  }
  return knb;
}

template <int HEUN, int LIM>
__device__ __forceinline__ double cell_adj(const AdjArgs& a, const BlockDev& B, int I, int J, const double* FLx,
                                           const double* FRx, const double* FLy, const double* FRy) {
  double Pb[NV] = {0};
  const bool ring = I == 0 || J == 0 || I == B.nxp - 1 || J == B.nyp - 1;
  if (!ring) {
    gather_dir<LIM>(a, B, I, J, 1, FLx, FRx, Pb);
    gather_dir<LIM>(a, B, I, J, 2, FLy, FRy, Pb);
  }
  return cell_rest<HEUN, true>(a, B, I, J, Pb);
}

// 64 registers, eight 128-thread CTAs per SM: the pass waits on its neighbour loads, and
// more loads in flight pay for the spills (measured, 4 x 256^2: 8 CTAs 10 % faster than 4)
template <int HEUN, int LIM>
__global__ void __launch_bounds__(128, ADJ_CELL_CTAS) adj_cells(AdjArgs a, long long nthr, const double* FLx,
                                                    const double* FRx, const double* FLy, const double* FRy) {
  pdl_enter();
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int b, I, J;
  double knb = 0.0;
  // threads past a block's edge stay for the warp sum below
  if (k < nthr && locate(a.blk, a.nblk, k, b, I, J))
    knb = cell_adj<HEUN, LIM>(a, a.blk[b], I, J, FLx, FRx, FLy, FRy);
  // the Kn derivative: warp sum, one atomic per warp
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) knb += __shfl_xor_sync(0xffffffffu, knb, o);
  if ((threadIdx.x & 31) == 0 && knb != 0.0) atomicAdd(a.knb, knb);
}

// The cell pass split in two (the default; MBM_ADJ_SPLIT=0 keeps it whole): at 64
// registers the whole pass kept fifteen nine-vectors live across its stage-2 Data0 term
// and spilled them (about 80 MB of DRAM writes per launch at 4 x 256^2).  The Data0 term,
// a function of Data0 and the output adjoint alone, moves to the primitives pass of stage
// 2; the gather of the reconstruction and slope adjoints (the neighbour loads) stores Pb;
// a pointwise pass takes it through the relaxation and Primitive.  The same operations
// in the same order per cell; only dJ/dKn's atomic sums are grouped differently.

// pass A of stage 2 with the Data0 term: the projected primitives as adj_prims, and the
// Data0 adjoint of every cell (zero off the interior), which starts that adjoint layer
__global__ void adj_prims_d0(AdjArgs a, long long nthr) {
  pdl_enter();
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int b, I, J;
  double knb = 0.0;
  if (k < nthr && locate(a.blk, a.nblk, k, b, I, J)) {
    const BlockDev B = a.blk[b];
    double U[NV], P[NV];
    load9(a.x, B, I, J, U);
    mbm_adj::prim(U, P);
    const bool ring = I == 0 || J == 0 || I == B.nxp - 1 || J == B.nyp - 1;
    if (!ring) {
      double Q[NV];
      mbm_adj::relax_p(P, Q, a.dt, a.Kn, a.F, 2 * a.heun + 1);
#pragma unroll
      for (int m = 0; m < NV; m++) P[m] = Q[m];
    }
    const long long i = cidx(B, I, J);
#pragma unroll
    for (int m = 0; m < NV; m++) a.P[i + m * B.plane] = P[m];
    double Vb[NV] = {0};
    if (inner(B, I, J)) data0_adj(a, B, I, J, Vb, &knb);
#pragma unroll
    for (int m = 0; m < NV; m++) a.ld0[i + m * B.plane] = Vb[m];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) knb += __shfl_xor_sync(0xffffffffu, knb, o);
  if ((threadIdx.x & 31) == 0 && knb != 0.0) atomicAdd(a.knb, knb);
}

// pass C1: the reconstruction and slope adjoints Pb of every cell (zero on the ring)
template <int LIM>
__global__ void __launch_bounds__(128, ADJ_CELL_CTAS) adj_gather(AdjArgs a, long long nthr, const double* FLx,
                                                     const double* FRx, const double* FLy, const double* FRy) {
  pdl_enter();
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int b, I, J;
  if (k >= nthr || !locate(a.blk, a.nblk, k, b, I, J)) return;
  const BlockDev B = a.blk[b];
  const bool ring = I == 0 || J == 0 || I == B.nxp - 1 || J == B.nyp - 1;
  const long long i0 = cidx(B, I, J);
#pragma unroll 1
  for (int m = 0; m < NV; m++) {        // (0 + x term) + y term, as the whole pass sums them
    const long long i = i0 + m * B.plane;
    double v = 0.0;
    if (!ring) {
      v += gather_comp<LIM>(a, B, I, J, 1, FLx, FRx, i);
      v += gather_comp<LIM>(a, B, I, J, 2, FLy, FRy, i);
    }
    a.Pb[i] = v;
  }
}

// pass C2: per cell, Pb through the relaxation and Primitive to the stage input, with the
// update's relaxation term (the Data0 term is in pass A)
#ifndef ADJ_POINT_CTAS
// resident 128-thread CTAs per SM the pointwise pass is compiled for: 6 (80 registers, 64
// bytes of spills) ran the reverse sweep 1 ms faster than 4 (no spills), 5 or 8 (4 x 256^2)
#define ADJ_POINT_CTAS 6
#endif
template <int HEUN>
__global__ void __launch_bounds__(128, ADJ_POINT_CTAS) adj_point(AdjArgs a, long long nthr) {
  pdl_enter();
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int b, I, J;
  double knb = 0.0;
  if (k < nthr && locate(a.blk, a.nblk, k, b, I, J)) {
    const BlockDev B = a.blk[b];
    const long long i = cidx(B, I, J);
    double Pb[NV];
#pragma unroll
    for (int m = 0; m < NV; m++) Pb[m] = a.Pb[i + m * B.plane];
    knb = cell_rest<HEUN, false>(a, B, I, J, Pb);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) knb += __shfl_xor_sync(0xffffffffu, knb, o);
  if ((threadIdx.x & 31) == 0 && knb != 0.0) atomicAdd(a.knb, knb);
}

// adjoint of the ghost fill: ghost adjoint -> its source cell (wall signs), then
// zero; one thread per (ghost cell, component)
__global__ void adj_ghosts(const BlockDev* __restrict__ blk, const GhostEntry* __restrict__ map, int n, double* l) {
  pdl_enter();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * NV) return;
  const int i = (int)(t / NV), m = (int)(t - (long long)i * NV);
  const GhostEntry e = map[i];
  const BlockDev D = blk[e.dst_blk];
  double* g = l + D.off + e.dst + m * D.plane;
  const double v = *g;
  *g = 0.0;
  if (e.src < 0 || v == 0.0) return;          // Dirichlet ghosts have no source
  const int sblk = e.src_blk_flags & 0xffff;
  const bool fx = (e.src_blk_flags >> 16) & 1, fy = (e.src_blk_flags >> 17) & 1;
  const BlockDev S = blk[sblk];
  const bool flip = (fx && (m == 1 || m == 5 || m == 7)) != (fy && (m == 2 || m == 5 || m == 8));
  atomicAdd(l + S.off + e.src + m * S.plane, flip ? -v : v);
}

// J = sum over interior cells of f(P) of the final state, and dJ/dU; f by `kind`:
//   0  q1^2 + q2^2                                (heat flux)
//   1  theta                                      (temperature)
//   2  (T11 - theta)^2 + 2 T12^2 + (T22 - theta)^2 (deviatoric temperature tensor)
// each CTA writes its partial sum (fixed order: warp shuffles, then the warps in
// order), so J does not depend on scheduling and finite differences of it are clean
__global__ void adj_functional(const BlockDev* __restrict__ blk, int nblk, const double* x, double* l,
                               long long nthr, double* part, int kind) {
  __shared__ double ws[4];
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int b, I, Jj;
  double jv = 0.0;
  if (k < nthr && locate(blk, nblk, k, b, I, Jj)) {
    const BlockDev B = blk[b];
    if (inner(B, I, Jj)) {
      double U[NV], P[NV], Pb[NV] = {0}, Ub[NV] = {0};
      load9(x, B, I, Jj, U);
      mbm_adj::prim(U, P);
      if (kind == 1) {
        jv = P[3];
        Pb[3] = 1.0;
      } else if (kind == 2) {
        const double s11 = P[4] - P[3], s22 = P[6] - P[3];
        jv = s11 * s11 + 2 * P[5] * P[5] + s22 * s22;
        Pb[4] = 2 * s11;
        Pb[5] = 4 * P[5];
        Pb[6] = 2 * s22;
        Pb[3] = -2 * (s11 + s22);
      } else {
        jv = P[7] * P[7] + P[8] * P[8];
        Pb[7] = 2 * P[7];
        Pb[8] = 2 * P[8];
      }
      mbm_adj::prim_adj(U, Pb, Ub);
      const long long i = cidx(B, I, Jj);
      for (int m = 0; m < NV; m++) l[i + m * B.plane] = Ub[m];
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) jv += __shfl_xor_sync(0xffffffffu, jv, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = jv;
  __syncthreads();
  if (threadIdx.x == 0) part[blockIdx.x] = ((ws[0] + ws[1]) + ws[2]) + ws[3];
}

// J = the partial sums added in a fixed order by one CTA
__global__ void sum_partials(const double* part, int n, double* J) {
  __shared__ double ws[8];
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += part[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < 8; w++) t += ws[w];
    *J = t;
  }
}

// ------------------------------------------------------------------ row march --
// The same stage adjoint in one pass, marching up a strip of rows like the forward
// stage kernel.  One warp: lanes <-> columns C = I0-3 .. I0+28, outputs the 26 columns
// I0 .. I0+25 (lanes 3..28) of the non-ring cells of a row segment [J0, J1).  Iteration
// r brings row r: its projected primitives into a four-row window, the stage-output
// adjoint of row r-1 into a three-row window; then the y face (r-2 | r-1) -- its HLL
// adjoint, the slope adjoint of row r-2 and its limiter derivatives, scattered into the
// per-row accumulators of rows r-3 .. r-1 -- and, with row r-3 complete in y, its x faces
// (shuffles), the x slope terms, and the cell step (relaxation, Primitive, update term,
// Data0) for the 26 output cells.  Each slope and limiter derivative is evaluated once,
// nothing but the adjoint layers goes through global memory.  It is an independent second
// implementation of the stage adjoint (MBM_ADJ_MARCH=1; tests require both to agree);
// its 23 KB of shared memory per warp leave 8 warps per SM, too few to hide its
// dependency chains, and it runs 25 % slower than the three-pass version, the default.
struct AdjWindow {
  double P[4][NV][32];      // projected primitives, rows r-3 .. r
  double L[3][NV][32];      // stage-output adjoint (zero off the interior), rows r-3 .. r-1
  double A[3][NV][32];      // y-direction accumulators of the primitive adjoint, rows r-3 .. r-1
};
constexpr int AWARPS = 4;

__device__ __forceinline__ int s3(int q) { return (q + 6) % 3; }
__device__ __forceinline__ int s4(int q) { return (q + 8) & 3; }

__device__ __forceinline__ void benign9(double* U) {
  U[0] = 1.0; U[1] = 0.0; U[2] = 0.0; U[3] = 1.5; U[4] = 1.0;
  U[5] = 0.0; U[6] = 1.0; U[7] = 0.0; U[8] = 0.0;
}

template <int HEUN, int LIM>
__device__ __forceinline__ double march_item(const AdjArgs& a, const Work w, const int lane, AdjWindow& win) {
  const BlockDev B = a.blk[w.blk];
  const int nxp = B.nxp, nyp = B.nyp;
  const long long pitch = B.pitch, plane = B.plane;
  const double* __restrict__ x = a.x + B.off;
  const double* __restrict__ lout = a.lout + B.off;
  const int C = w.I0 - 3 + lane;
  const bool col_in = C >= 0 && C < nxp;
  const bool col_ring = C == 0 || C == nxp - 1;
  const bool col_inner = C >= NG && C <= nxp - 1 - NG;
  const bool out_lane = lane >= 3 && lane <= 28 && C <= nxp - 2;
  const double rdx = mbm_adj::rcp(B.dx), rdy = mbm_adj::rcp(B.dy);
  const double hdx = 0.5 * B.dx, hdy = 0.5 * B.dy;
  const double s = HEUN ? 0.5 : 1.0;
  const double cx = s * a.dt * rdx, cy = s * a.dt * rdy;
  const int rs = w.J0 - 3;
  double knb = 0.0;
  double grp[NV];                     // right-state adjoint of the previous y face
#pragma unroll
  for (int m = 0; m < NV; m++) grp[m] = 0.0;
  for (int r = rs; r <= w.J1 + 2; r++) {
    // (A) row r: projected primitives; stage-output adjoint of row r-1
    {
      double U[NV], P[NV];
      const bool ok = col_in && r >= 0 && r < nyp;
      if (ok) {
#pragma unroll
        for (int m = 0; m < NV; m++) U[m] = x[m * plane + (long long)r * pitch + C + 1];
      } else {
        benign9(U);
      }
      mbm_adj::prim(U, P);
      if (ok && !(col_ring || r == 0 || r == nyp - 1)) {
        double Q[NV];
        mbm_adj::relax_p(P, Q, a.dt, a.Kn, a.F, 2 * HEUN + 1);
#pragma unroll
        for (int m = 0; m < NV; m++) P[m] = Q[m];
      }
#pragma unroll
      for (int m = 0; m < NV; m++) win.P[s4(r)][m][lane] = P[m];
      const int q = r - 1;
      const bool lin = col_inner && q >= NG && q <= nyp - 1 - NG;
#pragma unroll
      for (int m = 0; m < NV; m++)
        win.L[s3(q)][m][lane] = lin ? lout[m * plane + (long long)q * pitch + C + 1] : 0.0;
    }
    // (B) y face (q | q+1), q = r-2: HLL adjoint, slope adjoint of row q
    if (r >= rs + 3) {
      const int q = r - 2;
#pragma unroll
      for (int m = 0; m < NV; m++) win.A[s3(r - 1)][m][lane] = 0.0;   // row r-1: first contribution now
      double fb[NV];
      bool any = false;
#pragma unroll
      for (int m = 0; m < NV; m++) {
        fb[m] = cy * (win.L[s3(q + 1)][m][lane] - win.L[s3(q)][m][lane]);
        any = any || fb[m] != 0.0;
      }
      any = any && out_lane;
      double gl[NV] = {0}, gr[NV] = {0};
      if (any) {
        double PL[NV], PR[NV];
#pragma unroll
        for (int m = 0; m < NV; m++) {
          const double pm = win.P[s4(q - 1)][m][lane], p0 = win.P[s4(q)][m][lane];
          const double p1 = win.P[s4(q + 1)][m][lane], p2 = win.P[s4(q + 2)][m][lane];
          PL[m] = p0 + hdy * (mbm_adj::limit_val(LIM, p0 - pm, p1 - p0) * rdy);
          PR[m] = p1 - hdy * (mbm_adj::limit_val(LIM, p1 - p0, p2 - p1) * rdy);
        }
        mbm_adj::hll_p_adj(PL, PR, fb, gl, gr, 2);
      }
      if (out_lane) {
#pragma unroll
        for (int m = 0; m < NV; m++) {
          double acc = win.A[s3(q)][m][lane] + gl[m] + grp[m];          // direct terms of row q
          const double ls = hdy * (gl[m] - grp[m]);                     // adjoint of S_y(q)
          if (ls != 0.0) {
            const double pm = win.P[s4(q - 1)][m][lane], p0 = win.P[s4(q)][m][lane];
            const double p1 = win.P[s4(q + 1)][m][lane];
            double g1, g2;
            mbm_adj::limit_grad(LIM, p0 - pm, p1 - p0, &g1, &g2);
            win.A[s3(q - 1)][m][lane] -= ls * g1 * rdy;
            acc += ls * (g1 - g2) * rdy;
            win.A[s3(q + 1)][m][lane] += ls * g2 * rdy;
          }
          win.A[s3(q)][m][lane] = acc;
          grp[m] = gr[m];
        }
      }
    }
    // (C) row c = r-3, complete in y: x faces, x slope terms, the cell step
    if (r >= rs + 6) {
      const int c = r - 3;
      const bool xface = lane >= 1 && lane <= 29;
      double P0[NV], PL[NV], PR[NV], fbx[NV], glx[NV] = {0}, grx[NV] = {0};
      bool anyx = false;
#pragma unroll
      for (int m = 0; m < NV; m++) {
        const double p = win.P[s4(c)][m][lane];
        const double pm = __shfl_up_sync(0xffffffffu, p, 1);
        const double pp = __shfl_down_sync(0xffffffffu, p, 1);
        const double pp2 = __shfl_down_sync(0xffffffffu, p, 2);
        const double lam = win.L[s3(c)][m][lane];
        const double lamr = __shfl_down_sync(0xffffffffu, lam, 1);
        P0[m] = p;
        fbx[m] = xface ? cx * (lamr - lam) : 0.0;
        anyx = anyx || fbx[m] != 0.0;
        PL[m] = p + hdx * (mbm_adj::limit_val(LIM, p - pm, pp - p) * rdx);
        PR[m] = pp - hdx * (mbm_adj::limit_val(LIM, pp - p, pp2 - pp) * rdx);
      }
      if (anyx) mbm_adj::hll_p_adj(PL, PR, fbx, glx, grx, 1);
      double Pb[NV];
#pragma unroll
      for (int m = 0; m < NV; m++) {
        const double p = P0[m];
        const double pm = __shfl_up_sync(0xffffffffu, p, 1);
        const double pp = __shfl_down_sync(0xffffffffu, p, 1);
        double grm = __shfl_up_sync(0xffffffffu, grx[m], 1);
        if (lane == 0) grm = 0.0;
        const double ls = hdx * (glx[m] - grm);                          // adjoint of S_x(lane)
        double ga = 0.0, gb = 0.0;
        if (ls != 0.0) {
          double g1, g2;
          mbm_adj::limit_grad(LIM, p - pm, pp - p, &g1, &g2);
          ga = ls * g1 * rdx;
          gb = ls * g2 * rdx;
        }
        double bl = __shfl_up_sync(0xffffffffu, gb, 1);
        double ar = __shfl_down_sync(0xffffffffu, ga, 1);
        if (lane == 0) bl = 0.0;
        if (lane == 31) ar = 0.0;
        Pb[m] = (out_lane ? win.A[s3(c)][m][lane] : 0.0) + glx[m] + grm + (ga - gb) + bl - ar;
      }
      if (out_lane) {
        const long long ic = (long long)c * pitch + C + 1;
        double U[NV], Pr[NV], Qb[NV] = {0}, Ub[NV] = {0}, Vb[NV] = {0};
#pragma unroll
        for (int m = 0; m < NV; m++) U[m] = x[m * plane + ic];
        mbm_adj::prim(U, Pr);
        bool anyP = false;
#pragma unroll
        for (int m = 0; m < NV; m++) anyP = anyP || Pb[m] != 0.0;
        if (anyP) mbm_adj::relax_p_adj(Pr, Pb, Qb, &knb, a.dt, a.Kn, 2 * HEUN + 1);
        if (col_inner && c >= NG && c <= nyp - 1 - NG) {
          double Rb[NV], Q[NV], Cb[NV] = {0};
#pragma unroll
          for (int m = 0; m < NV; m++) Rb[m] = s * win.L[s3(c)][m][lane];
          mbm_adj::relax_p(Pr, Q, a.dt, a.Kn, a.F, 2 * HEUN);
          mbm_adj::cons_adj(Q, Rb, Cb);
          mbm_adj::relax_p_adj(Pr, Cb, Qb, &knb, a.dt, a.Kn, 2 * HEUN);
          if (HEUN) {
            double V[NV], W[NV], Q2[NV], C2[NV] = {0}, Pd[NV] = {0};
#pragma unroll
            for (int m = 0; m < NV; m++) V[m] = a.d0[B.off + m * plane + ic];
            mbm_adj::prim(V, W);
            mbm_adj::relax_p(W, Q2, a.dt, a.Kn, a.F, -1);
            mbm_adj::cons_adj(Q2, Rb, C2);
            mbm_adj::relax_p_adj(W, C2, Pd, &knb, a.dt, a.Kn, -1);
            mbm_adj::prim_adj(V, Pd, Vb);
          }
        }
        bool anyQ = false;
#pragma unroll
        for (int m = 0; m < NV; m++) anyQ = anyQ || Qb[m] != 0.0;
        if (anyQ) mbm_adj::prim_adj(U, Qb, Ub);
        if (HEUN) {           // stage 2 starts both adjoint layers (their ring is cleared beforehand)
#pragma unroll
          for (int m = 0; m < NV; m++) {
            a.lx[B.off + m * plane + ic] = Ub[m];
            a.ld0[B.off + m * plane + ic] = Vb[m];
          }
        } else if (anyQ) {
#pragma unroll
          for (int m = 0; m < NV; m++) a.lx[B.off + m * plane + ic] += Ub[m];
        }
      }
    }
  }
  return knb;
}

template <int HEUN, int LIM>
__global__ void __launch_bounds__(32 * AWARPS, 2) adj_march(AdjArgs a) {
  extern __shared__ __align__(16) unsigned char adj_smem[];
  AdjWindow* win = reinterpret_cast<AdjWindow*>(adj_smem);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double knb = 0.0;
  for (;;) {
    int w = 0;
    if (lane == 0) w = atomicAdd(a.queue, 1);
    w = __shfl_sync(0xffffffffu, w, 0);
    if (w >= a.nwork) break;
    knb += march_item<HEUN, LIM>(a, a.work[w], lane, win[warp]);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) knb += __shfl_xor_sync(0xffffffffu, knb, o);
  if (lane == 0 && knb != 0.0) atomicAdd(a.knb, knb);
}

constexpr int ADJ_SMEM = (int)sizeof(AdjWindow) * AWARPS;

template <int HEUN, int LIM>
static void march_attr() {
  cudaFuncSetAttribute(adj_march<HEUN, LIM>, cudaFuncAttributeMaxDynamicSharedMemorySize, ADJ_SMEM);
}

// CTAs per SM of the row-marching pass (allows its dynamic shared memory first)
int adjoint_march_ctas() {
  march_attr<0, 0>(); march_attr<0, 1>(); march_attr<0, 2>(); march_attr<0, 3>(); march_attr<0, 4>();
  march_attr<1, 0>(); march_attr<1, 1>(); march_attr<1, 2>(); march_attr<1, 3>(); march_attr<1, 4>();
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, adj_march<1, 4>, 32 * AWARPS, ADJ_SMEM);
  return n > 0 ? n : 1;
}

template <int HEUN>
static void march_lim(const AdjArgs& a, int grid, cudaStream_t s) {
  switch (a.limiter) {
    case 0: adj_march<HEUN, 0><<<grid, 32 * AWARPS, ADJ_SMEM, s>>>(a); break;
    case 1: adj_march<HEUN, 1><<<grid, 32 * AWARPS, ADJ_SMEM, s>>>(a); break;
    case 2: adj_march<HEUN, 2><<<grid, 32 * AWARPS, ADJ_SMEM, s>>>(a); break;
    case 3: adj_march<HEUN, 3><<<grid, 32 * AWARPS, ADJ_SMEM, s>>>(a); break;
    default: adj_march<HEUN, 4><<<grid, 32 * AWARPS, ADJ_SMEM, s>>>(a); break;
  }
}

// one stage's adjoint by the row-marching pass; a.queue must be zero
cudaError_t adjoint_stage_march(const AdjArgs& a, int grid, cudaStream_t s) {
  if (a.heun) march_lim<1>(a, grid, s);
  else march_lim<0>(a, grid, s);
  return cudaGetLastError();
}

template <int HEUN, int LIM>
static void faces_cells(const AdjArgs& a0, long long nthr, unsigned G, double* FLx, double* FRx, double* FLy,
                        double* FRy, cudaStream_t s) {
  launch_k(adj_faces<HEUN, LIM>, dim3(G), dim3(128), 0, s, a0, nthr, FLx, FRx, FLy, FRy);
  if (a0.Pb) {
    launch_k(adj_gather<LIM>, dim3(G), dim3(128), 0, s, a0, nthr, (const double*)FLx, (const double*)FRx,
             (const double*)FLy, (const double*)FRy);
    launch_k(adj_point<HEUN>, dim3(G), dim3(128), 0, s, a0, nthr);
  } else {
    launch_k(adj_cells<HEUN, LIM>, dim3(G), dim3(128), 0, s, a0, nthr, (const double*)FLx, (const double*)FRx,
             (const double*)FLy, (const double*)FRy);
  }
}

template <int HEUN>
static void faces_cells_lim(const AdjArgs& a0, long long nthr, unsigned G, double* FLx, double* FRx,
                            double* FLy, double* FRy, cudaStream_t s) {
  switch (a0.limiter) {
    case 0: faces_cells<HEUN, 0>(a0, nthr, G, FLx, FRx, FLy, FRy, s); break;
    case 1: faces_cells<HEUN, 1>(a0, nthr, G, FLx, FRx, FLy, FRy, s); break;
    case 2: faces_cells<HEUN, 2>(a0, nthr, G, FLx, FRx, FLy, FRy, s); break;
    case 3: faces_cells<HEUN, 3>(a0, nthr, G, FLx, FRx, FLy, FRy, s); break;
    default: faces_cells<HEUN, 4>(a0, nthr, G, FLx, FRx, FLy, FRy, s); break;
  }
}

cudaError_t adjoint_stage(const AdjArgs& a0, long long nthr, double* FLx, double* FRx, double* FLy,
                          double* FRy, cudaStream_t s) {
  const int T = 128;
  const unsigned G = (unsigned)(nthr / T);
  if (a0.Pb && a0.heun)
    launch_k(adj_prims_d0, dim3(G), dim3(T), 0, s, a0, nthr);
  else
    launch_k(adj_prims, dim3(G), dim3(T), 0, s, a0, nthr);
  if (a0.heun) faces_cells_lim<1>(a0, nthr, G, FLx, FRx, FLy, FRy, s);
  else faces_cells_lim<0>(a0, nthr, G, FLx, FRx, FLy, FRy, s);
  return cudaGetLastError();
}

cudaError_t adjoint_ghosts(const BlockDev* blk, const GhostEntry* map, int n, double* l, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  launch_k(adj_ghosts, dim3((unsigned)(((long long)n * NV + 255) / 256)), dim3(256), 0, s, blk, map, n, l);
  return cudaGetLastError();
}

// nthr: 128 threads per 32 x 4 tile of every block; part: nthr / 128 doubles of scratch
cudaError_t adjoint_functional(const BlockDev* blk, int nblk, const double* x, double* l, long long nthr,
                               double* part, double* J, int kind, cudaStream_t s) {
  const unsigned G = (unsigned)(nthr / 128);
  adj_functional<<<G, 128, 0, s>>>(blk, nblk, x, l, nthr, part, kind);
  sum_partials<<<1, 256, 0, s>>>(part, (int)G, J);
  return cudaGetLastError();
}

}  // namespace mbm
