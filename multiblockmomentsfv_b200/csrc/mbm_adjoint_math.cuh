// mbm_adjoint_math.cuh -- reverse-mode (adjoint) derivatives of the per-cell and
// per-face maps of one Heun stage, written by hand.
//
// The adjoint differentiates the mathematical maps the reference computes, in
// primitive variables P = {rho, u, v, theta, T11, T12, T22, q1, q2}:
//   Conservative  P -> U              (src/Flux.c:61-74)
//   Primitive     U -> P              (src/Flux.c:30-56)
//   relaxation    P -> P'             (ProductionsDirect, src/Flux.c:196-267, in P form:
//                                      rho, theta kept, T_ij - theta delta_ij scaled by
//                                      R(z), q by R(2z/3), z = rho sqrt(theta) dt / Kn,
//                                      velocity pushed by dt F for flags 0 and 2)
//   face flux     (PL, PR) -> flux    (FnumHLLE with the Grad-13 flux, src/Flux.c:79-119,
//                                      308-379; for y faces the x/y components swap)
//   limiter       (d1, d2) -> slope   (Limit1, src/Limiter.c:42-59; one-sided
//                                      derivatives at the kinks: the branch taken)
// The forward pass computes U -> P -> U round trips and rotations the adjoint
// treats as exact identities; the difference is rounding, far below the 1e-6 the
// gradient is checked to.  Functions named *_adj take the output adjoint and
// ADD the input adjoint into the argument arrays.
#pragma once

#include <math.h>

#ifdef __CUDACC__
#include "mbm_newton.cuh"
#endif

#ifndef MBM_HD
#ifdef __CUDACC__
#define MBM_HD __host__ __device__ __forceinline__
#else
#define MBM_HD static inline
#endif
#endif

namespace mbm_adj {

constexpr int NV = 9;

// 1/x and sqrt(x): on the device the Newton-refined hardware approximations
// (mbm_newton.cuh; the derivatives need no bit-exact values), one multiply per
// quotient after the reciprocal
MBM_HD double rcp(double x) {
#ifdef __CUDA_ARCH__
  return mbm_newton::frcp(x);
#else
  return 1.0 / x;
#endif
}

MBM_HD double root(double x) {
#ifdef __CUDA_ARCH__
  return mbm_newton::fsqrt(x);
#else
  return sqrt(x);
#endif
}

// ---------------------------------------------------------------- Conservative
MBM_HD void cons(const double* P, double* U) {
  const double r = P[0], u = P[1], v = P[2], th = P[3];
  const double E = 0.5 * r * (u * u + v * v) + 1.5 * r * th;
  U[0] = r;
  U[1] = r * u;
  U[2] = r * v;
  U[3] = E;
  U[4] = r * (P[4] + u * u);
  U[5] = r * (P[5] + u * v);
  U[6] = r * (P[6] + v * v);
  U[7] = P[7] + E * u + r * (P[4] * u + P[5] * v);
  U[8] = P[8] + E * v + r * (P[5] * u + P[6] * v);
}

// P_bar += (dU/dP)^T U_bar
MBM_HD void cons_adj(const double* P, const double* Ub, double* Pb) {
  const double r = P[0], u = P[1], v = P[2], th = P[3];
  const double T11 = P[4], T12 = P[5], T22 = P[6];
  const double vs = u * u + v * v;
  const double E = 0.5 * r * vs + 1.5 * r * th;
  // E feeds U3, U7 (E u), U8 (E v)
  const double Eb = Ub[3] + Ub[7] * u + Ub[8] * v;
  double rb = Ub[0] + Ub[1] * u + Ub[2] * v + Ub[4] * (T11 + u * u) + Ub[5] * (T12 + u * v) +
              Ub[6] * (T22 + v * v) + Ub[7] * (T11 * u + T12 * v) + Ub[8] * (T12 * u + T22 * v);
  double ub = Ub[1] * r + Ub[4] * 2 * r * u + Ub[5] * r * v + Ub[7] * (E + r * T11) + Ub[8] * r * T12;
  double vb = Ub[2] * r + Ub[5] * r * u + Ub[6] * 2 * r * v + Ub[7] * r * T12 + Ub[8] * (E + r * T22);
  rb += Eb * (0.5 * vs + 1.5 * th);
  ub += Eb * r * u;
  vb += Eb * r * v;
  Pb[0] += rb;
  Pb[1] += ub;
  Pb[2] += vb;
  Pb[3] += Eb * 1.5 * r;
  Pb[4] += Ub[4] * r + Ub[7] * r * u;
  Pb[5] += Ub[5] * r + Ub[7] * r * v + Ub[8] * r * u;
  Pb[6] += Ub[6] * r + Ub[8] * r * v;
  Pb[7] += Ub[7];
  Pb[8] += Ub[8];
}

// ------------------------------------------------------------------ Primitive
MBM_HD void prim(const double* U, double* P) {
  const double r = U[0], ir = rcp(r);
  const double u = U[1] * ir, v = U[2] * ir;
  const double vs = u * u + v * v;
  P[0] = r;
  P[1] = u;
  P[2] = v;
  P[3] = (2 * U[3] * ir - vs) * (1.0 / 3);
  P[4] = U[4] * ir - u * u;
  P[5] = U[5] * ir - u * v;
  P[6] = U[6] * ir - v * v;
  P[7] = U[7] - U[3] * u - r * (P[4] * u + P[5] * v);
  P[8] = U[8] - U[3] * v - r * (P[5] * u + P[6] * v);
}

// U_bar += (dP/dU)^T P_bar
MBM_HD void prim_adj(const double* U, const double* Pb_in, double* Ub) {
  double P[NV];
  prim(U, P);
  const double r = U[0], u = P[1], v = P[2], E = U[3];
  const double ir = rcp(r), ir2 = ir * ir;
  const double T11 = P[4], T12 = P[5], T22 = P[6];
  double Pb[NV];
  for (int n = 0; n < NV; n++) Pb[n] = Pb_in[n];
  double rb = Pb[0], ub = Pb[1], vb = Pb[2];
  double U3b = 0, U4b = 0, U5b = 0, U6b = 0;
  // q2 = U8 - E v - r (T12 u + T22 v)
  Ub[8] += Pb[8];
  U3b += -Pb[8] * v;
  vb += -Pb[8] * (E + r * T22);
  rb += -Pb[8] * (T12 * u + T22 * v);
  double T12b = -Pb[8] * r * u, T22b = -Pb[8] * r * v;
  ub += -Pb[8] * r * T12;
  // q1 = U7 - E u - r (T11 u + T12 v)
  Ub[7] += Pb[7];
  U3b += -Pb[7] * u;
  ub += -Pb[7] * (E + r * T11);
  rb += -Pb[7] * (T11 * u + T12 * v);
  double T11b = -Pb[7] * r * u;
  T12b += -Pb[7] * r * v;
  vb += -Pb[7] * r * T12;
  T11b += Pb[4];
  T12b += Pb[5];
  T22b += Pb[6];
  // T22 = U6/r - v^2 ; T12 = U5/r - u v ; T11 = U4/r - u^2
  U6b += T22b * ir;
  rb += -T22b * U[6] * ir2;
  vb += -T22b * 2 * v;
  U5b += T12b * ir;
  rb += -T12b * U[5] * ir2;
  ub += -T12b * v;
  vb += -T12b * u;
  U4b += T11b * ir;
  rb += -T11b * U[4] * ir2;
  ub += -T11b * 2 * u;
  // th = (2 U3/r - u^2 - v^2)/3
  const double thb = Pb[3];
  U3b += thb * (2.0 / 3) * ir;
  rb += -thb * (2.0 / 3) * U[3] * ir2;
  ub += -thb * (2.0 / 3) * u;
  vb += -thb * (2.0 / 3) * v;
  // u = U1/r, v = U2/r
  Ub[1] += ub * ir;
  Ub[2] += vb * ir;
  rb += -(ub * U[1] + vb * U[2]) * ir2;
  Ub[0] += rb;
  Ub[3] += U3b;
  Ub[4] += U4b;
  Ub[5] += U5b;
  Ub[6] += U6b;
}

// ----------------------------------------------------------------- relaxation
// damping factors and their derivatives (src/Flux.c:213-223)
MBM_HD double rdamp(double z, int flag, double* dz) {
  double N, D, Nd, Dd;
  switch (flag) {
    case -1:
    case 0: N = 1 + 0.5 * z - 0.25 * z * z; Nd = 0.5 - 0.5 * z; D = 1 + z + 0.25 * z * z; Dd = 1 + 0.5 * z; break;
    case 1: N = 1 + z; Nd = 1; D = 1 + z + 0.25 * z * z; Dd = 1 + 0.5 * z; break;
    case 2: *dz = 0.0; return 1.0;
    default: N = 1; Nd = 0; D = 1 + 0.5 * z; Dd = 0.5; break;
  }
  const double iD = rcp(D);
  *dz = (Nd * D - N * Dd) * iD * iD;
  return N * iD;
}

// relaxation in primitive form: P -> Q (ProductionsDirect's state, src/Flux.c:230-267)
MBM_HD void relax_p(const double* P, double* Q, double dt, double Kn, double F, int flag) {
  const double r = P[0], th = P[3];
  const double z = r * root(th) * rcp(Kn) * dt;
  double dd;
  const double d1 = rdamp(z, flag, &dd);
  const double d2 = rdamp(2.0 / 3 * z, flag, &dd);
  Q[0] = r;
  Q[1] = P[1] + ((flag == 0 || flag == 2) ? dt * F : 0.0);
  Q[2] = P[2];
  Q[3] = th;
  Q[4] = d1 * (P[4] - th) + th;
  Q[5] = d1 * P[5];
  Q[6] = d1 * (P[6] - th) + th;
  Q[7] = d2 * P[7];
  Q[8] = d2 * P[8];
}

// P_bar += (dQ/dP)^T Q_bar, *Kn_bar += (dQ/dKn) . Q_bar
MBM_HD void relax_p_adj(const double* P, const double* Qb, double* Pb, double* Knb, double dt, double Kn,
                        int flag) {
  const double r = P[0], th = P[3];
  const double z = r * root(th) * rcp(Kn) * dt;
  double r1, r2;
  const double d1 = rdamp(z, flag, &r1);
  const double d2 = rdamp(2.0 / 3 * z, flag, &r2);
  Pb[0] += Qb[0];
  Pb[1] += Qb[1];
  Pb[2] += Qb[2];
  Pb[3] += Qb[3] + (Qb[4] + Qb[6]) * (1 - d1);
  Pb[4] += Qb[4] * d1;
  Pb[5] += Qb[5] * d1;
  Pb[6] += Qb[6] * d1;
  Pb[7] += Qb[7] * d2;
  Pb[8] += Qb[8] * d2;
  const double d1b = Qb[4] * (P[4] - th) + Qb[5] * P[5] + Qb[6] * (P[6] - th);
  const double d2b = Qb[7] * P[7] + Qb[8] * P[8];
  const double zb = d1b * r1 + d2b * (2.0 / 3) * r2;
  if (z != 0.0) {
    Pb[0] += zb * z * rcp(r);
    Pb[3] += 0.5 * zb * z * rcp(th);
    *Knb += -zb * z * rcp(Kn);
  }
}

// ------------------------------------------------------------------ face flux
// Grad-13 flux along x in primitive variables (src/Flux.c:79-119 with U = Conservative(P))
MBM_HD void gflux_x(const double* P, double* F) {
  const double r = P[0], u = P[1], v = P[2], th = P[3];
  const double T11 = P[4], T12 = P[5], T22 = P[6], q1 = P[7], q2 = P[8];
  const double vs = u * u + v * v;
  const double E = 0.5 * r * vs + 1.5 * r * th;
  F[0] = r * u;
  F[1] = r * (T11 + u * u);
  F[2] = r * (T12 + u * v);
  F[3] = E * u + r * (T11 * u + T12 * v) + q1;
  F[4] = 1.2 * q1 + r * (3 * T11 * u + u * u * u);
  F[5] = 0.4 * q2 + r * (T11 * v + 2 * T12 * u + u * u * v);
  F[6] = 0.4 * q1 + r * (T22 * u + 2 * T12 * v + v * v * u);
  F[7] = 2 * (q1 + r * (T11 * u + T12 * v)) * u + E * u * u + 1.2 * q1 * u + 0.4 * q2 * v +
         0.5 * r * (T11 * vs + 5 * th * th + 7 * th * (T11 - th));
  F[8] = q2 * u + q1 * v + r * (u * v * (T11 + T22) + 1.5 * T12 * vs) + E * u * v + 0.4 * q2 * u +
         0.4 * q1 * v + 3.5 * r * th * T12;
}

// P_bar += (dF/dP)^T F_bar
MBM_HD void gflux_x_adj(const double* P, const double* Fb, double* Pb) {
  const double r = P[0], u = P[1], v = P[2], th = P[3];
  const double T11 = P[4], T12 = P[5], T22 = P[6], q1 = P[7], q2 = P[8];
  const double vs = u * u + v * v;
  const double E = 0.5 * r * vs + 1.5 * r * th;
  const double A = T11 * u + T12 * v;
  double rb = 0, ub = 0, vb = 0, thb = 0, T11b = 0, T12b = 0, T22b = 0, q1b = 0, q2b = 0, Eb = 0, vsb = 0;
  // F0 = r u
  rb += Fb[0] * u; ub += Fb[0] * r;
  // F1 = r (T11 + u^2)
  rb += Fb[1] * (T11 + u * u); T11b += Fb[1] * r; ub += Fb[1] * 2 * r * u;
  // F2 = r (T12 + u v)
  rb += Fb[2] * (T12 + u * v); T12b += Fb[2] * r; ub += Fb[2] * r * v; vb += Fb[2] * r * u;
  // F3 = E u + r A + q1
  Eb += Fb[3] * u; ub += Fb[3] * E; rb += Fb[3] * A; q1b += Fb[3];
  T11b += Fb[3] * r * u; T12b += Fb[3] * r * v; ub += Fb[3] * r * T11; vb += Fb[3] * r * T12;
  // F4 = 1.2 q1 + r (3 T11 u + u^3)
  q1b += Fb[4] * 1.2; rb += Fb[4] * (3 * T11 * u + u * u * u);
  T11b += Fb[4] * 3 * r * u; ub += Fb[4] * r * (3 * T11 + 3 * u * u);
  // F5 = 0.4 q2 + r (T11 v + 2 T12 u + u^2 v)
  q2b += Fb[5] * 0.4; rb += Fb[5] * (T11 * v + 2 * T12 * u + u * u * v);
  T11b += Fb[5] * r * v; T12b += Fb[5] * 2 * r * u;
  ub += Fb[5] * r * (2 * T12 + 2 * u * v); vb += Fb[5] * r * (T11 + u * u);
  // F6 = 0.4 q1 + r (T22 u + 2 T12 v + v^2 u)
  q1b += Fb[6] * 0.4; rb += Fb[6] * (T22 * u + 2 * T12 * v + v * v * u);
  T22b += Fb[6] * r * u; T12b += Fb[6] * 2 * r * v;
  ub += Fb[6] * r * (T22 + v * v); vb += Fb[6] * r * (2 * T12 + 2 * v * u);
  // F7 = 2 (q1 + r A) u + E u^2 + 1.2 q1 u + 0.4 q2 v + 0.5 r (T11 vs + 5 th^2 + 7 th (T11 - th))
  {
    const double w = Fb[7];
    q1b += w * (2 * u + 1.2 * u);
    rb += w * (2 * A * u + 0.5 * (T11 * vs + 5 * th * th + 7 * th * (T11 - th)));
    T11b += w * (2 * r * u * u + 0.5 * r * (vs + 7 * th));
    T12b += w * 2 * r * v * u;
    ub += w * (2 * (q1 + r * A) + 2 * r * T11 * u + 2 * E * u + 1.2 * q1);
    vb += w * (2 * r * T12 * u + 0.4 * q2);
    Eb += w * u * u;
    q2b += w * 0.4 * v;
    vsb += w * 0.5 * r * T11;
    thb += w * 0.5 * r * (10 * th + 7 * (T11 - th) - 7 * th);
  }
  // F8 = q2 u + q1 v + r (u v (T11 + T22) + 1.5 T12 vs) + E u v + 0.4 q2 u + 0.4 q1 v + 3.5 r th T12
  {
    const double w = Fb[8];
    q2b += w * (u + 0.4 * u);
    q1b += w * (v + 0.4 * v);
    rb += w * (u * v * (T11 + T22) + 1.5 * T12 * vs + 3.5 * th * T12);
    ub += w * (q2 + r * v * (T11 + T22) + E * v + 0.4 * q2);
    vb += w * (q1 + r * u * (T11 + T22) + E * u + 0.4 * q1);
    T11b += w * r * u * v;
    T22b += w * r * u * v;
    T12b += w * (1.5 * r * vs + 3.5 * r * th);
    vsb += w * 1.5 * r * T12;
    Eb += w * u * v;
    thb += w * 3.5 * r * T12;
  }
  // E = 0.5 r vs + 1.5 r th ; vs = u^2 + v^2
  rb += Eb * (0.5 * vs + 1.5 * th);
  vsb += Eb * 0.5 * r;
  thb += Eb * 1.5 * r;
  ub += vsb * 2 * u;
  vb += vsb * 2 * v;
  Pb[0] += rb; Pb[1] += ub; Pb[2] += vb; Pb[3] += thb;
  Pb[4] += T11b; Pb[5] += T12b; Pb[6] += T22b; Pb[7] += q1b; Pb[8] += q2b;
}

// x <-> y swap of primitives, moments and fluxes (the rotation of Grad13Flux2D for
// the normal (0,1), src/Flux.c:126-172, is this permutation)
MBM_HD void swap_xy(const double* a, double* b) {
  b[0] = a[0]; b[1] = a[2]; b[2] = a[1]; b[3] = a[3];
  b[4] = a[6]; b[5] = a[5]; b[6] = a[4]; b[7] = a[8]; b[8] = a[7];
}

// HLL flux of a face (FnumHLLE) in primitive form; dir 1 = x, 2 = y
MBM_HD void hll_p(const double* PL_, const double* PR_, double* flx, int dir) {
  double PL[NV], PR[NV], UL[NV], UR[NV], fL[NV], fR[NV];
  if (dir == 2) { swap_xy(PL_, PL); swap_xy(PR_, PR); }
  else for (int n = 0; n < NV; n++) { PL[n] = PL_[n]; PR[n] = PR_[n]; }
  const double cL = 2.0 * root(5.0 / 3 * PL[3]), cR = 2.0 * root(5.0 / 3 * PR[3]);
  cons(PL, UL); cons(PR, UR); gflux_x(PL, fL); gflux_x(PR, fR);
  const double lamL = (PL[1] - cL) < 0.0 ? PL[1] - cL : 0.0;
  const double lamR = (PR[1] + cR) > 0.0 ? PR[1] + cR : 0.0;
  const double alph = lamR - lamL;
  double f[NV];
  for (int n = 0; n < NV; n++)
    f[n] = alph > 0.0 ? (lamR * fL[n] - lamL * fR[n] + lamL * lamR * (UR[n] - UL[n])) / alph
                      : 0.5 * (fL[n] + fR[n]);
  if (dir == 2) swap_xy(f, flx);
  else for (int n = 0; n < NV; n++) flx[n] = f[n];
}

// PL_bar, PR_bar += (dflux/dP)^T flux_bar
MBM_HD void hll_p_adj(const double* PL_, const double* PR_, const double* fb_, double* PLb_, double* PRb_,
                      int dir) {
  // F = (lamR fL - lamL fR + lamL lamR (UR - UL)) / alph is linear in fL, fR, UL, UR
  // for fixed wave speeds, so their adjoints are fb times scalars and the wave-speed
  // adjoints need only the dot products of fb with fL, fR, UL, UR: no 9-vector of
  // either side is kept (register pressure of the face kernel)
  double PL[NV], PR[NV], fb[NV], T[NV];
  if (dir == 2) { swap_xy(PL_, PL); swap_xy(PR_, PR); swap_xy(fb_, fb); }
  else for (int n = 0; n < NV; n++) { PL[n] = PL_[n]; PR[n] = PR_[n]; fb[n] = fb_[n]; }
  const double cL = 2.0 * root(5.0 / 3 * PL[3]), cR = 2.0 * root(5.0 / 3 * PR[3]);
  const bool aL = (PL[1] - cL) < 0.0, aR = (PR[1] + cR) > 0.0;
  const double lamL = aL ? PL[1] - cL : 0.0;
  const double lamR = aR ? PR[1] + cR : 0.0;
  const double alph = lamR - lamL;
  double PLb[NV] = {0}, PRb[NV] = {0};
  if (alph > 0.0) {
    double A = 0, B = 0, DL = 0, DR = 0;
    gflux_x(PL, T);
    for (int n = 0; n < NV; n++) A += fb[n] * T[n];
    cons(PL, T);
    for (int n = 0; n < NV; n++) DL += fb[n] * T[n];
    gflux_x(PR, T);
    for (int n = 0; n < NV; n++) B += fb[n] * T[n];
    cons(PR, T);
    for (int n = 0; n < NV; n++) DR += fb[n] * T[n];
    const double D = DR - DL;
    const double ia = rcp(alph);
    const double Fd = (lamR * A - lamL * B + lamL * lamR * D) * ia;     // fb . F
    const double lRb = (A + lamL * D - Fd) * ia;                         // dF/dlamR . fb
    const double lLb = (-B + lamR * D + Fd) * ia;                        // dF/dlamL . fb
    // lamL = uL - cL (active), lamR = uR + cR (active); c = 2 sqrt(5 th / 3), dc/dth = (10/3)/c
    if (aL) { PLb[1] += lLb; PLb[3] += -lLb * (10.0 / 3) * rcp(cL); }
    if (aR) { PRb[1] += lRb; PRb[3] += lRb * (10.0 / 3) * rcp(cR); }
    const double kU = lamL * lamR * ia;
    for (int n = 0; n < NV; n++) T[n] = -kU * fb[n];
    cons_adj(PL, T, PLb);
    for (int n = 0; n < NV; n++) T[n] = fb[n] * lamR * ia;
    gflux_x_adj(PL, T, PLb);
    for (int n = 0; n < NV; n++) T[n] = kU * fb[n];
    cons_adj(PR, T, PRb);
    for (int n = 0; n < NV; n++) T[n] = -fb[n] * lamL * ia;
    gflux_x_adj(PR, T, PRb);
  } else {
    for (int n = 0; n < NV; n++) T[n] = 0.5 * fb[n];
    gflux_x_adj(PL, T, PLb);
    gflux_x_adj(PR, T, PRb);
  }
  if (dir == 2) {
    double a[NV], b[NV];
    swap_xy(PLb, a); swap_xy(PRb, b);
    for (int n = 0; n < NV; n++) { PLb_[n] += a[n]; PRb_[n] += b[n]; }
  } else {
    for (int n = 0; n < NV; n++) { PLb_[n] += PLb[n]; PRb_[n] += PRb[n]; }
  }
}

// ------------------------------------------------------------------- limiter
// partial derivatives (dL/dd1, dL/dd2) of Limit1 (src/Limiter.c:42-59); at kinks
// the branch the forward pass takes
MBM_HD void limit_grad(int lim, double d1, double d2, double* g1, double* g2) {
  switch (lim) {
    case 0: *g1 = 0; *g2 = 0; return;
    case 1: *g1 = 0.5; *g2 = 0.5; return;
    case 2: {
      const double s1 = d1 == 0 ? 0.0 : (d1 < 0 ? -1.0 : 1.0);
      const double s2 = d2 == 0 ? 0.0 : (d2 < 0 ? -1.0 : 1.0);
      const double k = 0.5 * (s1 + s2);
      if (fabs(d1) < fabs(d2)) { *g1 = k * s1; *g2 = 0; }
      else { *g1 = 0; *g2 = k * s2; }
      return;
    }
    case 3: {
      if (d1 == 0) { *g1 = 0; *g2 = 0; return; }
      const double th = d2 * rcp(d1);
      // L = d1 phi(th):  dL/dd1 = phi - th phi',  dL/dd2 = phi'
      double phi, dphi;
      if (th < 0.0) { phi = 0; dphi = 0; }
      else if (th < 0.5) { phi = 2 * th; dphi = 2; }
      else if (th < 1.0) { phi = 1; dphi = 0; }
      else if (th < 2.0) { phi = th; dphi = 1; }
      else { phi = 2; dphi = 0; }
      *g1 = phi - th * dphi;
      *g2 = dphi;
      return;
    }
    default: {
      const double eps = 1.0e-10;
      const double w1 = fabs(d1) + eps, w2 = fabs(d2) + eps;
      const double s1 = d1 < 0 ? -1.0 : 1.0, s2 = d2 < 0 ? -1.0 : 1.0;
      const double N = w1 * d2 + w2 * d1, D = w1 + w2;
      // dN/dd1 = s1 d2 + w2, dN/dd2 = w1 + s2 d1 ; dD/dd1 = s1, dD/dd2 = s2
      const double iD2 = rcp(D * D);
      *g1 = ((s1 * d2 + w2) * D - N * s1) * iD2;
      *g2 = ((w1 + s2 * d1) * D - N * s2) * iD2;
      return;
    }
  }
}

MBM_HD double limit_val(int lim, double d1, double d2) {
  switch (lim) {
    case 0: return 0.0;
    case 1: return 0.5 * (d1 + d2);
    case 2: {
      const double s1 = d1 == 0 ? 0.0 : (d1 < 0 ? -1.0 : 1.0);
      const double s2 = d2 == 0 ? 0.0 : (d2 < 0 ? -1.0 : 1.0);
      return 0.5 * (s1 + s2) * (fabs(d1) < fabs(d2) ? fabs(d1) : fabs(d2));
    }
    case 3: {
      const double th = d2 * rcp(d1);
      double phi;
      if (th < 0.0) phi = 0;
      else if (th < 0.5) phi = 2 * th;
      else if (th < 1.0) phi = 1;
      else if (th < 2.0) phi = th;
      else phi = 2;
      return d1 * phi;
    }
    default: {
      const double eps = 1.0e-10;
      const double w1 = fabs(d1) + eps, w2 = fabs(d2) + eps;
      return (w1 * d2 + w2 * d1) * rcp(w1 + w2);
    }
  }
}

}  // namespace mbm_adj
