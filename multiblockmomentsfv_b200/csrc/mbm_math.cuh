// mbm_math.cuh -- per-cell and per-face FP64 arithmetic of the Grad-13 Heun stage,
// in namespace mbm::MBM_ARITH (bitwise by default, fastmath under MBM_FAST_ARITH).
//
// Bitwise mode: every expression keeps the operand order and association of the
// reference expression it restates (file:line cited per function), the file is
// compiled with -fmad=false, and double division and sqrt are IEEE round-to-
// nearest on sm_100a, so results agree bit for bit with the reference compiled
// by gcc on x86-64 (SSE2, no contraction).
#pragma once

#include <cuda_runtime.h>
#include <math.h>

#include "mbm_internal.h"

#ifndef MBM_ARITH
#define MBM_ARITH bitwise
#endif
#ifndef MBM_FAST_ARITH
#define MBM_FAST_ARITH 0
#endif
#if MBM_FAST_ARITH
#define MBM_HD __host__ __device__ __forceinline__
#include "mbm_adjoint_math.cuh"   // primitive-form Conservative and Grad-13 flux
#include "mbm_newton.cuh"
#endif

namespace mbm {
namespace MBM_ARITH {

// the reference's max/min/sgn (src/tools.h:3-17): a > b ? a : b etc.
__device__ __forceinline__ double rmax(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double rmin(double a, double b) { return a < b ? a : b; }
__device__ __forceinline__ double rsgn(double a) { return a == 0 ? 0.0 : (a < 0 ? -1.0 : 1.0); }

// ---------------------------------------------------------------------------
// Correctly rounded division from a shared reciprocal.
//
// Markstein's correction step (P. Markstein, "Computation of elementary functions
// on the IBM RISC System/6000 processor", IBM J. Res. Develop. 34(1):111-119, 1990;
// J.-M. Muller et al., Handbook of Floating-Point Arithmetic, 2nd ed., 2018, ch. 4):
// with r = RN(1/y) and q = RN(x*r), the remainder e = x - q*y is exact in one FMA
// and RN(q + e*r) = RN(x/y), provided x, y and the quotient stay in the normal
// range.  One reciprocal then serves every quotient with the same denominator at
// three FP64 operations each, with the same bits as IEEE x/y.  The quotient is
// formed without a branch; a range flag (integer pipe only: |exponent| < 480 for
// x and y, or x = 0) is collected per function, and a function whose flag is set
// recomputes its quotients with IEEE division in a cold, outlined path.  Zero
// numerators take x*r, the signed zero of x/y.  Checked against x/y on the host
// for 2e8 random operand pairs and by every bitwise parity test.
//
// Fast arithmetic (MBM_FAST_ARITH, MBM_MODE_FAST): the quotient is RN(x*r) without
// the correction, within one unit in the last place of x/y, and no range flag is
// kept (the cold IEEE paths become dead code); the file is then compiled with
// multiply-add contraction.
#if MBM_FAST_ARITH
__device__ __forceinline__ bool mk_in(double) { return true; }

__device__ __forceinline__ double mk_div(double x, double, double r) { return x * r; }
#else
__device__ __forceinline__ bool mk_in(double x) {
  const long long b = __double_as_longlong(x);
  return (((unsigned)(b >> 52) & 0x7ffu) - 543u <= 960u) || ((b << 1) == 0);
}

__device__ __forceinline__ double mk_div(double x, double y, double r) {
  const double q = x * r;
  const double m = fma(fma(-q, y, x), r, q);
  return ((__double_as_longlong(x) << 1) == 0) ? q : m;
}
#endif

__device__ __noinline__ double div_ieee(double x, double y) { return x / y; }

// Reciprocal, square root and lone quotients.  Bitwise: IEEE division and sqrt.
// Fast arithmetic: the refined hardware approximations of mbm_newton.cuh.
#if MBM_FAST_ARITH
using mbm_newton::frcp;
using mbm_newton::fsqrt;
__device__ __forceinline__ double fdiv(double x, double y) { return x * frcp(y); }
#else
__device__ __forceinline__ double fdiv(double x, double y) { return x / y; }
__device__ __forceinline__ double fsqrt(double x) { return sqrt(x); }
#endif

struct Recip {        // 1/y for a denominator shared by several quotients
  double y, r;
  bool bad;           // set when any quotient left the safe range
  __device__ __forceinline__ explicit Recip(double y_) {
    y = y_;
#if MBM_FAST_ARITH
    r = frcp(y_);
#else
    r = __drcp_rn(y_);
#endif
#if MBM_FAST_ARITH
    bad = false;      // no range check: quotients are x * r, no IEEE fallback
#else
    const unsigned e = (unsigned)(__double_as_longlong(y_) >> 52) & 0x7ffu;
    bad = e - 543u > 960u;
#endif
  }
  __device__ __forceinline__ Recip(double y_, double r_) {   // r_ = RN(1/y_), y_ in range
    y = y_;
    r = r_;
    bad = false;
  }
  __device__ __forceinline__ double div(double x) {
    bad |= !mk_in(x);
    return mk_div(x, y, r);
  }
  __device__ __forceinline__ double exact(double x) const { return mk_div(x, y, r); }
};

struct V9 { double v[NV]; };

// Primitive (src/Flux.c:30-56)
__device__ __noinline__ V9 primitive_ieee(V9 u) {
  const double* U = u.v;
  V9 o;
  double* P = o.v;
  const double rho = U[0];
  const double v1 = U[1] / rho, v2 = U[2] / rho;
  const double vs = v1 * v1 + v2 * v2;
  const double th = (2 * U[3] / rho - vs) / 3;
  const double E = U[3];
  const double T11 = U[4] / rho - v1 * v1;
  const double T12 = U[5] / rho - v1 * v2;
  const double T22 = U[6] / rho - v2 * v2;
  P[0] = rho; P[1] = v1; P[2] = v2; P[3] = th;
  P[4] = T11; P[5] = T12; P[6] = T22;
  P[7] = U[7] - E * v1 - rho * (T11 * v1 + T12 * v2);
  P[8] = U[8] - E * v2 - rho * (T12 * v1 + T22 * v2);
  return o;
}

__device__ __forceinline__ void primitive(const double (&U)[NV], double (&P)[NV]) {
  const double rho = U[0];
  Recip R(rho);
  Recip third(3.0, 1.0 / 3.0);
  const double v1 = R.div(U[1]), v2 = R.div(U[2]);
  const double vs = v1 * v1 + v2 * v2;
  const double th = third.div(R.div(2 * U[3]) - vs);
  const double E = U[3];
  const double T11 = R.div(U[4]) - v1 * v1;
  const double T12 = R.div(U[5]) - v1 * v2;
  const double T22 = R.div(U[6]) - v2 * v2;
  P[0] = rho; P[1] = v1; P[2] = v2; P[3] = th;
  P[4] = T11; P[5] = T12; P[6] = T22;
  P[7] = U[7] - E * v1 - rho * (T11 * v1 + T12 * v2);
  P[8] = U[8] - E * v2 - rho * (T12 * v1 + T22 * v2);
  if (__builtin_expect(R.bad || third.bad, 0)) {
    V9 u;
#pragma unroll
    for (int n = 0; n < NV; n++) u.v[n] = U[n];
    const V9 o = primitive_ieee(u);
#pragma unroll
    for (int n = 0; n < NV; n++) P[n] = o.v[n];
  }
}

// moments with an explicit energy (src/Flux.c:65-73, 255-263)
__device__ __forceinline__ void moments_e(double rho, double v1, double v2, double E, double T11,
                                          double T12, double T22, double q1, double q2,
                                          double (&U)[NV]) {
  U[0] = rho;
  U[1] = rho * v1;
  U[2] = rho * v2;
  U[3] = E;
  U[4] = rho * (T11 + v1 * v1);
  U[5] = rho * (T12 + v1 * v2);
  U[6] = rho * (T22 + v2 * v2);
  U[7] = q1 + E * v1 + rho * (T11 * v1 + T12 * v2);
  U[8] = q2 + E * v2 + rho * (T12 * v1 + T22 * v2);
}

// Conservative (src/Flux.c:61-74 with src/primDef.h:9-20)
__device__ __forceinline__ void conservative(const double (&P)[NV], double (&U)[NV]) {
  const double vs = P[1] * P[1] + P[2] * P[2];
  const double E = 0.5 * P[0] * vs + 1.5 * P[0] * P[3];
  moments_e(P[0], P[1], P[2], E, P[4], P[5], P[6], P[7], P[8], U);
}

// Grad-13 flux along x of a moment vector (src/Flux.c:79-119).  D: the division
// policy -- shared reciprocals (fast) or IEEE (cold path).
template <bool IEEE>
__device__ __forceinline__ bool grad13_flux_x_t(const double (&U)[NV], double (&F)[NV]) {
  const double rho = U[0];
  Recip R(rho);
  Recip third(3.0, 1.0 / 3.0);
#define MBM_DIV(D, x) (IEEE ? (x) / D.y : D.div(x))
  const double v1 = MBM_DIV(R, U[1]), v2 = MBM_DIV(R, U[2]);
  const double vs = v1 * v1 + v2 * v2;
  const double th = MBM_DIV(third, MBM_DIV(R, 2 * U[3]) - vs);
  const double E = U[3];
  const double T11 = MBM_DIV(R, U[4]) - v1 * v1;
  const double T12 = MBM_DIV(R, U[5]) - v1 * v2;
  const double T22 = MBM_DIV(R, U[6]) - v2 * v2;
  const double q1 = U[7] - E * v1 - rho * (T11 * v1 + T12 * v2);
  const double q2 = U[8] - E * v2 - rho * (T12 * v1 + T22 * v2);
  const double M111 = MBM_DIV(R, 1.2 * q1);
  const double M121 = MBM_DIV(R, 0.4 * q2), M112 = M121;
  const double M221 = MBM_DIV(R, 0.4 * q1), M122 = M221;
#undef MBM_DIV
  const double R11 = 5 * th * th + 7 * th * (T11 - th);
  const double R12 = 7 * th * T12;
  F[0] = rho * v1;
  F[1] = rho * (T11 + v1 * v1);
  F[2] = rho * (T12 + v1 * v2);
  F[3] = E * v1 + rho * (T11 * v1 + T12 * v2) + q1;
  F[4] = rho * (M111 + 3 * T11 * v1 + v1 * v1 * v1);
  F[5] = rho * (M121 + T11 * v2 + 2 * T12 * v1 + v1 * v2 * v1);
  F[6] = rho * (M221 + T22 * v1 + 2 * T12 * v2 + v2 * v2 * v1);
  F[7] = 2 * (q1 + rho * (T11 * v1 + T12 * v2)) * v1 + E * v1 * v1 +
         rho * (M111 * v1 + M112 * v2) + 0.5 * rho * (T11 * vs + R11);
  F[8] = q2 * v1 + q1 * v2 + rho * (v1 * v2 * (T11 + T22) + 1.5 * T12 * vs) + E * v1 * v2 +
         rho * (M121 * v1 + M122 * v2) + 0.5 * rho * R12;
  return IEEE ? false : (R.bad || third.bad);
}

__device__ __noinline__ V9 grad13_flux_x_ieee(V9 u) {
  double U[NV], F[NV];
#pragma unroll
  for (int n = 0; n < NV; n++) U[n] = u.v[n];
  grad13_flux_x_t<true>(U, F);
  V9 o;
#pragma unroll
  for (int n = 0; n < NV; n++) o.v[n] = F[n];
  return o;
}

__device__ __forceinline__ void grad13_flux_x(const double (&U)[NV], double (&F)[NV]) {
  if (__builtin_expect(grad13_flux_x_t<false>(U, F), 0)) {
    V9 u;
#pragma unroll
    for (int n = 0; n < NV; n++) u.v[n] = U[n];
    const V9 o = grad13_flux_x_ieee(u);
#pragma unroll
    for (int n = 0; n < NV; n++) F[n] = o.v[n];
  }
}

// flux through a face of unit normal (nx, ny): rotate, x-flux, rotate back
// (src/Flux.c:126-172).  The products with 0 and +-1 are kept: they fix the
// signs of zeros exactly as the reference computes them.
__device__ __forceinline__ void flux_normal(const double (&U)[NV], double (&F)[NV], double nx,
                                            double ny) {
  const double tx = ny, ty = -nx;
  double W[NV], G[NV], a, b;
  W[0] = U[0];
  W[1] = U[1] * nx + U[2] * ny;
  W[2] = U[1] * tx + U[2] * ty;
  W[3] = U[3];
  a = U[4] * nx + U[5] * ny;
  b = U[5] * nx + U[6] * ny;
  W[4] = a * nx + b * ny;
  W[5] = a * tx + b * ty;
  a = U[4] * tx + U[5] * ty;
  b = U[5] * tx + U[6] * ty;
  W[6] = a * tx + b * ty;
  W[7] = U[7] * nx + U[8] * ny;
  W[8] = U[7] * tx + U[8] * ty;
  grad13_flux_x(W, G);
  F[0] = G[0];
  F[1] = G[1] * nx + G[2] * tx;
  F[2] = G[1] * ny + G[2] * ty;
  F[3] = G[3];
  a = G[4] * nx + G[5] * tx;
  b = G[5] * nx + G[6] * tx;
  F[4] = a * nx + b * tx;
  F[5] = a * ny + b * ty;
  a = G[4] * ny + G[5] * ty;
  b = G[5] * ny + G[6] * ty;
  F[6] = a * ny + b * ty;
  F[7] = G[7] * nx + G[8] * tx;
  F[8] = G[7] * ny + G[8] * ty;
}

// damping factor of the direct production integration (src/Flux.c:213-223)
template <int FLAG>
__device__ __forceinline__ double rdamp(double z) {
  if (FLAG == -1 || FLAG == 0) return fdiv(1 + 0.5 * z - 0.25 * z * z, 1 + z + 0.25 * z * z);
  if (FLAG == 1) return fdiv(1 + z, 1 + z + 0.25 * z * z);
  if (FLAG == 2) return MBM_FAST_ARITH ? 1.0 : fdiv(1 + 0.5 * z, 1 + 0.5 * z);   // the identity
  return fdiv(1.0, 1 + 0.5 * z);
}

// The collision number z = dt nu0 rho sqrt(theta) / Kn of ProductionsDirect
// (src/Flux.c:230-267 with CollFreq, src/Scenario.c:28-42; nu0 = 1): the same
// expression for every flag, so one evaluation serves all of a cell's flags.  Kn is in
// the safe range (checked when the kernel starts); the numerator's range decides
// between the shared-reciprocal quotient and IEEE division.
__device__ __forceinline__ double coll_of(const double (&P)[NV], double dt, const Recip& Kn) {
  const double nu0 = 1.0;
  const double num = nu0 * P[0] * fsqrt(P[3]);
  return (__builtin_expect(mk_in(num), 1) ? Kn.exact(num) : div_ieee(num, Kn.y)) * dt;
}

// ProductionsDirect (src/Flux.c:230-267) with ExternalForce (src/Scenario.c:28-42;
// force (F, 0)), starting from the primitives P of the input moments, given its damping
// factors d1 = rdamp<FLAG>(z), d2 = rdamp<FLAG>(2z/3).  Writes the relaxed moments.
template <int FLAG>
__device__ __forceinline__ void relax_d(const double (&P)[NV], double (&Out)[NV], double dt, double F,
                                        double d1, double d2) {
  const double rho = P[0], th = P[3];
  double v1 = P[1], v2 = P[2];
  double vs = v1 * v1 + v2 * v2;
  double E = 0.5 * rho * vs + 1.5 * rho * th;
  if (FLAG == 0 || FLAG == 2) {
    const double g0 = F, g1 = 0.0;
    v1 += dt * g0;
    v2 += dt * g1;
    vs = v1 * v1 + v2 * v2;
    E = 0.5 * rho * vs + 1.5 * rho * th;
  }
  const double T11 = d1 * (P[4] - th) + th;
  const double T12 = d1 * P[5];
  const double T22 = d1 * (P[6] - th) + th;
  moments_e(rho, v1, v2, E, T11, T12, T22, d2 * P[7], d2 * P[8], Out);
}

// ProductionsDirect of flag FLAG from the primitives P: writes the relaxed moments,
// returns 0.5*(1 - R(2z/3))
template <int FLAG>
__device__ __forceinline__ double relax(const double (&P)[NV], double (&Out)[NV], double dt,
                                        const Recip& Kn, double F) {
  const double coll = coll_of(P, dt, Kn);
  const double d1 = rdamp<FLAG>(coll);
  const double d2 = rdamp<FLAG>(2.0 / 3 * coll);
  relax_d<FLAG>(P, Out, dt, F, d1, d2);
  return 0.5 * (1 - d2);
}

#if MBM_FAST_ARITH
// Primitive(relax<FLAG>(P)) in primitive form (fast arithmetic): rho and theta kept,
// the velocity pushed by dt F for flags 0 and 2, T_ij - theta delta_ij scaled by
// R(z), q by R(2z/3) -- without forming the moments and dividing by rho again
template <int FLAG>
__device__ __forceinline__ void relax_prim(const double (&P)[NV], double (&Q)[NV], double dt,
                                           const Recip& Kn, double F) {
  const double rho = P[0], th = P[3];
  const double coll = rho * fsqrt(th) * Kn.r * dt;
  const double d1 = rdamp<FLAG>(coll);
  const double d2 = rdamp<FLAG>(2.0 / 3 * coll);
  Q[0] = rho;
  Q[1] = P[1] + ((FLAG == 0 || FLAG == 2) ? dt * F : 0.0);
  Q[2] = P[2];
  Q[3] = th;
  Q[4] = d1 * (P[4] - th) + th;
  Q[5] = d1 * P[5];
  Q[6] = d1 * (P[6] - th) + th;
  Q[7] = d2 * P[7];
  Q[8] = d2 * P[8];
}
#endif

#if MBM_FAST_ARITH
// The damping factors of flags 0 (= -1) and 1 at z and 2z/3 (src/Flux.c:213-223) from
// one reciprocal per argument (fast arithmetic): both share the denominator
// 1 + z + z^2/4 = (1 + z/2)^2, so with w = 1/(1 + z/2)
//   R_0(z) = (1 + z/2 - z^2/4) w^2,   R_1(z) = (1 + z) w^2.
struct Damp01 {
  double d1_0, d2_0;   // flag 0 / -1: R(z), R(2z/3)
  double d1_1, d2_1;   // flag 1
  __device__ __forceinline__ explicit Damp01(double z) {
    const double z2 = 2.0 / 3 * z;
    const double w1 = frcp(fma(0.5, z, 1.0)), w2 = frcp(fma(0.5, z2, 1.0));
    const double s1 = w1 * w1, s2 = w2 * w2;
    d1_0 = fma(z, fma(-0.25, z, 0.5), 1.0) * s1;
    d2_0 = fma(z2, fma(-0.25, z2, 0.5), 1.0) * s2;
    d1_1 = (1.0 + z) * s1;
    d2_1 = (1.0 + z2) * s2;
  }
};

// the moments of relax<-1>(P) (ProductionsDirect without the force, src/Flux.c:230-267)
// given its damping factors d1 = R(z), d2 = R(2z/3) (fast arithmetic)
__device__ __forceinline__ void relaxed_moments(const double (&P)[NV], double d1, double d2,
                                                double (&Out)[NV]) {
  const double rho = P[0], v1 = P[1], v2 = P[2], th = P[3];
  const double E = rho * fma(0.5, fma(v1, v1, v2 * v2), 1.5 * th);
  moments_e(rho, v1, v2, E, fma(d1, P[4] - th, th), d1 * P[5], fma(d1, P[6] - th, th), d2 * P[7], d2 * P[8],
            Out);
}

// relax<2>(Primitive(U)) in moment form (fast arithmetic): flag 2 leaves T and q as
// they are (R = 1), so only the push of the velocity by g = dt F changes the moments:
//   U1 + rho g,  E + g (U1 + rho g/2),  U4 + g (2 U1 + rho g),  U5 + g U2,
//   U7 + g (E + U4 + g (3 U1 + rho g)/2),  U8 + g (U5 + g U2/2)   (E = U3)
// -- no Primitive, no division
__device__ __forceinline__ void push_moments(const double (&U)[NV], double g, double (&R)[NV]) {
  const double rg = U[0] * g;
  R[0] = U[0];
  R[1] = U[1] + rg;
  R[2] = U[2];
  R[3] = fma(g, fma(0.5, rg, U[1]), U[3]);
  R[4] = fma(g, fma(2.0, U[1], rg), U[4]);
  R[5] = fma(g, U[2], U[5]);
  R[6] = U[6];
  R[7] = fma(g, U[3] + U[4] + 0.5 * g * fma(3.0, U[1], rg), U[7]);
  R[8] = fma(g, fma(0.5 * g, U[2], U[5]), U[8]);
}
// The same push applies to any moment vector whose temperature and heat flux stay
// fixed: relax<0>(P) = push_moments(relax<-1>(P), dt F), flag 0 differing from flag
// -1 only by the force acting on the velocity before the moments are formed.
#endif

// only the CFL share of relax<FLAG> (same z, same factor)
template <int FLAG>
__device__ __forceinline__ double relax_cfl(const double (&P)[NV], double dt, const Recip& Kn) {
  return 0.5 * (1 - rdamp<FLAG>(2.0 / 3 * coll_of(P, dt, Kn)));
}

// Limit1 (src/Limiter.c:26-59)
__device__ __forceinline__ double superbee_phi(double r) {
  if (r < 0.0) return 0.0;
  if (r < 0.5) return 2 * r;
  if (r < 1.0) return 1.0;
  if (r < 2.0) return r;
  return 2.0;
}

template <int LIM>
__device__ __forceinline__ double limit(double d1, double d2) {
  if (LIM == 0) return 0.0;
  if (LIM == 1) return 0.5 * (d1 + d2);
  if (LIM == 2) return 0.5 * (rsgn(d1) + rsgn(d2)) * rmin(fabs(d1), fabs(d2));
  if (LIM == 3) return d1 * superbee_phi(fdiv(d2, d1));
  const double eps = 1.0e-10;
  const double w1 = fabs(d1) + eps, w2 = fabs(d2) + eps;
  return fdiv(w1 * d2 + w2 * d1, w1 + w2);
}

#if MBM_FAST_ARITH
// Conservative(P) and the Grad-13 flux along x of the same state (src/Flux.c:61-119
// in primitive variables; fast arithmetic).  The flux's first four components are
// moments (F0..F3 = U1, U4, U5, U7) and the others are regrouped around them:
//   F4 = U1 (3 T11 + u^2) + 6/5 q1
//   F5 = v U4 + 2 u rho T12 + 2/5 q2,   F6 = u U6 + 2 v rho T12 + 2/5 q1
//   F7 = u (2 U7 - E u + 6/5 q1) + 2/5 q2 v + rho/2 (T11 (|v|^2 + 7 theta) - 2 theta^2)
//   F8 = 7/5 (q2 u + q1 v) + u v (rho (T11 + T22) + E) + rho T12 (3/2 |v|^2 + 7/2 theta)
// (E = U3; M111 = 6/5 q1/rho, M112 = M121 = 2/5 q2/rho, M122 = M221 = 2/5 q1/rho).
__device__ __forceinline__ void cons_flux_x(const double (&P)[NV], double (&U)[NV], double (&F)[NV]) {
  const double r = P[0], u = P[1], v = P[2], th = P[3];
  const double T11 = P[4], T12 = P[5], T22 = P[6], q1 = P[7], q2 = P[8];
  const double vs = u * u + v * v;
  const double E = 0.5 * r * vs + 1.5 * r * th;
  U[0] = r;
  U[1] = r * u;
  U[2] = r * v;
  U[3] = E;
  U[4] = r * (T11 + u * u);
  U[5] = r * (T12 + u * v);
  U[6] = r * (T22 + v * v);
  U[7] = q1 + E * u + r * (T11 * u + T12 * v);
  U[8] = q2 + E * v + r * (T12 * u + T22 * v);
  const double q1a = 1.2 * q1, q1b = 0.4 * q1, q2b = 0.4 * q2;
  const double rT12 = r * T12, t2 = rT12 + rT12;
  F[0] = U[1];
  F[1] = U[4];
  F[2] = U[5];
  F[3] = U[7];
  F[4] = fma(U[1], fma(3.0, T11, u * u), q1a);
  F[5] = fma(v, U[4], fma(u, t2, q2b));
  F[6] = fma(u, U[6], fma(v, t2, q1b));
  F[7] = fma(u, fma(-E, u, 2.0 * U[7]) + q1a,
             fma(q2b, v, 0.5 * r * fma(T11, vs + 7.0 * th, -2.0 * th * th)));
  F[8] = fma(1.4, fma(q2, u, q1 * v), fma(u * v, fma(r, T11 + T22, E), rT12 * fma(1.5, vs, 3.5 * th)));
}

// FnumHLLE (src/Flux.c:308-379) in primitive form (fast arithmetic): the Grad-13
// flux straight from the face states -- no Conservative -> Primitive round trip and
// no rotations (a y face swaps the x and y components, which is what the rotation
// to the normal (0,1) amounts to); c = 2 sqrt(5/3 theta) as sqrt(20/3 theta).  The
// wave speeds and the coefficients of
//   (lamR fL - lamL fR + lamL lamR (UR - UL)) / alpha
// come first, then each side's moments and flux are formed and added in turn, so one
// side's vectors are live at a time (alpha = 0, both speeds 0: the mean of the two
// fluxes, coefficients 1/2, -1/2, 0).  Mathematically the bitwise version below; the
// rounding differs.
template <int DIR>
__device__ __forceinline__ double hll(const double (&PL_)[NV], const double (&PR_)[NV],
                                      double (&flx)[NV]) {
  double PL[NV], PR[NV];
  if (DIR == 2) {
    mbm_adj::swap_xy(PL_, PL);
    mbm_adj::swap_xy(PR_, PR);
  } else {
#pragma unroll
    for (int n = 0; n < NV; n++) { PL[n] = PL_[n]; PR[n] = PR_[n]; }
  }
  const double cR = fsqrt(20.0 / 3 * PR[3]);
  const double cL = fsqrt(20.0 / 3 * PL[3]);
  const double vR = PR[1], vL = PL[1];
  const double cMax = fabs(0.5 * (vL + vR)) + rmax(cR, cL);
  const double lamL = rmin(vL - cL, 0.0);
  const double lamR = rmax(vR + cR, 0.0);
  const double alph = lamR - lamL;
  const double ra = frcp(alph);
  const bool pos = alph > 0.0;
  const double a = lamR * ra, b = lamL * ra;
  const double ca = pos ? a : 0.5, cb = pos ? b : -0.5, cc = pos ? lamL * a : 0.0;
  double U[NV], F[NV], f[NV];
  cons_flux_x(PL, U, F);
#pragma unroll
  for (int n = 0; n < NV; n++) f[n] = fma(-cc, U[n], ca * F[n]);
  cons_flux_x(PR, U, F);
#pragma unroll
  for (int n = 0; n < NV; n++) f[n] = fma(cc, U[n], fma(-cb, F[n], f[n]));
  if (DIR == 2) {
    mbm_adj::swap_xy(f, flx);
  } else {
#pragma unroll
    for (int n = 0; n < NV; n++) flx[n] = f[n];
  }
  return cMax;
}
#else
// FnumHLLE (src/Flux.c:308-379) for a face with left/right primitives.
// DIR = 1: x face (normal (1,0)), DIR = 2: y face (normal (0,1)).  The
// diffusive scale FFlux/GFlux return is 0, so lamDiff(0/(cMax*dx)) is 1 for
// every cMax and cMax/1.0 == cMax: the division is omitted without changing a bit.
template <int DIR>
__device__ __forceinline__ double hll(const double (&PL)[NV], const double (&PR)[NV],
                                      double (&flx)[NV]) {
  constexpr double nx = DIR == 1 ? 1.0 : 0.0, ny = DIR == 1 ? 0.0 : 1.0;
  const double cR = 2.0 * sqrt(5.0 / 3 * PR[3]);
  const double cL = 2.0 * sqrt(5.0 / 3 * PL[3]);
  double UL[NV], UR[NV], fL[NV], fR[NV];
  conservative(PL, UL);
  flux_normal(UL, fL, nx, ny);
  conservative(PR, UR);
  flux_normal(UR, fR, nx, ny);
  const double vR = PR[DIR], vL = PL[DIR];
  const double cMax = fabs(0.5 * (vL + vR)) + rmax(cR, cL);
  const double lamL = rmin(vL - cL, 0.0);
  const double lamR = rmax(vR + cR, 0.0);
  const double alph = lamR - lamL;
  if (alph > 0.0) {
    Recip A(alph);
    double num[NV];
#pragma unroll
    for (int n = 0; n < NV; n++) {
      num[n] = lamR * fL[n] - lamL * fR[n] + lamL * lamR * (UR[n] - UL[n]);
      flx[n] = A.div(num[n]);
    }
    if (__builtin_expect(A.bad, 0)) {
#pragma unroll
      for (int n = 0; n < NV; n++) flx[n] = div_ieee(num[n], alph);
    }
  } else {
#pragma unroll
    for (int n = 0; n < NV; n++) flx[n] = 0.5 * (fL[n] + fR[n]);
  }
  return cMax;
}
#endif

}  // namespace MBM_ARITH
}  // namespace mbm
