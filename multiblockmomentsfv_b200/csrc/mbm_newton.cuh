// mbm_newton.cuh -- reciprocal and square root from the hardware's approximations
// refined by one third-order step, for the fast arithmetic mode and the adjoint.
//
// frcp: with r0 from PTX rcp.approx.ftz.f64 and e = 1 - y r0 (one FMA), 1/y =
// r0 / (1 - e) = r0 (1 + e + e^2 + ...); the step r0 + r0 (e + e^2) leaves the
// truncation r0 e^3 (the approximation's |e| is about 2^-20, so below 2^-60).
// fsqrt: with s0 from rsqrt.approx.ftz.f64 and e = 1 - x s0^2, sqrt(x) =
// x s0 (1 - e)^(-1/2) = x s0 (1 + e/2 + 3e^2/8 + ...), the step to the second order
// in e.  Both are truncated Taylor series of the classical iterations (P. Markstein,
// IBM J. Res. Develop. 34(1), 1990; J.-M. Muller et al., Handbook of Floating-Point
// Arithmetic, 2nd ed., 2018, ch. 4-5).  Checked against correctly rounded results on
// 2e6 random operands with exponents -300..300 (mbm_fastmath_check,
// tests/test_gpu_fast.py): both within one unit in the last place; not claimed
// correctly rounded, so the bitwise mode does not use them.  Normal operands only
// (subnormals flush to zero); the root of 0 is 0.
#pragma once

#include <cuda_runtime.h>

namespace mbm_newton {

__device__ __forceinline__ double frcp(double y) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(y));
  const double e = fma(-y, r, 1.0);
  return fma(r, fma(e, e, e), r);
}

__device__ __forceinline__ double fsqrt(double x) {
  double s;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(s) : "d"(x));
  const double q = x * s;
  const double e = fma(-q, s, 1.0);
  const double t = e * fma(0.375, e, 0.5);
  return x == 0.0 ? 0.0 : fma(q, t, q);
}

}  // namespace mbm_newton
