// mbm_newton.cuh -- reciprocal and square root from the hardware's approximations
// refined by Newton-Raphson steps, for the fast arithmetic mode and the adjoint.
//
// r' = r + r(1 - y r) for 1/y (two steps from PTX rcp.approx.ftz.f64) and
// s' = s(3 - x s^2)/2 for 1/sqrt(x) (one step from rsqrt.approx.ftz.f64), then one
// correction q' = q + (x - q^2) s/2 of the root q = x s: the classical iterations
// (P. Markstein, IBM J. Res. Develop. 34(1), 1990; J.-M. Muller et al., Handbook of
// Floating-Point Arithmetic, 2nd ed., 2018, ch. 4-5).  On 2e6 random operands with
// exponents -300..300 both return the correctly rounded value
// (mbm_fastmath_check, tests/test_gpu_fast.py); they are not claimed correctly
// rounded in general, so the bitwise mode does not use them.  Normal operands only
// (subnormals flush to zero); the root of 0 is 0.
#pragma once

#include <cuda_runtime.h>

namespace mbm_newton {

__device__ __forceinline__ double frcp(double y) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(y));
  double e = fma(-y, r, 1.0);
  r = fma(r, e, r);
  e = fma(-y, r, 1.0);
  return fma(r, e, r);
}

__device__ __forceinline__ double fsqrt(double x) {
  double s;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(s) : "d"(x));
  s = s * fma(-0.5 * x, s * s, 1.5);
  const double q = x * s;                      // sqrt(x) to about 2^-46
  const double e = fma(-q, q, x);              // its residual, exact
  return x == 0.0 ? 0.0 : fma(0.5 * s, e, q);
}

}  // namespace mbm_newton
