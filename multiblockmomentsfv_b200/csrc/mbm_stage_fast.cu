// mbm_stage_fast.cu -- the Heun stage kernel in fast arithmetic (MBM_MODE_FAST):
// the same kernel source as the bitwise instantiation, with quotients from a shared
// reciprocal without Markstein's correction and multiply-add contraction (this
// file is compiled with -fmad=true).  Results differ from the reference in the last
// bits of single operations; the mode is held to the reference within 1e-10
// relative per field after one step and 1e-8 at the end time.
#define MBM_ARITH fastmath
#define MBM_FAST_ARITH 1
#include "mbm_stage.cuh"

namespace mbm {
namespace fastmath {
__global__ void fastmath_check_kernel(const double* __restrict__ x, int n, double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[2 * i] = frcp(x[i]);
  out[2 * i + 1] = fsqrt(x[i]);
}
}  // namespace fastmath
}  // namespace mbm

// The fast-arithmetic reciprocal and square root of n device values (out: 2n values,
// 1/x and sqrt(x) interleaved), for checking them against correctly rounded results.
extern "C" int mbm_fastmath_check(const double* x, int n, double* out) {
  if (!x || !out || n < 0) return 1;   // MBM_EINVAL
  if (n == 0) return 0;
  mbm::fastmath::fastmath_check_kernel<<<(n + 255) / 256, 256>>>(x, n, out);
  return cudaDeviceSynchronize() == cudaSuccess ? 0 : 4;   // MBM_OK / MBM_ECUDA
}
