// mbm_stage_fast.cu -- the Heun stage kernel in fast arithmetic (MBM_MODE_FAST):
// the same kernel source as the bitwise instantiation, with quotients from a shared
// reciprocal without Markstein's correction and multiply-add contraction (this
// file is compiled with -fmad=true).  Results differ from the reference in the last
// bits of single operations; the mode is held to the reference within 1e-10
// relative per field after one step and 1e-8 at the end time.
#define MBM_ARITH fastmath
#define MBM_FAST_ARITH 1
#include "mbm_stage.cuh"
