// mbm_internal.h -- device data structures shared by the kernels and the host side.
//
// HBM layout (one allocation per physical layer): every block stores its nine
// moments as nine planes (structure of arrays) of nyp rows x pitch doubles, with
// cell (I, J) of the padded grid (I, J = 0 .. nxp-1 / nyp-1, ghosts included) at
// element J*pitch + I + 1.  The leading pad column puts the first column a warp
// strip reads (I0 - 2, with I0 = 1 + 28k) on a 32-byte sector boundary; pitch is a
// multiple of 4 doubles so every row starts on one too.
//
// Physical layers: buf[0], buf[1] hold DATA and NEW, swapped by index when a step
// is accepted (the reference copies NEW into DATA, src/Main.c:236-240); buf[2] is
// TMP.  Each case keeps the index of its DATA buffer in CaseDev::cur.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>

namespace mbm {

constexpr int NV = 9;           // moments per cell (src/defs.h:11)
constexpr int NG = 3;           // ghost layers per edge (src/defs.h:14)
constexpr int STRIP = 28;        // output columns per warp strip (32 lanes - 2 - 2 halo)
constexpr int CTA_WARPS = 4;     // warps per CTA of the persistent stage kernel
constexpr int MAX_TRACE = 4096;  // progress records kept per case and Steps call

enum LayerSel : int { SEL_CUR = 0, SEL_OTHER = 1, SEL_TMP = 2 };

struct BlockDev {
  int nxp, nyp;        // padded extents (nx+6, ny+6)
  int pitch;           // row stride in doubles
  int case_id;
  long long off;       // element offset of the block's first plane in a layer buffer
  long long plane;     // elements per moment plane
  double dx, dy;
};

struct Work {          // one warp strip segment: columns [I0, I0+28), face rows [J0, J1)
  int blk, I0, J0, J1;
};

constexpr int GHOST_REMOTE = 1 << 18;   // src_blk_flags: src indexes the receive buffer

struct GhostEntry {    // final value of one ghost cell after the two-sweep fill
  int dst_blk;
  int dst;             // element index (J*pitch + I + 1) in block dst_blk
  int src;             // >= 0: element index in block src_blk; < 0: Dirichlet row -(src+1)
  int src_blk_flags;   // src_blk | (x-wall flip << 16) | (y-wall flip << 17) | GHOST_REMOTE
};

// The ghost fill scattered from its sources (SetBoundary fused into the stage kernel):
// one entry per ghost cell, listed under the work item that writes its owner -- the
// interior cell it is copied from, or, for a Dirichlet ghost, the interior cell nearest
// to it
struct GhostScatter {
  long long dst;       // element index of the ghost cell in the layer (block offset included)
  long long plane;     // plane stride of the ghost cell's block
  int src;             // element index of the owner in its block (the work item's block)
  int flags;           // x-wall flip | y-wall flip << 1
  int drow;            // >= 0: Dirichlet row (the value comes from the table); -1: a copy of the owner
  int pad_;
};

struct CaseDev {       // per-case step controller (src/Main.c:189-244)
  double t, tend, dt, CFLmax, CFLreg, Kn, F;
  double cfl_last;
  int limiter, cur;
  int nstep, nrej, attempts, max_attempts, step_cap;
  int done, status;
  int show_every, trace_n;
  int blk0, nblk;      // the case's blocks are blk0 .. blk0+nblk-1
  int nonfinite;       // set by a stage that wrote a NaN or infinity
  int ckpt_every;      // > 0: copy DATA to ckpt[nstep / ckpt_every] every that many steps
  int dtlog_cap;       // accepted dt values recorded into dtlog (adjoint runs)
  double* dtlog;
  double* ckpt;        // checkpoint layers (layer_elems doubles each)
  int accepted;        // the controller accepted the attempt just made
  // adjoint runs: the states D_a .. D_{b-1} and stage-1 states T_a .. T_{b-1} of the last
  // checkpoint segment [a, b), kept as the forward run makes them (not null: on)
  int tail_a, tail_b;
  double* tail_d;
  double* tail_t;
};

struct StageArgs {
  const BlockDev* blk;
  const Work* work;
  int nwork;
  CaseDev* cases;
  double* buf[3];
  unsigned long long* lam;   // [block][stage][3]: max lambda_x, lambda_y, CFL_prod bits
  int* queue;                // work-item counter of this stage (zero before the launch)
  int sel_in, sel_d0, sel_out;
  int heun;
  // the relaxation term (flag -1) of the stage-1 input (layer layout, interior cells),
  // written by stage 1 (fast arithmetic: never null, stage 1 reads it back; bitwise:
  // null leaves it unwritten); rlx_read = 1 makes stage 2 read it in place of forming
  // it again from Data0 (set only when the stage 1 of the same attempt, on the same
  // Data0, ran just before)
  double* rlx;
  int rlx_read;
  // fast arithmetic, stage 2 with rlx_read: 2 tensor maps (CUtensorMap, 128 bytes each)
  // per block, over the TMP layer and the relaxation layer, 3-D (column, row, moment
  // plane); not null: the window slots are filled by bulk tensor copies (TMA) instead
  // of per-lane cp.async
  const void* tmap;
  // the ghost fill of the output layer, done by the work items that write the owners
  // (null: not done here; a separate gather fills the ghosts).  gs_item[w]: the first
  // entry of gs and the entry count of work item w
  const int2* gs_item;
  const GhostScatter* gs;
  const double* dirichlet;   // Dirichlet rows (9 values each)
  // failure-detection test only (null otherwise): a device flag; while it is 1, warp 0 of
  // CTA 0 consumes it (sets it to 0) and withholds its first bulk copy, so that its
  // bounded wait runs out -- one launch, also when the launch is replayed from a graph
  int* tma_drop;
};

constexpr int TMAP_BYTES = 128;   // sizeof(CUtensorMap)

struct AdjArgs {       // one stage of the discrete adjoint (mbm_adjoint.cu)
  const BlockDev* blk;
  int nblk;
  const double* x;       // stage input layer (all cells)
  const double* d0;      // Data0 (stage 2)
  const double* lout;    // adjoint of the stage output (interior cells)
  double* lx;            // += adjoint of the stage input (all cells)
  double* ld0;           // += adjoint of Data0 (stage 2)
  double* P;             // projected primitives of the stage input (layer layout)
  double* Pb;            // not null: the cell pass split in two, Pb the reconstruction adjoint between them
  double* knb;           // += dJ/dKn
  double dt, Kn, F;
  int limiter, heun;
  const Work* work;      // row-marching pass: strips of ASTRIP columns x row segments
  int nwork;
  int* queue;            // its work-item counter (zero before the launch)
};

constexpr int ASTRIP = 26;   // output columns of one warp of the row-marching adjoint

__host__ __device__ inline int phys_layer(int sel, int cur) {
  return sel == SEL_CUR ? cur : (sel == SEL_OTHER ? 1 - cur : 2);
}

// buf[k] by selects: indexing a kernel parameter's array with a run-time k makes the
// compiler copy the whole parameter block to local memory (measured: 120 bytes per
// thread in the stage kernel, 5 % of its time)
__host__ __device__ inline double* layer_ptr(double* const (&buf)[3], int k) {
  return k == 0 ? buf[0] : (k == 1 ? buf[1] : buf[2]);
}

// Programmatic dependent launch of the step loop's kernels (stage, ghost fill,
// controller, checkpoint): a kernel launched with it is set up while the kernel before
// it on the stream finishes.  pdl_enter, at the top of each of those kernels, waits
// until the kernel before it has completed with its memory visible -- before it reads or
// writes anything; a no-op in a kernel launched without it.  The kernels do not release
// their dependents early (griddepcontrol.launch_dependents at entry): dependents that
// took SM slots while a persistent stage grid drained made a 4 x 256^2 step 14 % slower.
__device__ __forceinline__ void pdl_enter() {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 900
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
#endif
}

// host: whether the launches this thread makes use it (set around a step attempt)
extern thread_local bool tl_pdl;

// a launch of one of the step loop's kernels, with the programmatic-serialization
// attribute when tl_pdl is set
template <typename... KArgs, typename... Args>
inline cudaError_t launch_k(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                            Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  if (tl_pdl) {
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
  }
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

}  // namespace mbm
