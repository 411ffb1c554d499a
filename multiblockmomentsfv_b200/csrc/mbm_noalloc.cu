// mbm_noalloc.cu -- mbm_stage_noalloc: one Heun stage on caller-owned device
// buffers, with every piece of scratch the stage kernel needs held in one
// file-scope device array instead of allocated memory.
//
// Some callers cannot allocate device memory at all: a host framework whose
// memory pool owns the whole GPU (any cudaMalloc outside the pool breaks its
// accounting or fails), and real-time or certified loops that fix every
// allocation at start-up.  They hold their own moment buffers and only need
// the computation.  The context API (mbm_create) allocates; this entry point does
// not.
//
// The scratch lives in g_noalloc_scratch (NOALLOC_SCRATCH_BYTES below).  Every GPU
// that loads this library holds that array until the process exits.  In host code
// the array's name is only a host-side stand-in, so its device address is taken
// with cudaGetSymbolAddress, once per device, with that device current, on the
// first call made on that device; that first call should therefore come before any
// stream capture begins.  All calls share the array and it keeps the last call's
// contents: each call clears the parts that must start at zero (the work counter,
// the CFL maxima and the non-finite flag).  Two calls that overlap on the GPU (on
// different streams, or from different host threads) race on the array.  Each call
// waits for its stream before it returns (it reads the CFL maxima and the
// non-finite flag back to the host).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/mbm_b200.h"
#include "mbm_internal.h"

namespace mbm {
namespace bitwise {
cudaError_t launch_stage(int lim, const StageArgs& a, int grid, cudaStream_t s);
int stage_ctas_per_sm(int heun);
int stage_cta_warps();
}
void set_global_error(const std::string& msg);   // read back by mbm_last_error(NULL)
}  // namespace mbm

using namespace mbm;

namespace {

// scratch layout (bytes): controller | work counter | CFL maxima | block table | work table
constexpr int NOALLOC_MAX_BLOCKS = 64;
constexpr size_t OFF_CASE = 0;
constexpr size_t OFF_QUEUE = 256;
constexpr size_t OFF_LAM = 512;
constexpr size_t OFF_BLK = OFF_LAM + sizeof(unsigned long long) * 6 * NOALLOC_MAX_BLOCKS;
constexpr size_t OFF_WORK = (OFF_BLK + sizeof(BlockDev) * NOALLOC_MAX_BLOCKS + 255) & ~size_t(255);
constexpr size_t NOALLOC_SCRATCH_BYTES = 320 * 1024;
constexpr int NOALLOC_MAX_WORK = (int)((NOALLOC_SCRATCH_BYTES - OFF_WORK) / sizeof(Work));
constexpr int NOALLOC_SEGMENT_ROWS = 32;

static_assert(sizeof(CaseDev) <= OFF_QUEUE - OFF_CASE, "controller slot too small");
// the capacity the header and the error message state; a layout change must update them
static_assert(NOALLOC_MAX_WORK == 20064, "work-item capacity differs from the documented 20,064");
static_assert(NOALLOC_MAX_BLOCKS == 64, "block capacity differs from the documented 64");

__device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

std::mutex g_mu;
unsigned char* g_scratch_ptr[256];        // device address of the array, per device

thread_local Work h_work[NOALLOC_MAX_WORK];
thread_local BlockDev h_blk[NOALLOC_MAX_BLOCKS];
thread_local unsigned long long h_lam[6 * NOALLOC_MAX_BLOCKS];
thread_local CaseDev h_case;
thread_local int h_nonfinite;

int fail(int code, const std::string& msg) {
  set_global_error(msg);
  return code;
}

// [p, p + n doubles) and [q, q + n doubles) share an element
bool overlaps(const double* p, const double* q, long long n) {
  const uintptr_t a = (uintptr_t)p, b = (uintptr_t)q, len = (uintptr_t)n * sizeof(double);
  return a < b + len && b < a + len;
}

}  // namespace

extern "C" int mbm_stage_noalloc(const mbm_block_desc* blocks, int nblocks, const double* in,
                                 const double* data0, double* out, double Kn, double F, int limiter,
                                 double dt, int heun, double* cfl, void* stream) {
  if (!blocks || nblocks < 1 || !in || !out || (heun == 1 && !data0) || (heun != 0 && heun != 1))
    return fail(MBM_EINVAL, "mbm_stage_noalloc: bad argument");
  if (nblocks > NOALLOC_MAX_BLOCKS)
    return fail(MBM_EINVAL, "mbm_stage_noalloc: more than " + std::to_string(NOALLOC_MAX_BLOCKS) + " blocks");
  if (limiter < 0 || limiter > 4 || !(Kn > 1e-100 && Kn < 1e100) || !(dt > 0) || !std::isfinite(dt))
    return fail(MBM_EINVAL, "mbm_stage_noalloc: bad limiter, Kn or dt (dt must be positive and finite)");
  cudaStream_t s = (cudaStream_t)stream;

  // block table in the layout of include/mbm_b200.h, and the warp work items
  long long off = 0;
  int nwork = 0;
  for (int b = 0; b < nblocks; b++) {
    const mbm_block_desc& d = blocks[b];
    if (d.nx < 1 || d.ny < 1 || d.nx > (1 << 20) || d.ny > (1 << 20) ||
        !(d.dx > 1e-100 && d.dx < 1e100) || !(d.dy > 1e-100 && d.dy < 1e100))
      return fail(MBM_EINVAL, "mbm_stage_noalloc: bad block extents");
    BlockDev& h = h_blk[b];
    h.nxp = d.nx + 2 * NG;
    h.nyp = d.ny + 2 * NG;
    h.pitch = (h.nxp + 1 + 3) & ~3;
    h.case_id = 0;
    h.plane = ((long long)h.pitch * h.nyp + 31) & ~31LL;
    h.off = off;
    h.dx = d.dx;
    h.dy = d.dy;
    off += h.plane * NV;
    const int nfx = h.nxp - 3, nfy = h.nyp - 3;
    const int strips = (nfx + STRIP - 1) / STRIP;
    const int segs = (nfy + NOALLOC_SEGMENT_ROWS - 1) / NOALLOC_SEGMENT_ROWS;
    if (nwork + (long long)strips * segs > NOALLOC_MAX_WORK)
      return fail(MBM_EINVAL, "mbm_stage_noalloc: blocks exceed the scratch limit (" +
                                  std::to_string(NOALLOC_MAX_WORK) + " warp work items: " +
                                  std::to_string(STRIP) + "-column strips x " +
                                  std::to_string(NOALLOC_SEGMENT_ROWS) + "-row segments)");
    for (int sg = 0; sg < segs; sg++) {
      const int J0 = 1 + (int)((long long)nfy * sg / segs);
      const int J1 = 1 + (int)((long long)nfy * (sg + 1) / segs);
      for (int k = 0; k < strips; k++) h_work[nwork++] = Work{b, 1 + STRIP * k, J0, J1};
    }
  }
  // the kernel reads in (and data0) while other warps write out: out must share no
  // element with either (an in-place stage would read cells already overwritten)
  if (overlaps(out, in, off) || (heun == 1 && overlaps(out, data0, off)))
    return fail(MBM_EINVAL, "mbm_stage_noalloc: out overlaps in or data0 (an in-place stage is not allowed)");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) return fail(MBM_ENODEV, "no CUDA device");
  memset(&h_case, 0, sizeof h_case);
  h_case.dt = dt;
  h_case.Kn = Kn;
  h_case.F = F;
  h_case.limiter = limiter;
  h_case.cur = 0;              // buf[0] = in, buf[1] = out, buf[2] = data0
  h_case.done = 0;
  h_case.nblk = nblocks;

  unsigned char* scratch = nullptr;
  {
    std::lock_guard<std::mutex> g(g_mu);
    if (!g_scratch_ptr[dev]) {
      cudaError_t e = cudaGetSymbolAddress((void**)&g_scratch_ptr[dev], g_noalloc_scratch);
      if (e != cudaSuccess) {
        g_scratch_ptr[dev] = nullptr;
        return fail(MBM_ECUDA, cudaGetErrorString(e));
      }
    }
    scratch = g_scratch_ptr[dev];
  }
  CaseDev* dcase = (CaseDev*)(scratch + OFF_CASE);
  int* dqueue = (int*)(scratch + OFF_QUEUE);
  unsigned long long* dlam = (unsigned long long*)(scratch + OFF_LAM);
  BlockDev* dblk = (BlockDev*)(scratch + OFF_BLK);
  Work* dwork = (Work*)(scratch + OFF_WORK);

  cudaError_t e = cudaSuccess;
  if (!e) e = cudaMemcpyAsync(dcase, &h_case, sizeof(CaseDev), cudaMemcpyHostToDevice, s);
  if (!e) e = cudaMemcpyAsync(dblk, h_blk, sizeof(BlockDev) * nblocks, cudaMemcpyHostToDevice, s);
  if (!e) e = cudaMemcpyAsync(dwork, h_work, sizeof(Work) * nwork, cudaMemcpyHostToDevice, s);
  if (!e) e = cudaMemsetAsync(dqueue, 0, sizeof(int), s);
  if (!e) e = cudaMemsetAsync(dlam, 0, sizeof(unsigned long long) * 6 * nblocks, s);
  int sm = 0;
  if (!e) e = cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev);
  if (e) return fail(MBM_ECUDA, cudaGetErrorString(e));

  StageArgs a{};
  a.blk = dblk;
  a.work = dwork;
  a.nwork = nwork;
  a.cases = dcase;
  a.buf[0] = const_cast<double*>(in);
  a.buf[1] = out;
  a.buf[2] = const_cast<double*>(heun ? data0 : in);
  a.lam = dlam;
  a.queue = dqueue;
  a.heun = heun;
  a.sel_in = SEL_CUR;
  a.sel_d0 = heun ? SEL_TMP : SEL_CUR;
  a.sel_out = SEL_OTHER;
  const int cw = bitwise::stage_cta_warps();
  const long long grid = std::min<long long>((nwork + cw - 1) / cw, (long long)sm * bitwise::stage_ctas_per_sm(heun));
  e = bitwise::launch_stage(limiter, a, (int)grid, s);
  if (!e) e = cudaMemcpyAsync(h_lam, dlam, sizeof(unsigned long long) * 6 * nblocks, cudaMemcpyDeviceToHost, s);
  if (!e) e = cudaMemcpyAsync(&h_nonfinite, (const unsigned char*)dcase + offsetof(CaseDev, nonfinite), sizeof(int),
                              cudaMemcpyDeviceToHost, s);
  if (!e) e = cudaStreamSynchronize(s);
  if (e) return fail(MBM_ECUDA, cudaGetErrorString(e));
  if (cfl) {
    for (int b = 0; b < nblocks; b++) {      // Update's return value (src/Main.c:395)
      double v[3];
      memcpy(v, h_lam + ((size_t)b * 2 + heun) * 3, sizeof v);
      cfl[b] = dt * v[0] / h_blk[b].dx + dt * v[1] / h_blk[b].dy + v[2];
    }
  }
  // a NaN or infinity written to out: a NaN never enters the maxima above, so the CFL
  // values alone would not show it
  if (h_nonfinite)
    return fail(MBM_ENONFINITE, "mbm_stage_noalloc: the stage wrote a NaN or infinity");
  return MBM_OK;
}
