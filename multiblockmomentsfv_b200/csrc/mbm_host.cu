// mbm_host.cu -- the C ABI (include/mbm_b200.h): context, block validation, the
// resolved ghost map, the warp work table, the device-side step loop as a CUDA
// graph with a conditional while node, and the layer transfers.
#include <cuda.h>            // CUtensorMap and its encoder's types (the encoder is fetched at run time)
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <map>
#include <mutex>
#include <tuple>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <array>
#include <thread>
#include <vector>

#include "../../include/mbm_b200.h"
#include "mbm_internal.h"

namespace mbm {
namespace bitwise {
cudaError_t launch_stage(int lim, const StageArgs& a, int grid, cudaStream_t s);
int stage_ctas_per_sm(int heun);
int stage_cta_warps();
}
namespace fastmath {
cudaError_t launch_stage(int lim, const StageArgs& a, int grid, cudaStream_t s);
int stage_ctas_per_sm(int heun);
int stage_cta_warps();
}
cudaError_t launch_ghost(const BlockDev* blk, const CaseDev* cases, const GhostEntry* map, int n,
                         double* const buf[3], const double* dirichlet, int sel, cudaStream_t s,
                         const double* recv = nullptr);
cudaError_t launch_shard_pack(const BlockDev* blk, const CaseDev* cases, const int2* list, int n,
                              double* const buf[3], int sel, double* send, cudaStream_t s);
cudaError_t launch_shard_cfl(const CaseDev* cases, const BlockDev* blk, int nblk, unsigned long long* lam,
                             double* out, cudaStream_t s);
cudaError_t launch_control_ext(CaseDev* cases, const BlockDev* blk, unsigned long long* lam, double* trace,
                               int* queues, const double* cfl_ext, cudaStream_t s);
cudaError_t launch_control(CaseDev* cases, int ncases, const BlockDev* blk, unsigned long long* lam,
                           double* trace, int* queues, cudaGraphConditionalHandle h, int use_handle,
                           cudaStream_t s);
cudaError_t launch_frozen_prep(CaseDev* cases, const double* ddt, int* queues, cudaStream_t s);
cudaError_t launch_ckpt(const CaseDev* cases, const double* buf0, const double* buf1, const double* buf2,
                        long long layer_elems, int grid, cudaStream_t s);
cudaError_t adjoint_stage(const AdjArgs& a0, long long ncell, double* FLx, double* FRx, double* FLy,
                          double* FRy, cudaStream_t s);
cudaError_t adjoint_ghosts(const BlockDev* blk, const GhostEntry* map, int n, double* l, cudaStream_t s);
cudaError_t adjoint_stage_march(const AdjArgs& a, int grid, cudaStream_t s);
int adjoint_march_ctas();
cudaError_t adjoint_functional(const BlockDev* blk, int nblk, const double* x, double* l, long long ncell,
                               double* part, double* J, int kind, cudaStream_t s);
cudaError_t launch_fill_uniform(double* base, long long plane, cudaStream_t s);
cudaError_t launch_stage_cfl(const BlockDev* blk, int nblk, const CaseDev* cases,
                             unsigned long long* lam, int stage, double* out, cudaStream_t s);
cudaError_t launch_output_fields(const double* src, int nxp, int nyp, int pitch, long long plane, int single,
                                 void* dst, cudaStream_t s);
cudaError_t launch_fields_to_planes(const void* src, int single, int faithful, int nxp, int nyp, int pitch,
                                    long long plane, double* dst, cudaStream_t s);
cudaError_t launch_aos_to_planes(const double* aos, double* dst, int nxp, int nyp, int pitch,
                                 long long plane, cudaStream_t s);
cudaError_t launch_planes_to_aos(const double* src, double* aos, int nxp, int nyp, int pitch,
                                 long long plane, cudaStream_t s);
}  // namespace mbm

using namespace mbm;

static thread_local std::string g_create_error;

namespace mbm {
void set_global_error(const std::string& msg) { g_create_error = msg; }
}  // namespace mbm

struct LimGroup {      // the work items of every block whose case uses one limiter
  int lim, start, count;
  int grid[2];         // persistent grid of each Heun stage
};

struct mbm_ctx {
  mbm_params prm{};
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int nblk = 0, ncase = 0;
  std::vector<mbm_block_desc> desc;  // sync codes global (1-based over all blocks)
  std::vector<int> blk_case;        // case of each block
  std::vector<BlockDev> hblk;
  BlockDev* dblk = nullptr;
  long long layer_elems = 0;
  double* buf[3] = {nullptr, nullptr, nullptr};
  double* rlx = nullptr;            // the relaxation term of Data0 stage 1 stores for stage 2 (a layer)
  void* dtmap = nullptr;            // fast arithmetic: per block, tensor maps of TMP and rlx (stage-2 TMA)
  std::string tma_note;             // why the stage-2 bulk tensor copies are off, if they are
  int* dtma_drop = nullptr;         // failure-detection test: device flag, the next bulk-copy launch withholds one copy
  double* staging = nullptr;        // array-of-structs transfer buffer, one block
  GhostEntry* dghost = nullptr;
  int nghost = 0;
  std::vector<int> dir_off;         // [block*4+side] -> first Dirichlet row, -1 if none
  double* ddir = nullptr;
  int ndir = 0;
  // SetBoundary fused into the stage kernel: the ghost fill of each stage's output
  // scattered by the work items that write its sources (opt-in, MBM_GHOST_SCATTER=1:
  // at 4 x 1024^2 the separate gather launch costs less; never in a sharded context,
  // whose remote ghosts arrive from other ranks)
  bool gscatter = false;
  std::vector<int> gs_cell;          // host: per cell of every block (off / 9 + element), its first owned entry
  std::vector<GhostScatter> gs_ent;  // host: the entries in owner order
  GhostScatter* dgs = nullptr;       // per stage (gs_ent.size() apart): the entries in work-item order
  int2* dgs_item = nullptr;          // per stage (max_items apart): first entry and count of each item
  Work* dwork = nullptr;            // the work tables of the two Heun stages, max_items apart
  long long max_items = 0;
  int nwork[2] = {0, 0};
  std::vector<LimGroup> groups[2];  // limiter groups of each stage's table
  int nsm = 0, cta_warps = CTA_WARPS;   // stage kernel: warps per CTA
  int ctas_per_sm[2] = {1, 1};          // stage kernel: resident CTAs per SM of each Heun stage
  double seg_rows[2] = {0, 0};      // rows per work item of each Heun stage (ceil(rows / seg_rows) segments)
  CaseDev* dcase = nullptr;
  CaseDev* hcase = nullptr;         // pinned mirror, ncase entries
  unsigned long long* dlam = nullptr;
  int* dqueue = nullptr;            // work counters [stage][limiter]
  double* dtrace = nullptr;
  double* dcfl = nullptr;           // per-block stage CFL for mbm_update
  double* hcfl = nullptr;           // pinned
  cudaEvent_t ev = nullptr;
  // limiter groups of one stage run concurrently: forked from `stream`, joined back
  cudaStream_t aux[4] = {};
  // output staged on the device and copied to the host beside the next interval
  double* out_stage = nullptr;
  std::vector<size_t> out_off;     // bytes, per block (room for the Float64 payload)
  cudaStream_t out_stream = nullptr;
  cudaEvent_t out_ev = nullptr;
  cudaEvent_t fork_ev = nullptr, join_ev[4] = {};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  bool host_loop = false;           // MBM_HOST_LOOP=1: drive the step loop from the host
  // the step loop's kernels launched with programmatic dependent launch (MBM_PDL=0: off;
  // off too when a stage runs as several limiter groups on forked streams, or when the
  // step graph cannot be built with it)
  bool pdl = true;
  bool adjoint = false;             // graph body records checkpoints and dt (mbm_params.adjoint)
  bool fast = false;                // MBM_MODE_FAST: the fastmath stage kernel
  // a case split over ranks by block (mbm_create_sharded)
  bool sharded = false;
  std::vector<int> send_counts, recv_counts;
  int nsend = 0, nrecv = 0;
  int2* dsend_list = nullptr;
  double* shard_send = nullptr;
  double* shard_recv = nullptr;
  double* shard_cfl = nullptr;
  std::vector<int> shard_dir_off, shard_nt;   // Dirichlet rows of every block's edges (whole table)
  // adjoint work space (allocated on first use)
  double* adj_buf[9] = {nullptr};   // two adjoint layers, stage-1 adjoint, primitives, 4 face-adjoint layers,
                                    // the reconstruction adjoint between the two halves of the cell pass
  double* adj_ckpt = nullptr;
  double* adj_seg[2] = {nullptr};    // DATA states of a checkpoint segment (two: recomputation of
  double* adj_segT[2] = {nullptr};   //   the next one beside the reversal of this one); stage-1 states
  cudaStream_t adj_rstream = nullptr;   // the recomputation stream (low priority)
  cudaEvent_t adj_ready[2] = {nullptr}, adj_free[2] = {nullptr}, adj_start = nullptr;
  double* adj_dtlog = nullptr;
  double* adj_scal = nullptr;       // [0] dJ/dKn, [1] J
  double* adj_dtrep = nullptr;      // dt values of mbm_replay
  double* adj_part = nullptr;       // per-CTA partial sums of J
  // the row-marching adjoint pass (MBM_ADJ_MARCH=1; the three-pass one is the default)
  bool adj_march = false;
  Work* adj_work = nullptr;
  bool adj_work_ready = false;
  int adj_nwork = 0, adj_grid = 0;
  int* adj_queue = nullptr;
  int adj_nsteps = 0, adj_every = 0, adj_nrep = 0;
  int functional = 0;               // the adjoint's J (mbm_set_functional)
  std::string err;
};

// ------------------------------------------------------------------ helpers --
// timing events of one call, destroyed on every return path
struct LocalEvents {
  cudaEvent_t e[3] = {nullptr, nullptr, nullptr};
  ~LocalEvents() {
    for (cudaEvent_t x : e)
      if (x) cudaEventDestroy(x);
  }
};

static int fail(mbm_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  else g_create_error = msg;
  return code;
}

#define CK(call)                                                                       \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return fail(c, e_ == cudaErrorMemoryAllocation ? MBM_ENOMEM : MBM_ECUDA,         \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                 \
  } while (0)

static double wait_timeout_s() {
  const char* s = getenv("MBM_WAIT_TIMEOUT_S");
  double v = s ? atof(s) : 0.0;
  return v > 0 ? v : 3600.0;
}

// bounded host wait for everything queued on the context's stream so far
static int wait_stream(mbm_ctx* c) {
  cudaError_t e = cudaEventRecord(c->ev, c->stream);
  if (e != cudaSuccess) return fail(c, MBM_ECUDA, std::string("cudaEventRecord: ") + cudaGetErrorString(e));
  const auto t0 = std::chrono::steady_clock::now();
  const double limit = wait_timeout_s();
  int spins = 0;
  for (;;) {
    e = cudaEventQuery(c->ev);
    if (e == cudaSuccess) return MBM_OK;
    if (e != cudaErrorNotReady) return fail(c, MBM_ECUDA, std::string("device: ") + cudaGetErrorString(e));
    const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (el > limit) return fail(c, MBM_ETIMEOUT, "device work did not finish within MBM_WAIT_TIMEOUT_S");
    if (++spins > 64) std::this_thread::sleep_for(std::chrono::microseconds(spins > 1000 ? 500 : 20));
  }
}

static int kind_of(int code) { return code > 0 ? 0 : code == 0 ? 1 : code == -1 ? 2 : 3; }  // sync/open/wall/dirichlet

// blocks of a case are [lo, hi); sync codes are global 1-based block numbers here
static int validate(const mbm_block_desc* b, int n, std::string& why, int lo = 0, int hi = -1) {
  if (!b || n < 1 || n > 65535) { why = "need 1..65535 blocks"; return MBM_EINVAL; }
  if (hi < 0) hi = n;
  for (int i = lo; i < hi; i++) {
    if (b[i].nx < 1 || b[i].ny < 1 || b[i].nx > (1 << 20) || b[i].ny > (1 << 20)) {
      why = "block " + std::to_string(i + 1) + ": bad cell counts"; return MBM_EINVAL;
    }
    if (!(b[i].dx > 1e-100 && b[i].dx < 1e100) || !(b[i].dy > 1e-100 && b[i].dy < 1e100)) {
      why = "block " + std::to_string(i + 1) + ": dx, dy must be in (1e-100, 1e100)"; return MBM_EINVAL;
    }
    for (int s = 0; s < 4; s++) {
      int code = b[i].bc[s];
      if (code > 0 && (code - 1 < lo || code - 1 >= hi)) { why = "block " + std::to_string(i + 1) + ": sync partner " + std::to_string(code) + " does not exist"; return MBM_EINVAL; }
      if (code > 0) {  // conforming interface (src/Boundary.c:101-103)
        const mbm_block_desc& p = b[code - 1];
        bool ok = s < 2 ? p.ny == b[i].ny : p.nx == b[i].nx;
        if (!ok) { why = "block " + std::to_string(i + 1) + ": sync edge extents differ"; return MBM_EINVAL; }
      }
    }
  }
  return MBM_OK;
}

// ---------------------------------------------------------------- ghost map --
// SetBoundary (src/Boundary.c:173-193) run on symbols instead of values: each cell
// holds "interior cell (block, index) times wall signs", "Dirichlet row", or
// "unknown".  Running both sweeps in the reference's order leaves every ghost cell
// with the source its final value comes from; the device then fills all ghosts in
// one gather.  Interior cells never change during the fill, so the gather is
// race-free and its result equals the sequential sweeps bit for bit.
namespace {
struct Sym { int kind, blk, cell, flags; };   // kind 0 cell, 1 Dirichlet row, 2 unknown
struct Resolved { int dst_blk, dst_cell, src, src_blk, flags, remote = -1; };   // remote: receive index
}  // namespace

static int resolve_ghosts(const mbm_block_desc* B, int nb, std::vector<Resolved>& out,
                          std::vector<int>& dir_off, int& ndir, std::string& why) {
  auto nxp = [&](int b) { return B[b].nx + 2 * NG; };
  auto nyp = [&](int b) { return B[b].ny + 2 * NG; };
  std::vector<std::vector<Sym>> S(nb);
  dir_off.assign((size_t)nb * 4, -1);
  ndir = 0;
  for (int b = 0; b < nb; b++) {
    S[b].resize((size_t)nxp(b) * nyp(b));
    for (int J = 0; J < nyp(b); J++)
      for (int I = 0; I < nxp(b); I++) {
        bool inner = I >= NG && I < nxp(b) - NG && J >= NG && J < nyp(b) - NG;
        S[b][(size_t)J * nxp(b) + I] = inner ? Sym{0, b, J * nxp(b) + I, 0} : Sym{2, 0, 0, 0};
      }
    for (int s = 0; s < 4; s++)
      if (kind_of(B[b].bc[s]) == 3) {
        dir_off[b * 4 + s] = ndir;
        ndir += (s < 2 ? nyp(b) : nxp(b)) * NG;
      }
  }
  // cell (I, J) of ghost layer n / source layer k on a side (src/Boundary.c:51-81)
  auto ghost = [&](int b, int side, int ti, int n, int& I, int& J) {
    switch (side) {
      case 0: I = NG - n; J = ti; break;
      case 1: I = nxp(b) - 1 - NG + n; J = ti; break;
      case 2: I = ti; J = NG - n; break;
      default: I = ti; J = nyp(b) - 1 - NG + n; break;
    }
  };
  auto inner = [&](int b, int side, int ti, int k, int& I, int& J) {
    switch (side) {
      case 0: I = NG - 1 + k; J = ti; break;
      case 1: I = nxp(b) - NG - k; J = ti; break;
      case 2: I = ti; J = NG - 1 + k; break;
      default: I = ti; J = nyp(b) - NG - k; break;
    }
  };
  static const int opposite[4] = {1, 0, 3, 2};
  auto fill = [&](int d, int s, int side, int kind) {   // FillEdge (src/Boundary.c:88-132)
    const int nt = side < 2 ? nyp(d) : nxp(d);
    for (int ti = 0; ti < nt; ti++)
      for (int n = 1; n <= NG; n++) {
        int gi, gj, si, sj;
        ghost(d, side, ti, n, gi, gj);
        Sym& g = S[d][(size_t)gj * nxp(d) + gi];
        if (kind == 0) {
          inner(s, opposite[side], ti, n, si, sj);
          g = S[s][(size_t)sj * nxp(s) + si];
        } else if (kind == 1) {
          inner(d, side, ti, 1, si, sj);
          g = S[d][(size_t)sj * nxp(d) + si];
        } else if (kind == 2) {
          inner(d, side, ti, n, si, sj);
          Sym v = S[d][(size_t)sj * nxp(d) + si];
          v.flags ^= side < 2 ? 1 : 2;
          g = v;
        } else {
          g = Sym{1, d, dir_off[d * 4 + side] + ti * NG + (n - 1), 0};
        }
      }
  };
  for (int b = 0; b < nb; b++)
    for (int side = 0; side < 4; side++) {
      int code = B[b].bc[side], k = kind_of(code);
      fill(b, k == 0 ? code - 1 : b, side, k);
    }
  for (int b = 0; b < nb; b++)
    for (int side = 0; side < 4; side++)
      if (B[b].bc[side] > 0) fill(b, B[b].bc[side] - 1, side, 0);

  out.clear();
  for (int b = 0; b < nb; b++)
    for (int J = 0; J < nyp(b); J++)
      for (int I = 0; I < nxp(b); I++) {
        bool inner_cell = I >= NG && I < nxp(b) - NG && J >= NG && J < nyp(b) - NG;
        if (inner_cell) continue;
        const Sym& v = S[b][(size_t)J * nxp(b) + I];
        if (v.kind == 2) {
          why = "block " + std::to_string(b + 1) + ": ghost cell (" + std::to_string(I) + "," +
                std::to_string(J) + ") is not set by the boundary fill (block too narrow?)";
          return MBM_EINVAL;
        }
        Resolved r;
        r.dst_blk = b;
        r.dst_cell = J * nxp(b) + I;
        r.flags = v.flags;
        if (v.kind == 0) { r.src = v.cell; r.src_blk = v.blk; }
        else { r.src = -(v.cell + 1); r.src_blk = 0; }
        out.push_back(r);
      }
  return MBM_OK;
}

// ------------------------------------------------------------------ create --
static int pitch_of(int nxp) { return (nxp + 1 + 3) & ~3; }

// Work items grouped by limiter (the stage kernel is specialised per limiter):
// blocks of cases with limiter L fill group L, strips within row segments.  Each Heun
// stage has its own table (the autotuner picks each stage's segment length).
static void build_work(mbm_ctx* c, double seg_rows, std::vector<Work>& w, std::vector<LimGroup>& groups) {
  w.clear();
  groups.clear();
  for (int lim = 0; lim < 5; lim++) {
    const int start = (int)w.size();
    for (int b = 0; b < c->nblk; b++) {
      if (c->hcase[c->blk_case[b]].limiter != lim) continue;
      const int nxp = c->hblk[b].nxp, nyp = c->hblk[b].nyp;
      const int nfx = nxp - 3, nfy = nyp - 3;          // face positions 1 .. nxp-3 / nyp-3
      const int strips = (nfx + STRIP - 1) / STRIP;
      const int segs = std::max(1, (int)std::ceil(nfy / seg_rows - 1e-9));
      for (int s = 0; s < segs; s++) {
        // equal-sized segments over face rows [1, nyp-3], the last one reaching nyp-2
        const int J0 = 1 + (int)((long long)nfy * s / segs);
        const int J1 = 1 + (int)((long long)nfy * (s + 1) / segs);
        for (int k = 0; k < strips; k++) w.push_back(Work{b, 1 + STRIP * k, J0, J1});
      }
    }
    const int count = (int)w.size() - start;
    if (count > 0) {
      LimGroup g{lim, start, count, {0, 0}};
      for (int h = 0; h < 2; h++)
        g.grid[h] = (int)std::min<long long>((count + c->cta_warps - 1) / c->cta_warps,
                                             (long long)c->nsm * c->ctas_per_sm[h]);
      groups.push_back(g);
    }
  }
}

// rebuild the work table for segments of `seg` rows; the table lives in the same
// device buffer (sized for 8-row segments)
// work items of a segment length (host only; the count build_work makes)
static long long count_items(const mbm_ctx* c, double seg_rows) {
  long long n = 0;
  for (int b = 0; b < c->nblk; b++) {
    const int nfx = c->hblk[b].nxp - 3, nfy = c->hblk[b].nyp - 3;
    n += (long long)((nfx + STRIP - 1) / STRIP) * std::max(1, (int)std::ceil(nfy / seg_rows - 1e-9));
  }
  return n;
}

// The ghost-fill entries of the work items of stage k's table: each item lists the
// entries owned by the cells it writes (output columns [I0, I0+28) and rows [J0, J1)
// within the interior; owners lie within NG of an edge).  Every entry belongs to
// exactly one item; if not, the separate gather fills the ghosts instead.
static int set_item_scatter(mbm_ctx* c, int k, const std::vector<Work>& work) {
  if (!c->gscatter) return MBM_OK;
  std::vector<int2> items(work.size());
  std::vector<GhostScatter> ents;
  ents.reserve(c->gs_ent.size());
  for (size_t i = 0; i < work.size(); i++) {
    const Work& w = work[i];
    const BlockDev& B = c->hblk[w.blk];
    const long long cb = B.off / NV;
    const int c0 = std::max(w.I0, NG), c1 = std::min(w.I0 + STRIP, B.nxp - NG);
    const int j0 = std::max(w.J0, NG), j1 = std::min(w.J1, B.nyp - NG);
    const int first = (int)ents.size();
    for (int J = j0; J < j1; J++) {
      const bool band_row = J < 2 * NG || J >= B.nyp - 2 * NG;
      for (int C = c0; C < c1; C++) {
        if (!band_row && C >= 2 * NG && C < B.nxp - 2 * NG) {
          C = B.nxp - 2 * NG - 1;      // on to the right band
          continue;
        }
        const size_t q = (size_t)(cb + (long long)J * B.pitch + C + 1);
        for (int e = c->gs_cell[q]; e < c->gs_cell[q + 1]; e++) ents.push_back(c->gs_ent[e]);
      }
    }
    items[i] = make_int2(first, (int)ents.size() - first);
  }
  if (ents.size() != c->gs_ent.size()) {
    c->gscatter = false;
    return MBM_OK;
  }
  CK(cudaMemcpyAsync(c->dgs + (size_t)k * c->gs_ent.size(), ents.data(), sizeof(GhostScatter) * ents.size(),
                     cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->dgs_item + (size_t)k * c->max_items, items.data(), sizeof(int2) * items.size(),
                     cudaMemcpyHostToDevice, c->stream));
  return MBM_OK;
}

// the work table of stage h (0, 1; -1: both) for segments of `seg` rows
static int set_segments(mbm_ctx* c, double seg, int h = -1) {
  for (int k = 0; k < 2; k++) {
    if (h >= 0 && k != h) continue;
    std::vector<Work> work;
    build_work(c, seg, work, c->groups[k]);
    c->nwork[k] = (int)work.size();
    CK(cudaMemcpyAsync(c->dwork + k * c->max_items, work.data(), sizeof(Work) * work.size(), cudaMemcpyHostToDevice,
                       c->stream));
    const int st = set_item_scatter(c, k, work);
    if (st) return st;
    c->seg_rows[k] = seg;
  }
  CK(cudaStreamSynchronize(c->stream));
  return MBM_OK;
}

// one Heun stage of every block: one persistent launch per limiter group
// (with several limiter groups, group k > 0 runs on aux stream k-1, so that one
// group's CTAs fill the SMs another group's tail leaves idle).  rlx_read (stage 2):
// the relaxation term of Data0 is read from what the stage 1 of the same attempt
// stored, instead of being formed again -- only where that stage 1 ran on the same
// Data0 just before.
static cudaError_t launch_stages(mbm_ctx* c, int heun, int sel_in, int sel_d0, int sel_out, int rlx_read,
                                 double* const* bufs = nullptr, bool fill = false) {
  const std::vector<LimGroup>& groups = c->groups[heun];
  const int ng = (int)groups.size();
  cudaError_t e0;
  if (ng > 1) {
    if ((e0 = cudaEventRecord(c->fork_ev, c->stream))) return e0;
    for (int k = 1; k < ng; k++)
      if ((e0 = cudaStreamWaitEvent(c->aux[k - 1], c->fork_ev, 0))) return e0;
  }
  for (int k = 0; k < ng; k++) {
    const LimGroup& g = groups[k];
    cudaStream_t st = k == 0 ? c->stream : c->aux[k - 1];
    StageArgs a{};
    a.blk = c->dblk;
    a.work = c->dwork + heun * c->max_items + g.start;
    a.nwork = g.count;
    a.cases = c->dcase;
    for (int l = 0; l < 3; l++) a.buf[l] = bufs ? bufs[l] : c->buf[l];
    a.lam = c->dlam;
    a.queue = c->dqueue + heun * 5 + g.lim;
    a.sel_in = sel_in; a.sel_d0 = sel_d0; a.sel_out = sel_out;
    a.heun = heun;
    a.rlx = c->rlx;
    a.rlx_read = heun == 1 && rlx_read;
    // bulk tensor copies: fast stage 2 on the context's own layers (the maps cover TMP
    // and rlx; the adjoint's recomputation passes other buffers and keeps cp.async)
    a.tmap = (c->fast && a.rlx_read && !bufs) ? c->dtmap : nullptr;
    if (a.tmap) a.tma_drop = c->dtma_drop;   // consumed on the device by the first launch
    if (fill && c->gscatter) {                // the output layer's ghost fill, scattered
      a.gs_item = c->dgs_item + heun * c->max_items + g.start;
      a.gs = c->dgs + heun * c->gs_ent.size();
      a.dirichlet = c->ddir;
    }
    cudaError_t e = c->fast ? fastmath::launch_stage(g.lim, a, g.grid[heun], st)
                            : bitwise::launch_stage(g.lim, a, g.grid[heun], st);
    if (e != cudaSuccess) return e;
  }
  for (int k = 1; k < ng; k++) {
    if ((e0 = cudaEventRecord(c->join_ev[k - 1], c->aux[k - 1]))) return e0;
    if ((e0 = cudaStreamWaitEvent(c->stream, c->join_ev[k - 1], 0))) return e0;
  }
  return cudaSuccess;
}

// programmatic dependent launch for the launches this thread makes while in scope
struct PdlScope {
  explicit PdlScope(bool on) { tl_pdl = on; }
  ~PdlScope() { tl_pdl = false; }
};

// the body of one step attempt: stage 1, fill TMP, stage 2, fill NEW, controller (the
// fills inside the stage kernels when they scatter them)
static cudaError_t launch_attempt(mbm_ctx* c, cudaGraphConditionalHandle h, int use_handle) {
  // the attempt's launches use programmatic dependent launch; the thread's others do not
  PdlScope pdl_scope(c->pdl && c->groups[0].size() <= 1 && c->groups[1].size() <= 1);
  cudaError_t e;
  const bool g = !c->gscatter;
  if ((e = launch_stages(c, 0, SEL_CUR, SEL_CUR, SEL_TMP, 0, nullptr, true))) return e;
  if (g && (e = launch_ghost(c->dblk, c->dcase, c->dghost, c->nghost, c->buf, c->ddir, SEL_TMP, c->stream))) return e;
  if ((e = launch_stages(c, 1, SEL_TMP, SEL_CUR, SEL_OTHER, 1, nullptr, true))) return e;
  if (g && (e = launch_ghost(c->dblk, c->dcase, c->dghost, c->nghost, c->buf, c->ddir, SEL_OTHER, c->stream))) return e;
  if ((e = launch_control(c->dcase, c->ncase, c->dblk, c->dlam, c->dtrace, c->dqueue, h, use_handle, c->stream)))
    return e;
  if (c->adjoint) return launch_ckpt(c->dcase, c->buf[0], c->buf[1], c->buf[2], c->layer_elems, 4 * c->nsm, c->stream);
  return cudaSuccess;
}

static int push_cases(mbm_ctx* c) {
  CK(cudaMemcpyAsync(c->dcase, c->hcase, sizeof(CaseDev) * c->ncase, cudaMemcpyHostToDevice, c->stream));
  // the records are pinned: the copy reads them when the stream reaches it, so the
  // host must not change them before then
  CK(cudaStreamSynchronize(c->stream));
  return MBM_OK;
}

// Autotuner: the stage kernel's work-item length (rows per warp segment) trades
// the per-segment warm-up (two extra primitive rows, one slope row, one face row)
// against load balance over the persistent grid.  On first use of a problem shape
// it times each Heun stage for each candidate on a uniform state at rest and keeps,
// per stage, the fastest (the two stages have their own work tables: at 4 x 1024^2
// stage 1 ran best at 24 rows, stage 2 at 29); the choice is cached per (strip rows,
// blocks, limiter mix, CTAs/SM) for the life of the process.
static std::mutex g_tune_mu;
static std::map<std::tuple<long long, int, int, int>, std::array<double, 2>> g_tune_cache;

// device time of each Heun stage with the current tables: one untimed pass of both,
// then two timed launches of each stage
static int time_each_stage(mbm_ctx* c, cudaEvent_t e0, cudaEvent_t e1, float* ms) {
  for (int heun = 0; heun < 2; heun++) {
    CK(cudaMemsetAsync(c->dqueue, 0, sizeof(int) * 10, c->stream));
    CK(launch_stages(c, heun, heun ? SEL_TMP : SEL_CUR, SEL_CUR, heun ? SEL_OTHER : SEL_TMP, 1));
  }
  for (int heun = 0; heun < 2; heun++) {
    CK(cudaEventRecord(e0, c->stream));
    for (int rep = 0; rep < 2; rep++) {
      CK(cudaMemsetAsync(c->dqueue, 0, sizeof(int) * 10, c->stream));
      CK(launch_stages(c, heun, heun ? SEL_TMP : SEL_CUR, SEL_CUR, heun ? SEL_OTHER : SEL_TMP, 1));
    }
    CK(cudaEventRecord(e1, c->stream));
    CK(cudaEventSynchronize(e1));
    CK(cudaEventElapsedTime(&ms[heun], e0, e1));
  }
  return MBM_OK;
}

static int autotune(mbm_ctx* c) {
  long long strip_rows = 0, cells = 0;
  for (auto& d : c->hblk) {
    strip_rows += (long long)((d.nxp - 3 + STRIP - 1) / STRIP) * (d.nyp - 3);
    cells += (long long)d.nxp * d.nyp;
  }
  int limmix = 0;
  for (const LimGroup& g : c->groups[0]) limmix |= 1 << g.lim;
  const auto key = std::make_tuple(strip_rows, c->nblk, limmix,
                                   (c->ctas_per_sm[0] * 256 + c->ctas_per_sm[1]) * c->cta_warps);
  {
    std::lock_guard<std::mutex> g(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      const int st = set_segments(c, it->second[0], 0);
      return st ? st : set_segments(c, it->second[1], 1);
    }
  }
  const char* env = getenv("MBM_AUTOTUNE");
  if (env && atoi(env) == 0) return set_segments(c, 32);
  for (int l = 0; l < 3; l++)
    for (auto& d : c->hblk) CK(launch_fill_uniform(c->buf[l] + d.off, d.plane, c->stream));
  for (int k = 0; k < c->ncase; k++) {
    c->hcase[k].dt = 1e-5;
    c->hcase[k].done = 0;
  }
  int st = push_cases(c);
  if (st) return st;
  LocalEvents ev;
  CK(cudaEventCreate(&ev.e[0]));
  CK(cudaEventCreate(&ev.e[1]));
  double best[2] = {32, 32};
  float best_ms[2] = {1e30f, 1e30f};
  // short segments buy parallelism on small grids, long ones save warm-up rows.  The
  // persistent grid's warps take the items from a queue, so the time jumps with the item
  // count: besides every even length, each wave count k gets the shortest length whose
  // items fill k waves of the resident warps without a partial one (the segment count is
  // ceil(rows / length), so these lengths are fractional).  4 x 1024^2 cells: 22 rows
  // (6,956 items, 3.92 waves) 3 % faster than 24, 20 rows 5 % slower, 21.4 rows (7,104
  // items, 4 waves) 1.7 % faster than 22.
  std::vector<double> cand;
  for (int seg = 8; seg <= 64; seg += 2) cand.push_back(seg);
  for (int h = 0; h < 2; h++) {              // the resident warps of each stage
    if (h == 1 && c->ctas_per_sm[1] == c->ctas_per_sm[0]) break;
    const long long W = (long long)c->nsm * c->ctas_per_sm[h] * c->cta_warps;
    const long long most = count_items(c, 8.0), least = count_items(c, 64.0);
    for (long long k = (least + W - 1) / W; k * W < most && k <= 64; k++) {
      double lo = 8.0, hi = 64.0;              // count_items(hi) <= k W < count_items(lo)
      for (int it = 0; it < 40; it++) {
        const double mid = 0.5 * (lo + hi);
        if (count_items(c, mid) <= k * W) hi = mid;
        else lo = mid;
      }
      cand.push_back(hi);
    }
  }
  for (double seg : cand) {             // each stage keeps its own fastest length
    st = set_segments(c, seg);
    float ms[2] = {0.f, 0.f};
    if (!st) st = time_each_stage(c, ev.e[0], ev.e[1], ms);
    if (st) return st;
    for (int k = 0; k < 2; k++)
      if (ms[k] < best_ms[k]) { best_ms[k] = ms[k]; best[k] = seg; }
  }
  for (int l = 0; l < 3; l++) CK(cudaMemsetAsync(c->buf[l], 0, sizeof(double) * c->layer_elems, c->stream));
  CK(cudaMemsetAsync(c->dlam, 0, sizeof(unsigned long long) * 6 * c->nblk, c->stream));
  for (int k = 0; k < c->ncase; k++) c->hcase[k].done = 1;
  if ((st = push_cases(c))) return st;
  {
    std::lock_guard<std::mutex> g(g_tune_mu);
    g_tune_cache[key] = {best[0], best[1]};
  }
  st = set_segments(c, best[0], 0);
  return st ? st : set_segments(c, best[1], 1);
}

// Tensor maps of the fast stage 2's bulk copies: for every block, its TMP layer and its
// relaxation layer as 3-D tensors (column x pitch, row x nyp, moment plane x 9; strides
// pitch and plane doubles), boxes of 32 columns x 1 row x 9 planes.  The TMA rules are
// checked here, on the host, before any map exists: 16-byte aligned bases and strides, an
// inner box of 256 bytes, and box origins (the strips' first columns, 28 k) on an even
// column, i.e. a 16-byte boundary.  Rows and columns outside a block read zeros.  The
// encoder comes from the driver at run time.  Opt-in (MBM_TMA=1): on this kernel the bulk
// copies measured 5-16 % slower in stage 2 than the per-lane copies (one lane issues and
// the whole warp polls an mbarrier per row and slot, where the per-lane copies overlap
// their issue with the row's work), so the per-lane copies are the default.
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static_assert(sizeof(CUtensorMap) == TMAP_BYTES, "tensor map size");
static_assert(STRIP % 2 == 0, "strip origins must stay on 16-byte boundaries");

static void make_stage2_maps(mbm_ctx* c) {
  const char* env = getenv("MBM_TMA");
  if (!env || atoi(env) != 1) { c->tma_note = "bulk tensor copies not requested (MBM_TMA=1 selects them)"; return; }
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q{};
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn ||
      q != cudaDriverEntryPointSuccess) {
    cudaGetLastError();
    c->tma_note = "cuTensorMapEncodeTiled unavailable";
    return;
  }
  const EncodeTiledFn encode = (EncodeTiledFn)fn;
  std::vector<CUtensorMap> maps((size_t)c->nblk * 2);
  for (int b = 0; b < c->nblk; b++) {
    const BlockDev& d = c->hblk[b];
    double* base[2] = {c->buf[2] + d.off, c->rlx + d.off};
    const cuuint64_t dims[3] = {(cuuint64_t)d.pitch, (cuuint64_t)d.nyp, (cuuint64_t)NV};
    const cuuint64_t strides[2] = {(cuuint64_t)d.pitch * sizeof(double), (cuuint64_t)d.plane * sizeof(double)};
    const cuuint32_t box[3] = {32, 1, (cuuint32_t)NV}, estr[3] = {1, 1, 1};
    if (strides[0] % 16 || strides[1] % 16 || d.pitch < 1) { c->tma_note = "unaligned strides"; return; }
    for (int k = 0; k < 2; k++) {
      if ((uintptr_t)base[k] % 16) { c->tma_note = "unaligned layer"; return; }
      if (encode(&maps[(size_t)b * 2 + k], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, base[k], dims, strides, box, estr,
                 CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
        c->tma_note = "tensor map encoding failed";
        return;
      }
    }
  }
  void* dm = nullptr;
  if (cudaMalloc(&dm, maps.size() * sizeof(CUtensorMap)) != cudaSuccess) {
    cudaGetLastError();
    c->tma_note = "no memory for the tensor maps";
    return;
  }
  if (cudaMemcpy(dm, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(dm);
    c->tma_note = "tensor map copy failed";
    return;
  }
  c->dtmap = dm;
  // failure-detection test hook: the first bulk-copy launch of this context withholds one
  // copy, so that a bounded wait runs out and the case stops with MBM_ETIMEOUT
  const char* drop = getenv("MBM_TMA_TEST_DROP");
  if (drop && atoi(drop) == 1) {
    const int one = 1;
    if (cudaMalloc(&c->dtma_drop, sizeof(int)) != cudaSuccess ||
        cudaMemcpy(c->dtma_drop, &one, sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess) {
      cudaGetLastError();
      cudaFree(c->dtma_drop);
      c->dtma_drop = nullptr;
    }
  }
}

// exchange plan of one rank of a case split over ranks by block (mbm_create_sharded)
struct ShardSetup {
  std::vector<int> send_counts, recv_counts;          // cells per peer rank
  std::vector<std::array<int, 2>> send;               // (local block, cell J*nxp+I), peers in rank order
  std::vector<int> dir_off, nt;                       // Dirichlet rows and edge lengths, [global block][side]
};

static int create_impl(const std::vector<mbm_block_desc>& glob, const std::vector<int>& blk_case,
                       const mbm_case_desc* cases, int ncases, const mbm_params* params,
                       const std::vector<Resolved>& res, const std::vector<int>& dir_off, int ndir,
                       const ShardSetup* shard, mbm_ctx** out);

extern "C" int mbm_create_batch(const mbm_block_desc* blocks, int nblocks, const mbm_case_desc* cases,
                                int ncases, const mbm_params* params, mbm_ctx** out) {
  if (!out || !params || !cases || ncases < 1) return fail(nullptr, MBM_EINVAL, "null argument");
  *out = nullptr;
  std::string why;
  if (!blocks || nblocks < 1 || nblocks > 65535) return fail(nullptr, MBM_EINVAL, "need 1..65535 blocks");
  if (params->mode != MBM_MODE_EXACT && params->mode != MBM_MODE_FAST)
    return fail(nullptr, MBM_EINVAL, "unknown arithmetic mode");
  // cases tile the block array; sync codes become global block numbers
  std::vector<mbm_block_desc> glob(blocks, blocks + nblocks);
  std::vector<int> blk_case(nblocks, -1);
  for (int k = 0; k < ncases; k++) {
    const mbm_case_desc& cd = cases[k];
    if (cd.nblocks < 1 || cd.first_block < 0 || cd.first_block + cd.nblocks > nblocks)
      return fail(nullptr, MBM_EINVAL, "case " + std::to_string(k) + ": block range outside the table");
    if (cd.limiter < 0 || cd.limiter > 4) return fail(nullptr, MBM_EINVAL, "limiter code must be 0..4");
    if (!(cd.Kn > 1e-100 && cd.Kn < 1e100)) return fail(nullptr, MBM_EINVAL, "Kn must be in (1e-100, 1e100)");
    for (int b = cd.first_block; b < cd.first_block + cd.nblocks; b++) {
      if (blk_case[b] >= 0) return fail(nullptr, MBM_EINVAL, "cases overlap");
      blk_case[b] = k;
      for (int s = 0; s < 4; s++)
        if (glob[b].bc[s] > 0) {
          if (glob[b].bc[s] > cd.nblocks)
            return fail(nullptr, MBM_EINVAL, "case " + std::to_string(k) + ": sync partner outside the case");
          glob[b].bc[s] += cd.first_block;
        }
    }
    if (validate(glob.data(), nblocks, why, cd.first_block, cd.first_block + cd.nblocks) != MBM_OK)
      return fail(nullptr, MBM_EINVAL, "case " + std::to_string(k) + ": " + why);
  }
  for (int b = 0; b < nblocks; b++)
    if (blk_case[b] < 0) return fail(nullptr, MBM_EINVAL, "block " + std::to_string(b + 1) + " belongs to no case");
  std::vector<Resolved> res;
  std::vector<int> dir_off;
  int ndir = 0;
  if (resolve_ghosts(glob.data(), nblocks, res, dir_off, ndir, why) != MBM_OK)
    return fail(nullptr, MBM_EINVAL, why);
  return create_impl(glob, blk_case, cases, ncases, params, res, dir_off, ndir, nullptr, out);
}

// the context proper, from a block table whose ghost map is resolved; shard: the
// exchange plan of a case split over ranks (nullptr otherwise)
static int create_impl(const std::vector<mbm_block_desc>& glob, const std::vector<int>& blk_case,
                       const mbm_case_desc* cases, int ncases, const mbm_params* params,
                       const std::vector<Resolved>& res, const std::vector<int>& dir_off, int ndir,
                       const ShardSetup* shard, mbm_ctx** out) {
  mbm_ctx* c = nullptr;
  const int nblocks = (int)glob.size();
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(nullptr, MBM_ENODEV, "no CUDA device");
  if (params->device < 0 || params->device >= ndev) return fail(nullptr, MBM_EINVAL, "bad device ordinal");

  c = new mbm_ctx();
  c->prm = *params;
  {
    const char* hl = getenv("MBM_HOST_LOOP");
    c->host_loop = hl && atoi(hl) != 0;
  }
  if (c->prm.max_attempts <= 0) c->prm.max_attempts = 10000000;
  c->adjoint = params->adjoint != 0 && ncases == 1;
  c->fast = params->mode == MBM_MODE_FAST;
  c->device = params->device;
  c->nblk = nblocks;
  c->ncase = ncases;
  c->desc = glob;
  c->blk_case = blk_case;
  c->dir_off = dir_off;
  c->ndir = ndir;
  auto bail = [&](int code) { g_create_error = c->err; mbm_destroy(c); return code; };
#define CKC(call)                                                                                 \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess) {                                                                      \
      c->err = std::string(#call) + ": " + cudaGetErrorString(e_);                                \
      return bail(e_ == cudaErrorMemoryAllocation ? MBM_ENOMEM : MBM_ECUDA);                      \
    }                                                                                             \
  } while (0)
  CKC(cudaSetDevice(c->device));
  if (params->stream) {
    c->stream = (cudaStream_t)params->stream;
  } else {
    CKC(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    c->own_stream = true;
  }
  CKC(cudaEventCreateWithFlags(&c->ev, cudaEventDisableTiming));
  CKC(cudaEventCreateWithFlags(&c->fork_ev, cudaEventDisableTiming));
  for (int k = 0; k < 4; k++) {
    CKC(cudaStreamCreateWithFlags(&c->aux[k], cudaStreamNonBlocking));
    CKC(cudaEventCreateWithFlags(&c->join_ev[k], cudaEventDisableTiming));
  }

  // block table and layer layout
  long long off = 0, max_cells = 0;
  for (int b = 0; b < nblocks; b++) {
    BlockDev d{};
    d.nxp = glob[b].nx + 2 * NG;
    d.nyp = glob[b].ny + 2 * NG;
    d.pitch = pitch_of(d.nxp);
    d.case_id = blk_case[b];
    d.plane = ((long long)d.pitch * d.nyp + 31) & ~31LL;
    d.off = off;
    d.dx = glob[b].dx;
    d.dy = glob[b].dy;
    off += d.plane * NV;
    max_cells = std::max(max_cells, (long long)d.nxp * d.nyp);
    c->hblk.push_back(d);
  }
  c->layer_elems = off;
  for (int l = 0; l < 3; l++) {
    CKC(cudaMalloc(&c->buf[l], sizeof(double) * off));
    CKC(cudaMemsetAsync(c->buf[l], 0, sizeof(double) * off, c->stream));
  }
  CKC(cudaMalloc(&c->rlx, sizeof(double) * off));
  CKC(cudaMemsetAsync(c->rlx, 0, sizeof(double) * off, c->stream));
  CKC(cudaMalloc(&c->staging, sizeof(double) * max_cells * (NV + 1)));   // layers, or 10 output fields
  CKC(cudaMalloc(&c->dblk, sizeof(BlockDev) * nblocks));
  CKC(cudaMemcpyAsync(c->dblk, c->hblk.data(), sizeof(BlockDev) * nblocks, cudaMemcpyHostToDevice, c->stream));
  if (c->fast) make_stage2_maps(c);

  // ghost map in device element indices
  std::vector<GhostEntry> gm(res.size());
  for (size_t i = 0; i < res.size(); i++) {
    const Resolved& r = res[i];
    const BlockDev& D = c->hblk[r.dst_blk];
    GhostEntry e;
    e.dst_blk = r.dst_blk;
    e.dst = (r.dst_cell / D.nxp) * D.pitch + r.dst_cell % D.nxp + 1;
    if (r.remote >= 0) {
      e.src = r.remote;
      e.src_blk_flags = (r.flags << 16) | GHOST_REMOTE;
      gm[i] = e;
      continue;
    }
    if (r.src >= 0) {
      const BlockDev& S = c->hblk[r.src_blk];
      e.src = (r.src / S.nxp) * S.pitch + r.src % S.nxp + 1;
    } else {
      e.src = r.src;
    }
    e.src_blk_flags = r.src_blk | (r.flags << 16);
    gm[i] = e;
  }
  c->nghost = (int)gm.size();
  CKC(cudaMalloc(&c->dghost, sizeof(GhostEntry) * std::max<size_t>(1, gm.size())));
  if (!gm.empty())
    CKC(cudaMemcpyAsync(c->dghost, gm.data(), sizeof(GhostEntry) * gm.size(), cudaMemcpyHostToDevice, c->stream));
  CKC(cudaMalloc(&c->ddir, sizeof(double) * NV * std::max(1, ndir)));
  CKC(cudaMemsetAsync(c->ddir, 0, sizeof(double) * NV * std::max(1, ndir), c->stream));
  {
    // the same fill listed under owners: a copied ghost under its source, a Dirichlet
    // ghost under the interior cell nearest to it; every owner must be an interior cell
    // within NG of its block's edge, else the gather stays
    const char* env = getenv("MBM_GHOST_SCATTER");
    bool ok = env && atoi(env) == 1 && !res.empty();
    std::vector<std::pair<long long, GhostScatter>> lst;
    lst.reserve(res.size());
    for (size_t i = 0; ok && i < res.size(); i++) {
      const Resolved& r = res[i];
      if (r.remote >= 0) { ok = false; break; }
      const BlockDev& D = c->hblk[r.dst_blk];
      int ob = r.dst_blk, oI, oJ;
      if (r.src >= 0) {
        ob = r.src_blk;
        oI = r.src % c->hblk[ob].nxp;
        oJ = r.src / c->hblk[ob].nxp;
      } else {
        oI = std::min(std::max(r.dst_cell % D.nxp, NG), D.nxp - 1 - NG);
        oJ = std::min(std::max(r.dst_cell / D.nxp, NG), D.nyp - 1 - NG);
      }
      const BlockDev& O = c->hblk[ob];
      const bool interior = oI >= NG && oI <= O.nxp - 1 - NG && oJ >= NG && oJ <= O.nyp - 1 - NG;
      const bool band = oI < 2 * NG || oI >= O.nxp - 2 * NG || oJ < 2 * NG || oJ >= O.nyp - 2 * NG;
      if (!interior || !band) { ok = false; break; }
      GhostScatter g;
      g.dst = D.off + gm[i].dst;
      g.plane = D.plane;
      g.src = oJ * O.pitch + oI + 1;
      g.flags = r.flags & 3;
      g.drow = r.src >= 0 ? -1 : -(r.src + 1);
      g.pad_ = 0;
      lst.emplace_back(O.off / NV + g.src, g);
    }
    if (ok) {     // owner order (the tables of the work items are built from it)
      std::stable_sort(lst.begin(), lst.end(),
                       [](const std::pair<long long, GhostScatter>& x, const std::pair<long long, GhostScatter>& y) {
                         return x.first < y.first;
                       });
      const long long ncell = c->layer_elems / NV;
      c->gs_cell.assign((size_t)ncell + 1, 0);
      for (auto& p : lst) c->gs_cell[(size_t)p.first + 1]++;
      for (long long k = 0; k < ncell; k++) c->gs_cell[(size_t)k + 1] += c->gs_cell[(size_t)k];
      c->gs_ent.resize(lst.size());
      for (size_t i = 0; i < lst.size(); i++) c->gs_ent[i] = lst[i].second;
      c->gscatter = true;
    }
  }

  // controllers, maxima, queues, trace, per-block CFL
  CKC(cudaMalloc(&c->dcase, sizeof(CaseDev) * ncases));
  CKC(cudaMallocHost(&c->hcase, sizeof(CaseDev) * ncases));
  memset(c->hcase, 0, sizeof(CaseDev) * ncases);
  for (int k = 0; k < ncases; k++) {
    CaseDev& h = c->hcase[k];
    h.Kn = cases[k].Kn;
    h.F = cases[k].F;
    h.limiter = cases[k].limiter;
    h.cur = 0;
    h.done = 1;
    h.blk0 = cases[k].first_block;
    h.nblk = cases[k].nblocks;
    h.max_attempts = c->prm.max_attempts;
  }
  CKC(cudaMemcpyAsync(c->dcase, c->hcase, sizeof(CaseDev) * ncases, cudaMemcpyHostToDevice, c->stream));
  CKC(cudaMalloc(&c->dqueue, sizeof(int) * 10));
  CKC(cudaMemsetAsync(c->dqueue, 0, sizeof(int) * 10, c->stream));
  CKC(cudaMalloc(&c->dlam, sizeof(unsigned long long) * 6 * nblocks));
  CKC(cudaMemsetAsync(c->dlam, 0, sizeof(unsigned long long) * 6 * nblocks, c->stream));
  CKC(cudaMalloc(&c->dtrace, sizeof(double) * 4 * MAX_TRACE * ncases));
  CKC(cudaMalloc(&c->dcfl, sizeof(double) * nblocks));
  CKC(cudaMallocHost(&c->hcfl, sizeof(double) * nblocks));

  // work table and grid
  CKC(cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, c->device));
  for (int hh = 0; hh < 2; hh++)
    c->ctas_per_sm[hh] = c->fast ? fastmath::stage_ctas_per_sm(hh) : bitwise::stage_ctas_per_sm(hh);
  c->cta_warps = c->fast ? fastmath::stage_cta_warps() : bitwise::stage_cta_warps();
  long long max_items = 0;
  for (auto& d : c->hblk) max_items += (long long)((d.nxp - 3 + STRIP - 1) / STRIP) * ((d.nyp - 3 + 7) / 8 + 1);
  c->max_items = std::max<long long>(1, max_items);
  CKC(cudaMalloc(&c->dwork, sizeof(Work) * 2 * c->max_items));
  if (c->gscatter) {
    CKC(cudaMalloc(&c->dgs, sizeof(GhostScatter) * 2 * c->gs_ent.size()));
    CKC(cudaMalloc(&c->dgs_item, sizeof(int2) * 2 * c->max_items));
  }
  {
    int st0 = params->segment_rows > 0 ? set_segments(c, std::max(8, params->segment_rows)) : autotune(c);
    if (st0) return bail(st0);
  }

  if (shard) {   // exchange buffers, send list, the CFL scalar; the step loop is driven per phase
    c->sharded = true;
    c->shard_dir_off = shard->dir_off;
    c->shard_nt = shard->nt;
    c->send_counts = shard->send_counts;
    c->recv_counts = shard->recv_counts;
    c->nsend = (int)shard->send.size();
    c->nrecv = 0;
    for (int v : shard->recv_counts) c->nrecv += v;
    std::vector<int2> sl(shard->send.size());
    for (size_t i = 0; i < sl.size(); i++) {
      const BlockDev& d = c->hblk[shard->send[i][0]];
      const int cell = shard->send[i][1];
      sl[i] = make_int2(shard->send[i][0], (cell / d.nxp) * d.pitch + cell % d.nxp + 1);
    }
    CKC(cudaMalloc(&c->dsend_list, sizeof(int2) * std::max<size_t>(1, sl.size())));
    if (!sl.empty())
      CKC(cudaMemcpyAsync(c->dsend_list, sl.data(), sizeof(int2) * sl.size(), cudaMemcpyHostToDevice, c->stream));
    CKC(cudaMalloc(&c->shard_send, sizeof(double) * NV * std::max(1, c->nsend)));
    CKC(cudaMalloc(&c->shard_recv, sizeof(double) * NV * std::max(1, c->nrecv)));
    CKC(cudaMemsetAsync(c->shard_recv, 0, sizeof(double) * NV * std::max(1, c->nrecv), c->stream));
    CKC(cudaMalloc(&c->shard_cfl, sizeof(double)));
    CKC(cudaMemsetAsync(c->shard_cfl, 0, sizeof(double), c->stream));
    int st = wait_stream(c);
    if (st != MBM_OK) return bail(st);
    *out = c;
    return MBM_OK;
  }

  // the step loop: while (any case live) { stage 1; fill TMP; stage 2; fill NEW; control }
  {
    const char* pe = getenv("MBM_PDL");
    c->pdl = !(pe && atoi(pe) == 0);
    auto build_graph = [&]() -> cudaError_t {
      cudaError_t e;
      cudaGraphConditionalHandle h;
      if ((e = cudaGraphCreate(&c->graph, 0))) return e;
      if ((e = cudaGraphConditionalHandleCreate(&h, c->graph, 1, cudaGraphCondAssignDefault))) return e;
      cudaGraphNodeParams np = {};
      np.type = cudaGraphNodeTypeConditional;
      np.conditional.handle = h;
      np.conditional.type = cudaGraphCondTypeWhile;
      np.conditional.size = 1;
      cudaGraphNode_t node;
      if ((e = cudaGraphAddNode(&node, c->graph, nullptr, 0, &np))) return e;
      cudaGraph_t body = np.conditional.phGraph_out[0];
      if ((e = cudaStreamBeginCaptureToGraph(c->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)))
        return e;
      const cudaError_t e1 = launch_attempt(c, h, 1);
      cudaGraph_t captured = nullptr;
      const cudaError_t e2 = cudaStreamEndCapture(c->stream, &captured);
      if (e1) return e1;
      if (e2) return e2;
      return cudaGraphInstantiate(&c->gexec, c->graph, 0);
    };
    cudaError_t eg = build_graph();
    if (eg != cudaSuccess && c->pdl) {   // without programmatic launches, once more
      if (c->gexec) cudaGraphExecDestroy(c->gexec);
      if (c->graph) cudaGraphDestroy(c->graph);
      c->gexec = nullptr;
      c->graph = nullptr;
      cudaGetLastError();
      c->pdl = false;
      eg = build_graph();
    }
    CKC(eg);
  }
  int st = wait_stream(c);
  if (st != MBM_OK) return bail(st);
  *out = c;
  return MBM_OK;
#undef CKC
}

extern "C" int mbm_create(const mbm_block_desc* blocks, int nblocks, const mbm_params* params,
                          mbm_ctx** out) {
  if (!params) return fail(nullptr, MBM_EINVAL, "null argument");
  mbm_case_desc one;
  one.first_block = 0;
  one.nblocks = nblocks;
  one.Kn = params->Kn;
  one.F = params->F;
  one.limiter = params->limiter;
  return mbm_create_batch(blocks, nblocks, &one, 1, params, out);
}

extern "C" int mbm_destroy(mbm_ctx* c) {
  if (!c) return MBM_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->gexec) cudaGraphExecDestroy(c->gexec);
  if (c->graph) cudaGraphDestroy(c->graph);
  for (int l = 0; l < 3; l++) cudaFree(c->buf[l]);
  cudaFree(c->rlx);
  cudaFree(c->dtmap);
  cudaFree(c->dtma_drop);
  cudaFree(c->staging);
  cudaFree(c->dblk);
  cudaFree(c->dghost);
  cudaFree(c->ddir);
  cudaFree(c->dgs);
  cudaFree(c->dgs_item);
  cudaFree(c->dwork);
  cudaFree(c->dcase);
  if (c->hcase) cudaFreeHost(c->hcase);
  cudaFree(c->dlam);
  cudaFree(c->dqueue);
  for (int k = 0; k < 9; k++) cudaFree(c->adj_buf[k]);
  cudaFree(c->adj_ckpt);
  for (int k = 0; k < 2; k++) {
    cudaFree(c->adj_seg[k]);
    cudaFree(c->adj_segT[k]);
    if (c->adj_ready[k]) cudaEventDestroy(c->adj_ready[k]);
    if (c->adj_free[k]) cudaEventDestroy(c->adj_free[k]);
  }
  if (c->adj_start) cudaEventDestroy(c->adj_start);
  if (c->adj_rstream) cudaStreamDestroy(c->adj_rstream);
  cudaFree(c->adj_dtlog);
  cudaFree(c->adj_dtrep);
  cudaFree(c->adj_part);
  cudaFree(c->adj_work);
  cudaFree(c->adj_queue);
  cudaFree(c->adj_scal);
  cudaFree(c->dsend_list);
  cudaFree(c->shard_send);
  cudaFree(c->shard_recv);
  cudaFree(c->shard_cfl);
  cudaFree(c->dtrace);
  cudaFree(c->dcfl);
  if (c->hcfl) cudaFreeHost(c->hcfl);
  if (c->ev) cudaEventDestroy(c->ev);
  if (c->fork_ev) cudaEventDestroy(c->fork_ev);
  if (c->out_stream) cudaStreamSynchronize(c->out_stream);
  cudaFree(c->out_stage);
  if (c->out_ev) cudaEventDestroy(c->out_ev);
  if (c->out_stream) cudaStreamDestroy(c->out_stream);
  for (int k = 0; k < 4; k++) {
    if (c->join_ev[k]) cudaEventDestroy(c->join_ev[k]);
    if (c->aux[k]) cudaStreamDestroy(c->aux[k]);
  }
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return MBM_OK;
}

// ---------------------------------------------------------------- transfers --
static int layer_sel(int layer) {
  return layer == MBM_L_DATA ? SEL_CUR : layer == MBM_L_NEW ? SEL_OTHER : SEL_TMP;
}

static bool bad_layer(int layer) { return layer < 0 || layer > 2; }

static int phys_of(mbm_ctx* c, int layer, int block) {
  return phys_layer(layer_sel(layer), c->hcase[c->blk_case[block]].cur);
}

extern "C" int mbm_upload(mbm_ctx* c, int layer, int block, const double* cells) {
  if (!c || !cells || bad_layer(layer) || block < 0 || block >= c->nblk) return fail(c, MBM_EINVAL, "mbm_upload: bad argument");
  CK(cudaSetDevice(c->device));
  const BlockDev& d = c->hblk[block];
  CK(cudaMemcpyAsync(c->staging, cells, sizeof(double) * d.nxp * d.nyp * NV, cudaMemcpyHostToDevice, c->stream));
  CK(launch_aos_to_planes(c->staging, c->buf[phys_of(c, layer, block)] + d.off, d.nxp, d.nyp, d.pitch, d.plane, c->stream));
  return wait_stream(c);
}

extern "C" int mbm_download(mbm_ctx* c, int layer, int block, double* cells) {
  if (!c || !cells || bad_layer(layer) || block < 0 || block >= c->nblk) return fail(c, MBM_EINVAL, "mbm_download: bad argument");
  CK(cudaSetDevice(c->device));
  const BlockDev& d = c->hblk[block];
  CK(launch_planes_to_aos(c->buf[phys_of(c, layer, block)] + d.off, c->staging, d.nxp, d.nyp, d.pitch, d.plane, c->stream));
  CK(cudaMemcpyAsync(cells, c->staging, sizeof(double) * d.nxp * d.nyp * NV, cudaMemcpyDeviceToHost, c->stream));
  return wait_stream(c);
}

extern "C" int mbm_load_fields(mbm_ctx* c, int block, int single, const void* payload, int faithful) {
  if (!c || !payload || block < 0 || block >= c->nblk || (single != 0 && single != 1) ||
      (faithful != 0 && faithful != 1))
    return fail(c, MBM_EINVAL, "mbm_load_fields: bad argument");
  CK(cudaSetDevice(c->device));
  const BlockDev& d = c->hblk[block];
  const size_t bytes = (size_t)(d.nxp - 4) * (d.nyp - 4) * 10 * (single ? sizeof(float) : sizeof(double));
  CK(cudaMemcpyAsync(c->staging, payload, bytes, cudaMemcpyHostToDevice, c->stream));
  CK(launch_fields_to_planes(c->staging, single, faithful, d.nxp, d.nyp, d.pitch, d.plane,
                             c->buf[phys_of(c, MBM_L_DATA, block)] + d.off, c->stream));
  return wait_stream(c);
}

extern "C" int mbm_output_fields(mbm_ctx* c, int block, int single, void* out) {
  if (!c || !out || block < 0 || block >= c->nblk) return fail(c, MBM_EINVAL, "mbm_output_fields: bad argument");
  CK(cudaSetDevice(c->device));
  const BlockDev& d = c->hblk[block];
  const size_t bytes = (size_t)(d.nxp - 4) * (d.nyp - 4) * 10 * (single ? sizeof(float) : sizeof(double));
  CK(launch_output_fields(c->buf[phys_of(c, MBM_L_DATA, block)] + d.off, d.nxp, d.nyp, d.pitch, d.plane,
                          single, c->staging, c->stream));
  CK(cudaMemcpyAsync(out, c->staging, bytes, cudaMemcpyDeviceToHost, c->stream));
  return wait_stream(c);
}

extern "C" int mbm_output_fields_async(mbm_ctx* c, int block, int single, void* host) {
  if (!c || !host || block < 0 || block >= c->nblk) return fail(c, MBM_EINVAL, "mbm_output_fields_async: bad argument");
  CK(cudaSetDevice(c->device));
  if (!c->out_stage) {   // one payload area per block, an own stream for the copies
    std::vector<size_t> offs;
    size_t off = 0;
    for (auto& d : c->hblk) {
      offs.push_back(off);
      off += ((size_t)(d.nxp - 4) * (d.nyp - 4) * 10 * sizeof(double) + 255) & ~(size_t)255;
    }
    CK(cudaMalloc(&c->out_stage, off));
    c->out_off = offs;
  }
  // each resource on its own, so that a call after a failed one completes the set
  if (!c->out_stream) CK(cudaStreamCreateWithFlags(&c->out_stream, cudaStreamNonBlocking));
  if (!c->out_ev) CK(cudaEventCreateWithFlags(&c->out_ev, cudaEventDisableTiming));
  const BlockDev& d = c->hblk[block];
  const size_t bytes = (size_t)(d.nxp - 4) * (d.nyp - 4) * 10 * (single ? sizeof(float) : sizeof(double));
  char* dst = (char*)c->out_stage + c->out_off[block];
  CK(launch_output_fields(c->buf[phys_of(c, MBM_L_DATA, block)] + d.off, d.nxp, d.nyp, d.pitch, d.plane,
                          single, dst, c->stream));
  CK(cudaEventRecord(c->out_ev, c->stream));
  CK(cudaStreamWaitEvent(c->out_stream, c->out_ev, 0));
  CK(cudaMemcpyAsync(host, dst, bytes, cudaMemcpyDeviceToHost, c->out_stream));
  return MBM_OK;
}

extern "C" int mbm_output_wait(mbm_ctx* c) {
  if (!c) return fail(c, MBM_EINVAL, "mbm_output_wait: null context");
  if (!c->out_stream) return MBM_OK;
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->out_stream));
  return MBM_OK;
}

extern "C" int mbm_host_alloc(size_t bytes, void** p) {
  if (!p) return fail(nullptr, MBM_EINVAL, "mbm_host_alloc: null argument");
  *p = nullptr;
  const cudaError_t e = cudaMallocHost(p, bytes > 0 ? bytes : 1);
  if (e != cudaSuccess) return fail(nullptr, e == cudaErrorMemoryAllocation ? MBM_ENOMEM : MBM_ECUDA, cudaGetErrorString(e));
  return MBM_OK;
}

extern "C" int mbm_host_free(void* p) {
  if (p) cudaFreeHost(p);
  return MBM_OK;
}

extern "C" int mbm_set_dirichlet(mbm_ctx* c, int block, int side, const double* values) {
  if (!c || !values || block < 0 || block >= c->nblk || side < 0 || side > 3) return fail(c, MBM_EINVAL, "mbm_set_dirichlet: bad argument");
  const int row = c->dir_off[block * 4 + side];
  if (row < 0) return fail(c, MBM_EINVAL, "mbm_set_dirichlet: edge is not a Dirichlet edge");
  CK(cudaSetDevice(c->device));
  const BlockDev& d = c->hblk[block];
  const int nt = side < 2 ? d.nyp : d.nxp;
  CK(cudaMemcpyAsync(c->ddir + (size_t)row * NV, values, sizeof(double) * nt * NG * NV, cudaMemcpyHostToDevice, c->stream));
  return wait_stream(c);
}

// ------------------------------------------------------------- stage calls --
static void live_all(mbm_ctx* c, double dt, double t) {
  for (int k = 0; k < c->ncase; k++) {
    c->hcase[k].dt = dt;
    c->hcase[k].t = t;
    c->hcase[k].done = 0;
  }
}

extern "C" int mbm_set_boundary(mbm_ctx* c, int layer, double t) {
  if (c && c->sharded) return fail(c, MBM_EINVAL, "mbm_set_boundary: the context holds part of a sharded case (mbm_shard_*)");
  (void)t;   // Dirichlet values are the host-set table; the reference's states are steady
  if (!c || bad_layer(layer)) return fail(c, MBM_EINVAL, "mbm_set_boundary: bad argument");
  CK(cudaSetDevice(c->device));
  for (int k = 0; k < c->ncase; k++) c->hcase[k].done = 0;
  int st = push_cases(c);
  if (st) return st;
  CK(launch_ghost(c->dblk, c->dcase, c->dghost, c->nghost, c->buf, c->ddir, layer_sel(layer), c->stream));
  return wait_stream(c);
}

static int run_stage(mbm_ctx* c, int out_layer, int in_layer, int d0_layer, int heun, double* cfl,
                     int rlx_read = 0) {
  CK(cudaMemsetAsync(c->dqueue, 0, sizeof(int) * 10, c->stream));
  CK(launch_stages(c, heun, layer_sel(in_layer), layer_sel(d0_layer), layer_sel(out_layer), rlx_read));
  CK(launch_stage_cfl(c->dblk, c->nblk, c->dcase, c->dlam, heun, c->dcfl, c->stream));
  CK(cudaMemcpyAsync(c->hcfl, c->dcfl, sizeof(double) * c->nblk, cudaMemcpyDeviceToHost, c->stream));
  int st = wait_stream(c);
  if (st) return st;
  if (cfl) memcpy(cfl, c->hcfl, sizeof(double) * c->nblk);
  return MBM_OK;
}

extern "C" int mbm_update(mbm_ctx* c, int out_layer, int in_layer, int data0_layer, double dt,
                          double t, int heun, double* cfl) {
  if (c && c->sharded) return fail(c, MBM_EINVAL, "mbm_update: the context holds part of a sharded case (mbm_shard_*)");
  if (!c || bad_layer(out_layer) || bad_layer(in_layer) || bad_layer(data0_layer) || (heun != 0 && heun != 1) ||
      out_layer == in_layer || out_layer == data0_layer)
    return fail(c, MBM_EINVAL, "mbm_update: bad argument");
  CK(cudaSetDevice(c->device));
  live_all(c, dt, t);
  int st = push_cases(c);
  if (st) return st;
  return run_stage(c, out_layer, in_layer, data0_layer, heun, cfl);
}

extern "C" int mbm_time_update(mbm_ctx* c, double dt, double t, double* cfl) {
  if (c && c->sharded) return fail(c, MBM_EINVAL, "mbm_time_update: the context holds part of a sharded case (mbm_shard_*)");
  if (!c) return fail(c, MBM_EINVAL, "mbm_time_update: null context");
  std::vector<double> v(c->nblk);
  double c1 = 0.0, c2 = 0.0;
  int st = mbm_update(c, MBM_L_TMP, MBM_L_DATA, MBM_L_DATA, dt, t, 0, v.data());
  if (st) return st;
  for (double x : v) if (x > c1) c1 = x;
  if ((st = mbm_set_boundary(c, MBM_L_TMP, t + dt))) return st;
  st = run_stage(c, MBM_L_NEW, MBM_L_TMP, MBM_L_DATA, 1, v.data(), 1);   // stage 1 ran on DATA
  if (st) return st;
  for (double x : v) if (x > c2) c2 = x;
  if ((st = mbm_set_boundary(c, MBM_L_NEW, t + dt))) return st;
  if (cfl) *cfl = c1 > (c2 > 0.0 ? c2 : 0.0) ? c1 : (c2 > 0.0 ? c2 : 0.0);
  return MBM_OK;
}

// Steps for every case at once: each case has its own t, tend and dt; the loop
// ends when every case is done (t >= tend, max_steps reached, or a failure).
// the step loop of every case, launched; mbm_steps_batch_wait collects it
extern "C" int mbm_steps_batch_async(mbm_ctx* c, const double* t, const double* tend, double CFLmax,
                                     double CFLreg, int max_steps) {
  if (!c || !t || !tend || max_steps < 0) return fail(c, MBM_EINVAL, "mbm_steps: bad argument");
  if (c->sharded) return fail(c, MBM_EINVAL, "mbm_steps: the context holds part of a sharded case (mbm_shard_*)");
  CK(cudaSetDevice(c->device));
  bool any = false;
  for (int k = 0; k < c->ncase; k++) {
    CaseDev& h = c->hcase[k];
    h.t = t[k];
    h.tend = tend[k];
    h.dt = 0.0001;               // DT_INITIAL, reset on every call (src/Main.c:28,193)
    h.CFLmax = CFLmax;
    h.CFLreg = CFLreg;
    h.nstep = h.nrej = h.attempts = 0;
    h.step_cap = max_steps;
    h.status = 0;
    h.nonfinite = 0;
    h.trace_n = 0;
    h.show_every = c->prm.show_every;
    h.max_attempts = c->prm.max_attempts;
    h.done = (t[k] < tend[k]) ? 0 : 1;
    any = any || !h.done;
  }
  int st = push_cases(c);
  if (st) return st;
  if (any && !c->host_loop) {
    CK(cudaMemsetAsync(c->dqueue, 0, sizeof(int) * 10, c->stream));
    CK(cudaGraphLaunch(c->gexec, c->stream));
  } else if (any) {
    // the graph body launched from the host, 16 attempts between checks of the
    // controller state (kernels of finished cases return at once); for tools that
    // cannot look inside conditional graph nodes
    CK(cudaMemsetAsync(c->dqueue, 0, sizeof(int) * 10, c->stream));
    for (;;) {
      for (int k = 0; k < 16; k++) CK(launch_attempt(c, 0, 0));
      CK(cudaMemcpyAsync(c->hcase, c->dcase, sizeof(CaseDev) * c->ncase, cudaMemcpyDeviceToHost, c->stream));
      if ((st = wait_stream(c))) return st;
      bool live = false;
      for (int k = 0; k < c->ncase; k++) live = live || !c->hcase[k].done;
      if (!live) break;
    }
  }
  return MBM_OK;
}

extern "C" int mbm_steps_batch_wait(mbm_ctx* c, double* t, int* nsteps, int* nrej) {
  if (!c || !t) return fail(c, MBM_EINVAL, "mbm_steps: bad argument");
  CK(cudaSetDevice(c->device));
  int st;
  CK(cudaMemcpyAsync(c->hcase, c->dcase, sizeof(CaseDev) * c->ncase, cudaMemcpyDeviceToHost, c->stream));
  if ((st = wait_stream(c))) return st;
  int worst = 0;
  for (int k = 0; k < c->ncase; k++) {
    const CaseDev& h = c->hcase[k];
    t[k] = h.t;
    if (nsteps) nsteps[k] = h.nstep;
    if (nrej) nrej[k] = h.nrej;
    if (h.status) worst = h.status;
  }
  if (worst == 2) return fail(c, MBM_ENONFINITE, "a stage wrote NaN or infinity, or CFL or dt became non-finite");
  if (worst == 3) return fail(c, MBM_ETIMEOUT, "a bounded device wait for a bulk copy ran out");
  if (worst == 5) return fail(c, MBM_ESTEPLIMIT, "step attempts exceeded max_attempts");
  return MBM_OK;
}

extern "C" int mbm_steps_batch(mbm_ctx* c, double* t, const double* tend, double CFLmax, double CFLreg,
                               int max_steps, int* nsteps, int* nrej) {
  int st = mbm_steps_batch_async(c, t, tend, CFLmax, CFLreg, max_steps);
  if (st) return st;
  return mbm_steps_batch_wait(c, t, nsteps, nrej);
}

extern "C" int mbm_steps_capped(mbm_ctx* c, double* t, double tend, double CFLmax, double CFLreg,
                                int max_steps, int* nsteps, int* nrej) {
  if (!c || !t) return fail(c, MBM_EINVAL, "mbm_steps: bad argument");
  std::vector<double> tt(c->ncase, *t), te(c->ncase, tend);
  std::vector<int> ns(c->ncase), nr(c->ncase);
  int st = mbm_steps_batch(c, tt.data(), te.data(), CFLmax, CFLreg, max_steps, ns.data(), nr.data());
  *t = tt[0];
  if (nsteps) *nsteps = ns[0];
  if (nrej) *nrej = nr[0];
  return st;
}

extern "C" int mbm_steps(mbm_ctx* c, double* t, double tend, double CFLmax, double CFLreg, int* nsteps,
                         int* nrej) {
  return mbm_steps_capped(c, t, tend, CFLmax, CFLreg, 0, nsteps, nrej);
}

extern "C" int mbm_config(mbm_ctx* c, int* segment_rows, int* work_items, int* ctas) {
  if (!c) return fail(c, MBM_EINVAL, "mbm_config: null context");
  int g = 0;
  for (const LimGroup& x : c->groups[0]) g = std::max(g, std::max(x.grid[0], x.grid[1]));
  if (segment_rows) *segment_rows = (int)std::lround(c->seg_rows[0]);
  if (work_items) *work_items = c->nwork[0];
  if (ctas) *ctas = g;
  return MBM_OK;
}

extern "C" int mbm_bulk_copies(mbm_ctx* c, int* on) {
  if (!c || !on) return fail(c, MBM_EINVAL, "mbm_bulk_copies: bad argument");
  *on = c->dtmap != nullptr;
  if (!c->dtmap && !c->tma_note.empty()) c->err = c->tma_note;
  return MBM_OK;
}

extern "C" int mbm_dependent_launch(mbm_ctx* c, int* on) {
  if (!c || !on) return fail(c, MBM_EINVAL, "mbm_dependent_launch: bad argument");
  *on = c->pdl && c->groups[0].size() <= 1 && c->groups[1].size() <= 1 ? 1 : 0;
  return MBM_OK;
}

extern "C" int mbm_ghost_scatter(mbm_ctx* c, int* on) {
  if (!c || !on) return fail(c, MBM_EINVAL, "mbm_ghost_scatter: bad argument");
  *on = c->gscatter ? 1 : 0;
  return MBM_OK;
}

extern "C" int mbm_config_stage(mbm_ctx* c, int heun, double* segment_rows, int* work_items, int* ctas) {
  if (!c || (heun != 0 && heun != 1)) return fail(c, MBM_EINVAL, "mbm_config_stage: bad argument");
  int g = 0;
  for (const LimGroup& x : c->groups[heun]) g = std::max(g, x.grid[heun]);
  if (segment_rows) *segment_rows = c->seg_rows[heun];
  if (work_items) *work_items = c->nwork[heun];
  if (ctas) *ctas = g;
  return MBM_OK;
}

extern "C" int mbm_attempts(mbm_ctx* c, int* attempts) {
  if (!c || !attempts) return fail(c, MBM_EINVAL, "mbm_attempts: bad argument");
  int a = 0;
  for (int k = 0; k < c->ncase; k++) a = std::max(a, c->hcase[k].attempts);
  *attempts = a;
  return MBM_OK;
}

extern "C" int mbm_case_status(mbm_ctx* c, int* status, int n) {
  if (!c || !status || n < 0 || n > c->ncase) return fail(c, MBM_EINVAL, "mbm_case_status: bad argument");
  for (int k = 0; k < n; k++) {
    const int s = c->hcase[k].status;
    status[k] = s == 2 ? MBM_ENONFINITE : s == 3 ? MBM_ETIMEOUT : s == 5 ? MBM_ESTEPLIMIT : MBM_OK;
  }
  return MBM_OK;
}

extern "C" int mbm_time_stage(mbm_ctx* c, int heun, double dt, int reps, double* ms) {
  if (!c || !ms || reps < 1 || (heun != 0 && heun != 1)) return fail(c, MBM_EINVAL, "mbm_time_stage: bad argument");
  CK(cudaSetDevice(c->device));
  for (int k = 0; k < c->ncase; k++) {
    c->hcase[k].dt = dt;
    c->hcase[k].done = 0;
  }
  int st = push_cases(c);
  if (st) return st;
  const int si = heun ? SEL_TMP : SEL_CUR, so = heun ? SEL_OTHER : SEL_TMP;
  LocalEvents ev;
  cudaEvent_t& e0 = ev.e[0];
  cudaEvent_t& e1 = ev.e[1];
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaMemsetAsync(c->dqueue, 0, sizeof(int) * 10, c->stream));
  CK(launch_stages(c, heun, si, SEL_CUR, so, 1));      // warm-up launch
  // the per-launch queue reset is a 40-byte memset, inside the timed region
  CK(cudaEventRecord(e0, c->stream));
  for (int r = 0; r < reps; r++) {
    CK(cudaMemsetAsync(c->dqueue, 0, sizeof(int) * 10, c->stream));
    CK(launch_stages(c, heun, si, SEL_CUR, so, 1));
  }
  CK(cudaEventRecord(e1, c->stream));
  CK(launch_stage_cfl(c->dblk, c->nblk, c->dcase, c->dlam, heun, c->dcfl, c->stream));
  st = wait_stream(c);
  float el = 0.f;
  if (!st) CK(cudaEventElapsedTime(&el, e0, e1));
  if (st) return st;
  *ms = el / reps;
  return MBM_OK;
}

extern "C" int mbm_trace(mbm_ctx* c, double* rec, int cap, int* n) {
  return mbm_trace_case(c, 0, rec, cap, n);
}

extern "C" int mbm_trace_case(mbm_ctx* c, int k, double* rec, int cap, int* n) {
  if (!c || k < 0 || k >= c->ncase || (cap > 0 && !rec)) return fail(c, MBM_EINVAL, "mbm_trace: bad argument");
  const int m = std::min(cap, c->hcase[k].trace_n);
  if (m > 0) {
    CK(cudaSetDevice(c->device));
    CK(cudaMemcpy(rec, c->dtrace + (size_t)k * MAX_TRACE * 4, sizeof(double) * 4 * m, cudaMemcpyDeviceToHost));
  }
  if (n) *n = m;
  return MBM_OK;
}

// ------------------------------------------------------------------ adjoint --
// Discrete adjoint of a Steps run (hand-written reverse of Update and SetBoundary,
// mbm_adjoint.cu), dt frozen from the forward run, checkpoints every k steps.

// threads of an adjoint launch: one per cell, in 128-thread tiles of 32 x 4 cells per block
static long long adj_threads(mbm_ctx* c) {
  long long n = 0;
  for (auto& d : c->hblk) n += 128LL * ((d.nxp + 31) / 32) * ((d.nyp + 3) / 4);
  return n;
}

static int adj_alloc(mbm_ctx* c, int nsteps, int every) {
  for (int k = 0; k < 9; k++)      // each one missing (mbm_replay may have made the first)
    if (!c->adj_buf[k]) CK(cudaMalloc(&c->adj_buf[k], sizeof(double) * c->layer_elems));
  if (!c->adj_scal) CK(cudaMalloc(&c->adj_scal, sizeof(double) * 2));
  if (!c->adj_part) CK(cudaMalloc(&c->adj_part, sizeof(double) * ((adj_threads(c) + 127) / 128)));
  if (!c->adj_work_ready) {   // row-marching work: strips of ASTRIP columns x 32-row segments of the non-ring cells
    const char* env = getenv("MBM_ADJ_MARCH");
    c->adj_march = env && atoi(env) == 1;
    std::vector<Work> wl;
    for (int b = 0; b < c->nblk; b++) {
      const BlockDev& d = c->hblk[b];
      const int rows = d.nyp - 2, segs = (rows + 31) / 32;
      for (int sg = 0; sg < segs; sg++) {
        const int J0 = 1 + (int)((long long)rows * sg / segs), J1 = 1 + (int)((long long)rows * (sg + 1) / segs);
        for (int I0 = 1; I0 <= d.nxp - 2; I0 += ASTRIP) wl.push_back(Work{b, I0, J0, J1});
      }
    }
    if (!c->adj_work) CK(cudaMalloc(&c->adj_work, sizeof(Work) * std::max<size_t>(1, wl.size())));
    CK(cudaMemcpyAsync(c->adj_work, wl.data(), sizeof(Work) * wl.size(), cudaMemcpyHostToDevice, c->stream));
    const int st = wait_stream(c);
    if (st) return st;
    c->adj_work_ready = true;     // the table is complete on the device
    c->adj_nwork = (int)wl.size();
    c->adj_grid = std::max(1, std::min((c->adj_nwork + 3) / 4, c->nsm * adjoint_march_ctas()));
  }
  if (!c->adj_queue) CK(cudaMalloc(&c->adj_queue, sizeof(int)));
  if (!c->adj_rstream) {
    int lo = 0, hi = 0;
    CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));    // lo: the least urgent
    CK(cudaStreamCreateWithPriority(&c->adj_rstream, cudaStreamNonBlocking, lo));
  }
  for (int k = 0; k < 2; k++) {      // each one missing
    if (!c->adj_ready[k]) CK(cudaEventCreateWithFlags(&c->adj_ready[k], cudaEventDisableTiming));
    if (!c->adj_free[k]) CK(cudaEventCreateWithFlags(&c->adj_free[k], cudaEventDisableTiming));
  }
  if (!c->adj_start) CK(cudaEventCreateWithFlags(&c->adj_start, cudaEventDisableTiming));
  if (nsteps > c->adj_nsteps || every != c->adj_every) {
    cudaFree(c->adj_ckpt);
    cudaFree(c->adj_dtlog);
    c->adj_ckpt = c->adj_dtlog = nullptr;
    for (int k = 0; k < 2; k++) {
      cudaFree(c->adj_seg[k]);
      cudaFree(c->adj_segT[k]);
      c->adj_seg[k] = c->adj_segT[k] = nullptr;
    }
    const int nck = nsteps / every + 1;
    CK(cudaMalloc(&c->adj_ckpt, sizeof(double) * c->layer_elems * nck));
    for (int k = 0; k < 2; k++) {
      CK(cudaMalloc(&c->adj_seg[k], sizeof(double) * c->layer_elems * (every + 1)));
      CK(cudaMalloc(&c->adj_segT[k], sizeof(double) * c->layer_elems * every));
    }
    CK(cudaMalloc(&c->adj_dtlog, sizeof(double) * nsteps));
    c->adj_nsteps = nsteps;
    c->adj_every = every;
  }
  return MBM_OK;
}

// the case record for frozen-dt stages: buffer selectors relative to cur = 0, not done
static int frozen_begin(mbm_ctx* c) {
  CaseDev& h = c->hcase[0];
  h.cur = 0;
  h.done = 0;
  return push_cases(c);
}

// one frozen-dt Heun step: in (full layer) -> out (full layer) through tmp (the
// stage-1 state, ghosts filled); out = nullptr stops after stage 1.  ddt points at
// the step's dt in device memory (copied into the case record on the stream, so
// consecutive steps queue without a host round trip)
static int frozen_step(mbm_ctx* c, const double* in, double* out, const double* ddt, double* tmp) {
  double* bufs[3] = {const_cast<double*>(in), out, tmp};
  PdlScope pdl_scope(c->pdl && c->groups[0].size() <= 1 && c->groups[1].size() <= 1);
  CK(launch_frozen_prep(c->dcase, ddt, c->dqueue, c->stream));
  CK(launch_stages(c, 0, SEL_CUR, SEL_CUR, SEL_TMP, 0, bufs, true));
  if (!c->gscatter) CK(launch_ghost(c->dblk, c->dcase, c->dghost, c->nghost, bufs, c->ddir, SEL_TMP, c->stream));
  if (!out) return MBM_OK;
  CK(launch_stages(c, 1, SEL_TMP, SEL_CUR, SEL_OTHER, 1, bufs, true));
  if (!c->gscatter) CK(launch_ghost(c->dblk, c->dcase, c->dghost, c->nghost, bufs, c->ddir, SEL_OTHER, c->stream));
  return MBM_OK;
}


// reverse of one step: lam (adjoint of D_{n+1}, interior) -> lam_next (adjoint of
// D_n); Tn = stage 1 of D_n with its ghost fill
static int adj_step(mbm_ctx* c, const double* Dn, const double* Tn, double dt, double* lam, double* lam_next) {
  // the three-pass kernels wait on the device for the one before
  PdlScope pdl_scope(c->pdl && !c->adj_march);
  double* lamT = c->adj_buf[2];
  double* P = c->adj_buf[3];
  const char* se = getenv("MBM_ADJ_SPLIT");     // the cell pass in two halves unless 0
  double* Pbuf = (se && atoi(se) == 0) ? nullptr : c->adj_buf[8];
  const long long nc = adj_threads(c);
  const CaseDev& h = c->hcase[0];
  // the three-pass cell pass writes every cell of lamT and lam_next in stage 2; the
  // row-marching pass writes the non-ring cells, so the ring starts at zero
  if (c->adj_march) {
    CK(cudaMemsetAsync(lamT, 0, sizeof(double) * c->layer_elems, c->stream));
    CK(cudaMemsetAsync(lam_next, 0, sizeof(double) * c->layer_elems, c->stream));
  }
  AdjArgs a{};
  a.work = c->adj_work;
  a.nwork = c->adj_nwork;
  a.queue = c->adj_queue;
  a.blk = c->dblk;
  a.nblk = c->nblk;
  a.P = P;
  a.Pb = Pbuf;
  a.knb = c->adj_scal;
  a.dt = dt;
  a.Kn = h.Kn;
  a.F = h.F;
  a.limiter = h.limiter;
  // stage 2: NEW = stage2(TMP, D_n)
  a.heun = 1;
  a.x = Tn;
  a.d0 = Dn;
  a.lout = lam;
  a.lx = lamT;
  a.ld0 = lam_next;
  if (c->adj_march) {
    CK(cudaMemsetAsync(c->adj_queue, 0, sizeof(int), c->stream));
    CK(adjoint_stage_march(a, c->adj_grid, c->stream));
  } else {
    CK(adjoint_stage(a, nc, c->adj_buf[4], c->adj_buf[5], c->adj_buf[6], c->adj_buf[7], c->stream));
  }
  CK(adjoint_ghosts(c->dblk, c->dghost, c->nghost, lamT, c->stream));
  // stage 1: TMP = stage1(D_n)
  a.heun = 0;
  a.x = Dn;
  a.d0 = Dn;
  a.lout = lamT;
  a.lx = lam_next;
  a.ld0 = nullptr;
  if (c->adj_march) {
    CK(cudaMemsetAsync(c->adj_queue, 0, sizeof(int), c->stream));
    CK(adjoint_stage_march(a, c->adj_grid, c->stream));
  } else {
    CK(adjoint_stage(a, nc, c->adj_buf[4], c->adj_buf[5], c->adj_buf[6], c->adj_buf[7], c->stream));
  }
  CK(adjoint_ghosts(c->dblk, c->dghost, c->nghost, lam_next, c->stream));
  return MBM_OK;
}

extern "C" int mbm_adjoint_run(mbm_ctx* c, double* t, int nsteps, int every, double CFLreg, double* J,
                               double* grad, double* grad_Kn, double* dts_out, double* ms) {
  if (c && c->sharded) return fail(c, MBM_EINVAL, "mbm_adjoint_run: the context holds part of a sharded case (mbm_shard_*)");
  if (!c || !t || nsteps < 1 || every < 1 || c->ncase != 1) return fail(c, MBM_EINVAL, "mbm_adjoint_run: bad argument");
  if (!c->adjoint) return fail(c, MBM_EINVAL, "mbm_adjoint_run: context created without mbm_params.adjoint");
  CK(cudaSetDevice(c->device));
  int st = adj_alloc(c, nsteps, every);
  if (st) return st;
  const size_t bytes = sizeof(double) * c->layer_elems;
  LocalEvents ev;
  cudaEvent_t& e0 = ev.e[0];
  cudaEvent_t& e1 = ev.e[1];
  cudaEvent_t& e2 = ev.e[2];
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventCreate(&e2));
  // forward: Steps with a step cap, recording dt and checkpoints (step 0 = the input state)
  CaseDev& h = c->hcase[0];
  // the last segment [tail_a, nsteps) is kept by the forward run itself (into the segment
  // buffers the reverse sweep reads first), so the sweep starts without recomputing it
  // (MBM_ADJ_TAIL=0: recomputed like the others)
  const char* te = getenv("MBM_ADJ_TAIL");
  const bool keep_tail = !(te && atoi(te) == 0);
  const int tail_seg = (nsteps - 1) / every, tail_buf = tail_seg & 1;
  CK(cudaEventRecord(e0, c->stream));
  CK(cudaMemcpyAsync(c->adj_ckpt, c->buf[h.cur], bytes, cudaMemcpyDeviceToDevice, c->stream));
  h.ckpt = c->adj_ckpt;
  h.ckpt_every = every;
  h.dtlog = c->adj_dtlog;
  h.dtlog_cap = nsteps;
  if (keep_tail) {
    h.tail_a = tail_seg * every;
    h.tail_b = nsteps;
    h.tail_d = c->adj_seg[tail_buf];
    h.tail_t = c->adj_segT[tail_buf];
    if (h.tail_a == 0) CK(cudaMemcpyAsync(h.tail_d, c->buf[h.cur], bytes, cudaMemcpyDeviceToDevice, c->stream));
  }
  int n = 0, r = 0;
  st = mbm_steps_capped(c, t, 1e300, 1.0, CFLreg, nsteps, &n, &r);
  h.ckpt = nullptr;
  h.dtlog = nullptr;
  h.ckpt_every = 0;
  h.dtlog_cap = 0;
  h.tail_d = h.tail_t = nullptr;
  h.tail_a = h.tail_b = 0;
  if (st) return st;
  if ((st = push_cases(c))) return st;
  CK(cudaEventRecord(e1, c->stream));
  std::vector<double> dts(n);
  CK(cudaMemcpy(dts.data(), c->adj_dtlog, sizeof(double) * n, cudaMemcpyDeviceToHost));
  if (dts_out) {
    for (int k = 0; k < nsteps; k++) dts_out[k] = k < n ? dts[k] : 0.0;
  }
  // functional and its gradient at the final state
  double* lam = c->adj_buf[0];
  double* lam2 = c->adj_buf[1];
  CK(cudaMemsetAsync(c->adj_scal, 0, sizeof(double) * 2, c->stream));
  CK(cudaMemsetAsync(lam, 0, bytes, c->stream));
  CK(adjoint_functional(c->dblk, c->nblk, c->buf[h.cur], lam, adj_threads(c), c->adj_part, c->adj_scal + 1,
                        c->functional, c->stream));
  // reverse sweep over segments [s*every, min((s+1)*every, n)).  The recomputation of
  // segment s-1 from its checkpoint (frozen-dt forward steps, on the low-priority
  // recomputation stream, into the other of the two segment buffers) runs beside the
  // reversal of segment s on the context stream: the forward kernels are FP64-bound,
  // the adjoint passes wait on their neighbour loads, so the two share the SMs.  The
  // recomputation touches the case record, the work counters and the CFL maxima, the
  // reversal only the adjoint buffers.  Events order buffer reuse: recomputing into a
  // buffer waits until the reversal that read it is done (adj_free), reversing a
  // segment waits for its recomputation (adj_ready).
  const int cur0 = h.cur;
  if ((st = frozen_begin(c))) return st;
  CK(cudaEventRecord(c->adj_start, c->stream));
  CK(cudaStreamWaitEvent(c->adj_rstream, c->adj_start, 0));
  bool used[2] = {false, false};
  auto recompute = [&](int sg) -> int {
    const int a = sg * every, b = std::min(n, a + every), k2 = sg & 1;
    std::swap(c->stream, c->adj_rstream);      // frozen_step issues on c->stream
    int rc = MBM_OK;
    if (used[k2] && cudaStreamWaitEvent(c->stream, c->adj_free[k2], 0) != cudaSuccess) rc = MBM_ECUDA;
    if (!rc && cudaMemcpyAsync(c->adj_seg[k2], c->adj_ckpt + (size_t)sg * c->layer_elems, bytes,
                               cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess)
      rc = MBM_ECUDA;
    // the segment's states and stage-1 states (the last step's stage 1 only)
    for (int k = a; !rc && k < b; k++)
      rc = frozen_step(c, c->adj_seg[k2] + (size_t)(k - a) * c->layer_elems,
                       k < b - 1 ? c->adj_seg[k2] + (size_t)(k - a + 1) * c->layer_elems : nullptr,
                       c->adj_dtlog + k, c->adj_segT[k2] + (size_t)(k - a) * c->layer_elems);
    if (!rc && cudaEventRecord(c->adj_ready[k2], c->stream) != cudaSuccess) rc = MBM_ECUDA;
    std::swap(c->stream, c->adj_rstream);
    used[k2] = true;
    return rc;
  };
  const int nseg = (n - 1) / every + 1;
  if (keep_tail && n == nsteps) {      // the forward run kept the last segment
    CK(cudaEventRecord(c->adj_ready[tail_buf], c->stream));
    used[tail_buf] = true;
  } else if ((st = recompute(nseg - 1))) {
    return fail(c, st, "mbm_adjoint_run: recomputation failed");
  }
  for (int sg = nseg - 1; sg >= 0; sg--) {
    const int a = sg * every, b = std::min(n, a + every), k2 = sg & 1;
    if (sg > 0 && (st = recompute(sg - 1))) return fail(c, st, "mbm_adjoint_run: recomputation failed");
    CK(cudaStreamWaitEvent(c->stream, c->adj_ready[k2], 0));
    for (int k = b - 1; k >= a; k--) {
      if ((st = adj_step(c, c->adj_seg[k2] + (size_t)(k - a) * c->layer_elems,
                         c->adj_segT[k2] + (size_t)(k - a) * c->layer_elems, dts[k], lam, lam2)))
        return st;
      std::swap(lam, lam2);
    }
    CK(cudaEventRecord(c->adj_free[k2], c->stream));
  }
  h.cur = cur0;
  h.done = 1;
  if ((st = push_cases(c))) return st;
  // the frozen stages left CFL maxima no controller read: clear them for the next run
  CK(cudaMemsetAsync(c->dlam, 0, sizeof(unsigned long long) * 6 * c->nblk, c->stream));
  CK(cudaEventRecord(e2, c->stream));
  double sc[2];
  CK(cudaMemcpyAsync(sc, c->adj_scal, sizeof sc, cudaMemcpyDeviceToHost, c->stream));
  if ((st = wait_stream(c))) return st;
  float f_ms = 0.f, a_ms = 0.f;
  CK(cudaEventElapsedTime(&f_ms, e0, e1));
  CK(cudaEventElapsedTime(&a_ms, e1, e2));
  if (J) *J = sc[1];
  if (grad_Kn) *grad_Kn = sc[0];
  if (ms) { ms[0] = f_ms; ms[1] = a_ms; }
  if (grad) {   // adjoint of the input state, array of structs per block, ghosts zero
    size_t o = 0;
    for (int b = 0; b < c->nblk; b++) {
      const BlockDev& d = c->hblk[b];
      CK(launch_planes_to_aos(lam + d.off, c->staging, d.nxp, d.nyp, d.pitch, d.plane, c->stream));
      CK(cudaMemcpyAsync(grad + o, c->staging, sizeof(double) * d.nxp * d.nyp * NV, cudaMemcpyDeviceToHost,
                         c->stream));
      if ((st = wait_stream(c))) return st;
      o += (size_t)d.nxp * d.nyp * NV;
    }
  }
  return MBM_OK;
}

// frozen-dt forward: n Heun steps of DATA with the given dt values, no controller;
// *J (may be NULL) receives the heat-flux functional of the result
extern "C" int mbm_replay(mbm_ctx* c, const double* dts, int n, double* J) {
  if (c && c->sharded) return fail(c, MBM_EINVAL, "mbm_replay: the context holds part of a sharded case (mbm_shard_*)");
  if (!c || (n > 0 && !dts) || n < 0 || c->ncase != 1) return fail(c, MBM_EINVAL, "mbm_replay: bad argument");
  CK(cudaSetDevice(c->device));
  CaseDev& h = c->hcase[0];
  int cur = h.cur, st;
  if (n > c->adj_nrep) {
    cudaFree(c->adj_dtrep);
    c->adj_dtrep = nullptr;
    c->adj_nrep = 0;
    CK(cudaMalloc(&c->adj_dtrep, sizeof(double) * n));
    c->adj_nrep = n;
  }
  if (n > 0) CK(cudaMemcpyAsync(c->adj_dtrep, dts, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
  if ((st = frozen_begin(c))) return st;     // also orders the dt copy before the host returns
  for (int k = 0; k < n; k++) {
    if ((st = frozen_step(c, c->buf[cur], c->buf[1 - cur], c->adj_dtrep + k, c->buf[2]))) return st;
    cur = 1 - cur;
  }
  h.cur = cur;
  h.done = 1;
  if ((st = push_cases(c))) return st;
  CK(cudaMemsetAsync(c->dlam, 0, sizeof(unsigned long long) * 6 * c->nblk, c->stream));
  if (J) {
    if (!c->adj_buf[0]) CK(cudaMalloc(&c->adj_buf[0], sizeof(double) * c->layer_elems));
    if (!c->adj_scal) CK(cudaMalloc(&c->adj_scal, sizeof(double) * 2));
    if (!c->adj_part) CK(cudaMalloc(&c->adj_part, sizeof(double) * ((adj_threads(c) + 127) / 128)));
    CK(cudaMemsetAsync(c->adj_scal, 0, sizeof(double) * 2, c->stream));
    CK(adjoint_functional(c->dblk, c->nblk, c->buf[cur], c->adj_buf[0], adj_threads(c), c->adj_part, c->adj_scal + 1,
                          c->functional,
                          c->stream));
    double sc[2];
    CK(cudaMemcpyAsync(sc, c->adj_scal, sizeof sc, cudaMemcpyDeviceToHost, c->stream));
    if ((st = wait_stream(c))) return st;
    *J = sc[1];
  }
  return wait_stream(c);
}

// the functional J of mbm_adjoint_run and mbm_replay
extern "C" int mbm_set_functional(mbm_ctx* c, int kind) {
  if (!c || kind < MBM_J_HEAT_FLUX || kind > MBM_J_DEVIATORIC) return fail(c, MBM_EINVAL, "mbm_set_functional: bad argument");
  c->functional = kind;
  return MBM_OK;
}

// Kn and F of every case (the globals the reference's Steps reads)
extern "C" int mbm_set_physics(mbm_ctx* c, double Kn, double F) {
  if (!c || !(Kn > 1e-100 && Kn < 1e100)) return fail(c, MBM_EINVAL, "mbm_set_physics: bad argument");
  for (int k = 0; k < c->ncase; k++) {
    c->hcase[k].Kn = Kn;
    c->hcase[k].F = F;
  }
  return push_cases(c);
}

// ---------------------------------------------------------------- sharding --
// One case split over ranks by block.  Every rank resolves the ghost map of the whole
// block table (the same on every rank) and keeps the entries of its own blocks; an
// entry whose source cell lies on another rank reads it from a receive buffer.  The
// cells rank p sends to rank r are those entries of r's blocks with a source on p,
// in the order of the global map, so both sides agree on the order without talking.
static int shard_split(const mbm_block_desc* blocks, int nblocks, const int* owner, int nranks, int rank,
                       std::vector<Resolved>& res, std::vector<int>& dir_off, int& ndir,
                       std::vector<std::array<int, 2>>& send, std::vector<std::array<int, 3>>& recv,
                       std::vector<int>& send_counts, std::vector<int>& recv_counts, std::string& why) {
  if (!owner || nranks < 1 || rank < 0 || rank >= nranks) { why = "bad owner table, rank or rank count"; return MBM_EINVAL; }
  if (validate(blocks, nblocks, why) != MBM_OK) return MBM_EINVAL;
  for (int b = 0; b < nblocks; b++)
    if (owner[b] < 0 || owner[b] >= nranks) { why = "block " + std::to_string(b + 1) + ": owner out of range"; return MBM_EINVAL; }
  if (resolve_ghosts(blocks, nblocks, res, dir_off, ndir, why) != MBM_OK) return MBM_EINVAL;
  std::vector<std::vector<std::array<int, 2>>> S(nranks);
  std::vector<std::vector<std::array<int, 3>>> R(nranks);
  for (Resolved& r : res) {
    if (r.src < 0) continue;
    const int od = owner[r.dst_blk], os = owner[r.src_blk];
    if (od == os) continue;
    if (os == rank) S[od].push_back({r.src_blk, r.src});
    if (od == rank) {
      r.remote = (int)R[os].size();   // index within the peer's segment, offset added below
      R[os].push_back({r.dst_blk, r.dst_cell, r.flags});
    }
  }
  send_counts.assign(nranks, 0);
  recv_counts.assign(nranks, 0);
  std::vector<int> roff(nranks, 0);
  send.clear();
  recv.clear();
  for (int p = 0; p < nranks; p++) {
    send_counts[p] = (int)S[p].size();
    recv_counts[p] = (int)R[p].size();
    roff[p] = (int)recv.size();
    send.insert(send.end(), S[p].begin(), S[p].end());
    recv.insert(recv.end(), R[p].begin(), R[p].end());
  }
  for (Resolved& r : res)
    if (r.remote >= 0) r.remote += roff[owner[r.src_blk]];
  return MBM_OK;
}

extern "C" int mbm_shard_plan(const mbm_block_desc* blocks, int nblocks, const int* owner, int nranks, int rank,
                              int* send_counts, int* recv_counts, int* send_cells, int* recv_cells, int cap) {
  std::string why;
  std::vector<Resolved> res;
  std::vector<int> dir_off, sc, rc;
  std::vector<std::array<int, 2>> send;
  std::vector<std::array<int, 3>> recv;
  int ndir = 0;
  if (shard_split(blocks, nblocks, owner, nranks, rank, res, dir_off, ndir, send, recv, sc, rc, why) != MBM_OK)
    return fail(nullptr, MBM_EINVAL, why);
  for (int p = 0; p < nranks; p++) {
    if (send_counts) send_counts[p] = sc[p];
    if (recv_counts) recv_counts[p] = rc[p];
  }
  for (int i = 0; i < (int)send.size() && i < cap && send_cells; i++) {
    send_cells[2 * i] = send[i][0];
    send_cells[2 * i + 1] = send[i][1];
  }
  for (int i = 0; i < (int)recv.size() && i < cap && recv_cells; i++)
    for (int k = 0; k < 3; k++) recv_cells[3 * i + k] = recv[i][k];
  return MBM_OK;
}

extern "C" int mbm_create_sharded(const mbm_block_desc* blocks, int nblocks, const int* owner, int nranks,
                                  int rank, const mbm_params* params, mbm_ctx** out) {
  if (!out || !params) return fail(nullptr, MBM_EINVAL, "null argument");
  *out = nullptr;
  if (params->mode != MBM_MODE_EXACT && params->mode != MBM_MODE_FAST)
    return fail(nullptr, MBM_EINVAL, "unknown arithmetic mode");
  if (params->limiter < 0 || params->limiter > 4) return fail(nullptr, MBM_EINVAL, "limiter code must be 0..4");
  if (!(params->Kn > 1e-100 && params->Kn < 1e100)) return fail(nullptr, MBM_EINVAL, "Kn must be in (1e-100, 1e100)");
  std::string why;
  std::vector<Resolved> res;
  std::vector<int> dir_off, sc, rc;
  std::vector<std::array<int, 2>> send;
  std::vector<std::array<int, 3>> recv;
  int ndir = 0;
  if (shard_split(blocks, nblocks, owner, nranks, rank, res, dir_off, ndir, send, recv, sc, rc, why) != MBM_OK)
    return fail(nullptr, MBM_EINVAL, why);
  std::vector<int> g2l(nblocks, -1);
  std::vector<mbm_block_desc> loc;
  for (int b = 0; b < nblocks; b++)
    if (owner[b] == rank) {
      g2l[b] = (int)loc.size();
      loc.push_back(blocks[b]);
    }
  if (loc.empty()) return fail(nullptr, MBM_EINVAL, "rank " + std::to_string(rank) + " owns no block");
  for (auto& d : loc)   // the resolved map carries the interfaces; codes of remote partners read as open
    for (int s = 0; s < 4; s++)
      if (d.bc[s] > 0) d.bc[s] = g2l[d.bc[s] - 1] >= 0 ? g2l[d.bc[s] - 1] + 1 : 0;
  std::vector<Resolved> lres;
  for (const Resolved& r : res) {
    if (g2l[r.dst_blk] < 0) continue;
    Resolved q = r;
    q.dst_blk = g2l[r.dst_blk];
    if (r.src >= 0 && r.remote < 0) q.src_blk = g2l[r.src_blk];
    lres.push_back(q);
  }
  std::vector<int> ldir((size_t)loc.size() * 4, -1);
  for (int b = 0; b < nblocks; b++)
    if (g2l[b] >= 0)
      for (int s = 0; s < 4; s++) ldir[(size_t)g2l[b] * 4 + s] = dir_off[(size_t)b * 4 + s];
  ShardSetup setup;
  setup.dir_off = dir_off;
  for (int b = 0; b < nblocks; b++)
    for (int s2 = 0; s2 < 4; s2++) setup.nt.push_back(s2 < 2 ? blocks[b].ny + 2 * NG : blocks[b].nx + 2 * NG);
  setup.send_counts = sc;
  setup.recv_counts = rc;
  for (const auto& e : send) setup.send.push_back({g2l[e[0]], e[1]});
  mbm_case_desc one;
  one.first_block = 0;
  one.nblocks = (int)loc.size();
  one.Kn = params->Kn;
  one.F = params->F;
  one.limiter = params->limiter;
  std::vector<int> blk_case(loc.size(), 0);
  return create_impl(loc, blk_case, &one, 1, params, lres, ldir, ndir, &setup, out);
}

static int need_shard(mbm_ctx* c, const char* what) {
  if (!c) return fail(nullptr, MBM_EINVAL, std::string(what) + ": null context");
  if (!c->sharded) return fail(c, MBM_EINVAL, std::string(what) + ": context is not sharded");
  return MBM_OK;
}

extern "C" int mbm_shard_buffers(mbm_ctx* c, int* send_counts, int* recv_counts, int nranks, double** send,
                                 double** recv, double** cfl) {
  int st = need_shard(c, "mbm_shard_buffers");
  if (st) return st;
  if (nranks != (int)c->send_counts.size()) return fail(c, MBM_EINVAL, "mbm_shard_buffers: wrong rank count");
  for (int p = 0; p < nranks; p++) {
    if (send_counts) send_counts[p] = c->send_counts[p];
    if (recv_counts) recv_counts[p] = c->recv_counts[p];
  }
  if (send) *send = c->shard_send;
  if (recv) *recv = c->shard_recv;
  if (cfl) *cfl = c->shard_cfl;
  return MBM_OK;
}

// Dirichlet values of any block's edge: a ghost cell at a corner may take its value
// from the Dirichlet row of a block another rank owns, so every rank holds them all
extern "C" int mbm_shard_set_dirichlet(mbm_ctx* c, int block, int side, const double* values) {
  int st = need_shard(c, "mbm_shard_set_dirichlet");
  if (st) return st;
  if (!values || block < 0 || block * 4 >= (int)c->shard_dir_off.size() || side < 0 || side > 3)
    return fail(c, MBM_EINVAL, "mbm_shard_set_dirichlet: bad argument");
  const int row = c->shard_dir_off[block * 4 + side];
  if (row < 0) return fail(c, MBM_EINVAL, "mbm_shard_set_dirichlet: edge is not a Dirichlet edge");
  CK(cudaSetDevice(c->device));
  CK(cudaMemcpyAsync(c->ddir + (size_t)row * NV, values, sizeof(double) * c->shard_nt[block * 4 + side] * NG * NV,
                     cudaMemcpyHostToDevice, c->stream));
  return wait_stream(c);
}

extern "C" int mbm_shard_begin(mbm_ctx* c, double t, double tend, double CFLmax, double CFLreg, int max_steps) {
  int st = need_shard(c, "mbm_shard_begin");
  if (st) return st;
  if (max_steps < 0) return fail(c, MBM_EINVAL, "mbm_shard_begin: bad argument");
  CK(cudaSetDevice(c->device));
  CaseDev& h = c->hcase[0];
  h.t = t;
  h.tend = tend;
  h.dt = 0.0001;               // DT_INITIAL, reset on every call (src/Main.c:28,193)
  h.CFLmax = CFLmax;
  h.CFLreg = CFLreg;
  h.nstep = h.nrej = h.attempts = 0;
  h.step_cap = max_steps;
  h.status = 0;
  h.nonfinite = 0;
  h.trace_n = 0;
  h.show_every = c->prm.show_every;
  h.max_attempts = c->prm.max_attempts;
  h.done = (t < tend) ? 0 : 1;
  return push_cases(c);
}

extern "C" int mbm_shard_stage(mbm_ctx* c, int heun) {
  int st = need_shard(c, "mbm_shard_stage");
  if (st) return st;
  if (heun != 0 && heun != 1) return fail(c, MBM_EINVAL, "mbm_shard_stage: bad argument");
  CK(cudaSetDevice(c->device));
  CK(cudaMemsetAsync(c->dqueue + heun * 5, 0, sizeof(int) * 5, c->stream));
  CK(launch_stages(c, heun, heun ? SEL_TMP : SEL_CUR, SEL_CUR, heun ? SEL_OTHER : SEL_TMP, 1));
  return MBM_OK;
}

extern "C" int mbm_shard_pack(mbm_ctx* c, int layer) {
  int st = need_shard(c, "mbm_shard_pack");
  if (st) return st;
  if (bad_layer(layer)) return fail(c, MBM_EINVAL, "mbm_shard_pack: bad layer");
  CK(cudaSetDevice(c->device));
  CK(launch_shard_pack(c->dblk, c->dcase, c->dsend_list, c->nsend, c->buf, layer_sel(layer), c->shard_send, c->stream));
  return MBM_OK;
}

extern "C" int mbm_shard_fill(mbm_ctx* c, int layer) {
  int st = need_shard(c, "mbm_shard_fill");
  if (st) return st;
  if (bad_layer(layer)) return fail(c, MBM_EINVAL, "mbm_shard_fill: bad layer");
  CK(cudaSetDevice(c->device));
  const bool was_done = c->hcase[0].done != 0;
  if (was_done) {              // the fill kernel skips finished cases: the initial fill runs between calls
    c->hcase[0].done = 0;
    if ((st = push_cases(c))) return st;
  }
  CK(launch_ghost(c->dblk, c->dcase, c->dghost, c->nghost, c->buf, c->ddir, layer_sel(layer), c->stream,
                  c->shard_recv));
  if (was_done) {
    c->hcase[0].done = 1;
    if ((st = push_cases(c))) return st;
  }
  return MBM_OK;
}

extern "C" int mbm_shard_cfl(mbm_ctx* c) {
  int st = need_shard(c, "mbm_shard_cfl");
  if (st) return st;
  CK(cudaSetDevice(c->device));
  CK(launch_shard_cfl(c->dcase, c->dblk, c->nblk, c->dlam, c->shard_cfl, c->stream));
  return MBM_OK;
}

extern "C" int mbm_shard_control(mbm_ctx* c, int* done) {
  int st = need_shard(c, "mbm_shard_control");
  if (st) return st;
  CK(cudaSetDevice(c->device));
  CK(launch_control_ext(c->dcase, c->dblk, c->dlam, c->dtrace, c->dqueue, c->shard_cfl, c->stream));
  if (!done) return MBM_OK;    // enqueued only: attempts after the last one are no-ops on the device
  CK(cudaMemcpyAsync(c->hcase, c->dcase, sizeof(CaseDev), cudaMemcpyDeviceToHost, c->stream));
  if ((st = wait_stream(c))) return st;
  *done = c->hcase[0].done;
  return MBM_OK;
}

extern "C" int mbm_shard_end(mbm_ctx* c, double* t, int* nsteps, int* nrej) {
  int st = need_shard(c, "mbm_shard_end");
  if (st) return st;
  const CaseDev& h = c->hcase[0];
  if (t) *t = h.t;
  if (nsteps) *nsteps = h.nstep;
  if (nrej) *nrej = h.nrej;
  if (h.status == 2) return fail(c, MBM_ENONFINITE, "a stage wrote NaN or infinity, or CFL or dt became non-finite");
  if (h.status == 3) return fail(c, MBM_ETIMEOUT, "a bounded device wait for a bulk copy ran out");
  if (h.status == 5) return fail(c, MBM_ESTEPLIMIT, "step attempts exceeded max_attempts");
  return MBM_OK;
}

// ------------------------------------------------------------------- misc --
extern "C" int mbm_ghost_map(const mbm_block_desc* blocks, int nblocks, int* entries, int cap, int* n) {
  std::string why;
  if (validate(blocks, nblocks, why) != MBM_OK) return fail(nullptr, MBM_EINVAL, why);
  std::vector<Resolved> res;
  std::vector<int> dir_off;
  int ndir = 0;
  if (resolve_ghosts(blocks, nblocks, res, dir_off, ndir, why) != MBM_OK) return fail(nullptr, MBM_EINVAL, why);
  if (n) *n = (int)res.size();
  if (entries) {
    const int k = std::min<int>(cap, (int)res.size());
    for (int i = 0; i < k; i++) {
      entries[4 * i + 0] = res[i].dst_blk;
      entries[4 * i + 1] = res[i].dst_cell;
      entries[4 * i + 2] = res[i].src;
      entries[4 * i + 3] = res[i].src_blk | (res[i].flags << 16);
    }
  }
  return MBM_OK;
}

extern "C" const char* mbm_strerror(int s) {
  switch (s) {
    case MBM_OK: return "ok";
    case MBM_EINVAL: return "invalid argument";
    case MBM_ENONFINITE: return "non-finite state, CFL or time step";
    case MBM_ETIMEOUT: return "device wait timed out";
    case MBM_ECUDA: return "CUDA error";
    case MBM_ENOMEM: return "device out of memory";
    case MBM_ESTEPLIMIT: return "step attempt limit reached";
    case MBM_ENODEV: return "no CUDA device";
  }
  return "unknown status";
}

extern "C" const char* mbm_last_error(mbm_ctx* c) { return c ? c->err.c_str() : g_create_error.c_str(); }

extern "C" int mbm_version(void) { return 1; }
