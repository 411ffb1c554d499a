// mbm_host.cu -- the C ABI (include/mbm_b200.h): context, block validation, the
// resolved ghost map, the warp work table, the device-side step loop as a CUDA
// graph with a conditional while node, and the layer transfers.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/mbm_b200.h"
#include "mbm_internal.h"

namespace mbm {
cudaError_t launch_stage(int lim, const StageArgs& a, int grid, cudaStream_t s);
cudaError_t launch_ghost(const BlockDev* blk, const CaseDev* cases, const GhostEntry* map, int n,
                         double* const buf[3], const double* dirichlet, int sel, cudaStream_t s);
cudaError_t launch_control(CaseDev* cases, int ncases, const BlockDev* blk, unsigned long long* lam,
                           double* trace, cudaGraphConditionalHandle h, int use_handle,
                           cudaStream_t s);
cudaError_t launch_stage_cfl(const BlockDev* blk, int nblk, const CaseDev* cases,
                             unsigned long long* lam, int stage, double* out, cudaStream_t s);
cudaError_t launch_aos_to_planes(const double* aos, double* dst, int nxp, int nyp, int pitch,
                                 long long plane, cudaStream_t s);
cudaError_t launch_planes_to_aos(const double* src, double* aos, int nxp, int nyp, int pitch,
                                 long long plane, cudaStream_t s);
}  // namespace mbm

using namespace mbm;

static thread_local std::string g_create_error;

struct mbm_ctx {
  mbm_params prm{};
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int nblk = 0;
  std::vector<mbm_block_desc> desc;
  std::vector<BlockDev> hblk;
  BlockDev* dblk = nullptr;
  long long layer_elems = 0;
  double* buf[3] = {nullptr, nullptr, nullptr};
  double* staging = nullptr;        // array-of-structs transfer buffer, one block
  GhostEntry* dghost = nullptr;
  int nghost = 0;
  std::vector<int> dir_off;         // [block*4+side] -> first Dirichlet row, -1 if none
  double* ddir = nullptr;
  int ndir = 0;
  Work* dwork = nullptr;
  int nwork = 0;
  int grid = 0;
  CaseDev* dcase = nullptr;
  CaseDev* hcase = nullptr;         // pinned mirror
  unsigned long long* dlam = nullptr;
  double* dtrace = nullptr;
  double* dcfl = nullptr;           // per-block stage CFL for mbm_update
  double* hcfl = nullptr;           // pinned
  cudaEvent_t ev = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  std::string err;
};

// ------------------------------------------------------------------ helpers --
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

static int validate(const mbm_block_desc* b, int n, std::string& why) {
  if (!b || n < 1 || n > 65535) { why = "need 1..65535 blocks"; return MBM_EINVAL; }
  for (int i = 0; i < n; i++) {
    if (b[i].nx < 1 || b[i].ny < 1 || b[i].nx > (1 << 20) || b[i].ny > (1 << 20)) {
      why = "block " + std::to_string(i + 1) + ": bad cell counts"; return MBM_EINVAL;
    }
    if (!(b[i].dx > 0) || !(b[i].dy > 0)) { why = "block " + std::to_string(i + 1) + ": dx, dy must be > 0"; return MBM_EINVAL; }
    for (int s = 0; s < 4; s++) {
      int code = b[i].bc[s];
      if (code > n) { why = "block " + std::to_string(i + 1) + ": sync partner " + std::to_string(code) + " does not exist"; return MBM_EINVAL; }
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
struct Resolved { int dst_blk, dst_cell, src, src_blk, flags; };
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

static int build_work(const std::vector<BlockDev>& blk, int seg_rows, std::vector<Work>& w) {
  w.clear();
  for (int b = 0; b < (int)blk.size(); b++) {
    const int nxp = blk[b].nxp, nyp = blk[b].nyp;
    const int nfx = nxp - 3, nfy = nyp - 3;          // face positions 1 .. nxp-3 / nyp-3
    const int strips = (nfx + STRIP - 1) / STRIP;
    const int segs = std::max(1, (nfy + seg_rows - 1) / seg_rows);
    for (int s = 0; s < segs; s++) {
      // equal-sized segments over face rows [1, nyp-3], the last one reaching nyp-2
      const int J0 = 1 + (int)((long long)nfy * s / segs);
      const int J1 = 1 + (int)((long long)nfy * (s + 1) / segs);
      for (int k = 0; k < strips; k++) w.push_back(Work{b, 1 + STRIP * k, J0, J1});
    }
  }
  return (int)w.size();
}

extern "C" int mbm_create(const mbm_block_desc* blocks, int nblocks, const mbm_params* params,
                          mbm_ctx** out) {
  mbm_ctx* c = nullptr;
  if (!out || !params) return fail(nullptr, MBM_EINVAL, "null argument");
  *out = nullptr;
  std::string why;
  if (validate(blocks, nblocks, why) != MBM_OK) return fail(nullptr, MBM_EINVAL, why);
  if (params->limiter < 0 || params->limiter > 4) return fail(nullptr, MBM_EINVAL, "limiter code must be 0..4");
  if (params->mode != MBM_MODE_EXACT) return fail(nullptr, MBM_EINVAL, "unknown arithmetic mode");
  if (!(params->Kn > 0)) return fail(nullptr, MBM_EINVAL, "Kn must be > 0");
  std::vector<Resolved> res;
  std::vector<int> dir_off;
  int ndir = 0;
  if (resolve_ghosts(blocks, nblocks, res, dir_off, ndir, why) != MBM_OK)
    return fail(nullptr, MBM_EINVAL, why);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(nullptr, MBM_ENODEV, "no CUDA device");
  if (params->device < 0 || params->device >= ndev) return fail(nullptr, MBM_EINVAL, "bad device ordinal");

  c = new mbm_ctx();
  c->prm = *params;
  if (c->prm.max_attempts <= 0) c->prm.max_attempts = 10000000;
  c->device = params->device;
  c->nblk = nblocks;
  c->desc.assign(blocks, blocks + nblocks);
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

  // block table and layer layout
  long long off = 0, max_cells = 0;
  for (int b = 0; b < nblocks; b++) {
    BlockDev d{};
    d.nxp = blocks[b].nx + 2 * NG;
    d.nyp = blocks[b].ny + 2 * NG;
    d.pitch = pitch_of(d.nxp);
    d.case_id = 0;
    d.plane = ((long long)d.pitch * d.nyp + 31) & ~31LL;
    d.off = off;
    d.dx = blocks[b].dx;
    d.dy = blocks[b].dy;
    off += d.plane * NV;
    max_cells = std::max(max_cells, (long long)d.nxp * d.nyp);
    c->hblk.push_back(d);
  }
  c->layer_elems = off;
  for (int l = 0; l < 3; l++) {
    CKC(cudaMalloc(&c->buf[l], sizeof(double) * off));
    CKC(cudaMemsetAsync(c->buf[l], 0, sizeof(double) * off, c->stream));
  }
  CKC(cudaMalloc(&c->staging, sizeof(double) * max_cells * NV));
  CKC(cudaMalloc(&c->dblk, sizeof(BlockDev) * nblocks));
  CKC(cudaMemcpyAsync(c->dblk, c->hblk.data(), sizeof(BlockDev) * nblocks, cudaMemcpyHostToDevice, c->stream));

  // ghost map in device element indices
  std::vector<GhostEntry> gm(res.size());
  for (size_t i = 0; i < res.size(); i++) {
    const Resolved& r = res[i];
    const BlockDev& D = c->hblk[r.dst_blk];
    GhostEntry e;
    e.dst_blk = r.dst_blk;
    e.dst = (r.dst_cell / D.nxp) * D.pitch + r.dst_cell % D.nxp + 1;
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

  // work table and grid
  int sm = 0, per_sm = 0;
  CKC(cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, c->device));
  per_sm = 4;
  long long strip_rows = 0;
  for (auto& d : c->hblk) strip_rows += (long long)((d.nxp - 3 + STRIP - 1) / STRIP) * (d.nyp - 3);
  int seg = params->segment_rows;
  if (seg <= 0) {
    const long long target = 2LL * sm * per_sm * 4;   // two warp items per resident warp
    seg = (int)std::max<long long>(32, (strip_rows + target - 1) / target);
  }
  std::vector<Work> work;
  c->nwork = build_work(c->hblk, seg, work);
  CKC(cudaMalloc(&c->dwork, sizeof(Work) * work.size()));
  CKC(cudaMemcpyAsync(c->dwork, work.data(), sizeof(Work) * work.size(), cudaMemcpyHostToDevice, c->stream));
  c->grid = (int)std::min<long long>((c->nwork + 3) / 4, (long long)sm * per_sm);

  // controller, maxima, trace, per-block CFL
  CKC(cudaMalloc(&c->dcase, sizeof(CaseDev)));
  CKC(cudaMallocHost(&c->hcase, sizeof(CaseDev)));
  memset(c->hcase, 0, sizeof(CaseDev));
  c->hcase->Kn = params->Kn;
  c->hcase->F = params->F;
  c->hcase->limiter = params->limiter;
  c->hcase->cur = 0;
  c->hcase->done = 1;
  c->hcase->blk0 = 0;
  c->hcase->nblk = nblocks;
  c->hcase->max_attempts = c->prm.max_attempts;
  CKC(cudaMemcpyAsync(c->dcase, c->hcase, sizeof(CaseDev), cudaMemcpyHostToDevice, c->stream));
  CKC(cudaMalloc(&c->dlam, sizeof(unsigned long long) * 6 * nblocks));
  CKC(cudaMemsetAsync(c->dlam, 0, sizeof(unsigned long long) * 6 * nblocks, c->stream));
  CKC(cudaMalloc(&c->dtrace, sizeof(double) * 4 * MAX_TRACE));
  CKC(cudaMalloc(&c->dcfl, sizeof(double) * nblocks));
  CKC(cudaMallocHost(&c->hcfl, sizeof(double) * nblocks));

  // the step loop: while (any case live) { stage 1; fill TMP; stage 2; fill NEW; control }
  {
    cudaGraphConditionalHandle h;
    CKC(cudaGraphCreate(&c->graph, 0));
    CKC(cudaGraphConditionalHandleCreate(&h, c->graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    CKC(cudaGraphAddNode(&node, c->graph, nullptr, 0, &np));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    CKC(cudaStreamBeginCaptureToGraph(c->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    StageArgs a{};
    a.blk = c->dblk; a.work = c->dwork; a.nwork = c->nwork; a.cases = c->dcase;
    for (int l = 0; l < 3; l++) a.buf[l] = c->buf[l];
    a.lam = c->dlam;
    a.sel_in = SEL_CUR; a.sel_d0 = SEL_CUR; a.sel_out = SEL_TMP; a.heun = 0;
    cudaError_t e1 = launch_stage(params->limiter, a, c->grid, c->stream);
    cudaError_t e2 = launch_ghost(c->dblk, c->dcase, c->dghost, c->nghost, c->buf, c->ddir, SEL_TMP, c->stream);
    a.sel_in = SEL_TMP; a.sel_d0 = SEL_CUR; a.sel_out = SEL_OTHER; a.heun = 1;
    cudaError_t e3 = launch_stage(params->limiter, a, c->grid, c->stream);
    cudaError_t e4 = launch_ghost(c->dblk, c->dcase, c->dghost, c->nghost, c->buf, c->ddir, SEL_OTHER, c->stream);
    cudaError_t e5 = launch_control(c->dcase, 1, c->dblk, c->dlam, c->dtrace, h, 1, c->stream);
    cudaGraph_t captured = nullptr;
    CKC(cudaStreamEndCapture(c->stream, &captured));
    CKC(e1); CKC(e2); CKC(e3); CKC(e4); CKC(e5);
    CKC(cudaGraphInstantiate(&c->gexec, c->graph, 0));
  }
  int st = wait_stream(c);
  if (st != MBM_OK) return bail(st);
  *out = c;
  return MBM_OK;
#undef CKC
}

extern "C" int mbm_destroy(mbm_ctx* c) {
  if (!c) return MBM_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->gexec) cudaGraphExecDestroy(c->gexec);
  if (c->graph) cudaGraphDestroy(c->graph);
  for (int l = 0; l < 3; l++) cudaFree(c->buf[l]);
  cudaFree(c->staging);
  cudaFree(c->dblk);
  cudaFree(c->dghost);
  cudaFree(c->ddir);
  cudaFree(c->dwork);
  cudaFree(c->dcase);
  if (c->hcase) cudaFreeHost(c->hcase);
  cudaFree(c->dlam);
  cudaFree(c->dtrace);
  cudaFree(c->dcfl);
  if (c->hcfl) cudaFreeHost(c->hcfl);
  if (c->ev) cudaEventDestroy(c->ev);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return MBM_OK;
}

// ---------------------------------------------------------------- transfers --
static int layer_sel(int layer) {
  return layer == MBM_L_DATA ? SEL_CUR : layer == MBM_L_NEW ? SEL_OTHER : SEL_TMP;
}

static bool bad_layer(int layer) { return layer < 0 || layer > 2; }

extern "C" int mbm_upload(mbm_ctx* c, int layer, int block, const double* cells) {
  if (!c || !cells || bad_layer(layer) || block < 0 || block >= c->nblk) return fail(c, MBM_EINVAL, "mbm_upload: bad argument");
  CK(cudaSetDevice(c->device));
  const BlockDev& d = c->hblk[block];
  const int phys = phys_layer(layer_sel(layer), c->hcase->cur);
  CK(cudaMemcpyAsync(c->staging, cells, sizeof(double) * d.nxp * d.nyp * NV, cudaMemcpyHostToDevice, c->stream));
  CK(launch_aos_to_planes(c->staging, c->buf[phys] + d.off, d.nxp, d.nyp, d.pitch, d.plane, c->stream));
  return wait_stream(c);
}

extern "C" int mbm_download(mbm_ctx* c, int layer, int block, double* cells) {
  if (!c || !cells || bad_layer(layer) || block < 0 || block >= c->nblk) return fail(c, MBM_EINVAL, "mbm_download: bad argument");
  CK(cudaSetDevice(c->device));
  const BlockDev& d = c->hblk[block];
  const int phys = phys_layer(layer_sel(layer), c->hcase->cur);
  CK(launch_planes_to_aos(c->buf[phys] + d.off, c->staging, d.nxp, d.nyp, d.pitch, d.plane, c->stream));
  CK(cudaMemcpyAsync(cells, c->staging, sizeof(double) * d.nxp * d.nyp * NV, cudaMemcpyDeviceToHost, c->stream));
  return wait_stream(c);
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
static int push_case(mbm_ctx* c) {
  CK(cudaMemcpyAsync(c->dcase, c->hcase, sizeof(CaseDev), cudaMemcpyHostToDevice, c->stream));
  return MBM_OK;
}

extern "C" int mbm_set_boundary(mbm_ctx* c, int layer, double t) {
  (void)t;   // Dirichlet values are the host-set table; the reference's states are steady
  if (!c || bad_layer(layer)) return fail(c, MBM_EINVAL, "mbm_set_boundary: bad argument");
  CK(cudaSetDevice(c->device));
  c->hcase->done = 0;
  int st = push_case(c);
  if (st) return st;
  CK(launch_ghost(c->dblk, c->dcase, c->dghost, c->nghost, c->buf, c->ddir, layer_sel(layer), c->stream));
  return wait_stream(c);
}

static int run_stage(mbm_ctx* c, int out_layer, int in_layer, int d0_layer, int heun, double* cfl) {
  StageArgs a{};
  a.blk = c->dblk; a.work = c->dwork; a.nwork = c->nwork; a.cases = c->dcase;
  for (int l = 0; l < 3; l++) a.buf[l] = c->buf[l];
  a.lam = c->dlam;
  a.sel_in = layer_sel(in_layer); a.sel_d0 = layer_sel(d0_layer); a.sel_out = layer_sel(out_layer);
  a.heun = heun;
  CK(launch_stage(c->prm.limiter, a, c->grid, c->stream));
  CK(launch_stage_cfl(c->dblk, c->nblk, c->dcase, c->dlam, heun, c->dcfl, c->stream));
  CK(cudaMemcpyAsync(c->hcfl, c->dcfl, sizeof(double) * c->nblk, cudaMemcpyDeviceToHost, c->stream));
  int st = wait_stream(c);
  if (st) return st;
  if (cfl) memcpy(cfl, c->hcfl, sizeof(double) * c->nblk);
  return MBM_OK;
}

extern "C" int mbm_update(mbm_ctx* c, int out_layer, int in_layer, int data0_layer, double dt,
                          double t, int heun, double* cfl) {
  if (!c || bad_layer(out_layer) || bad_layer(in_layer) || bad_layer(data0_layer) || (heun != 0 && heun != 1) ||
      out_layer == in_layer || out_layer == data0_layer)
    return fail(c, MBM_EINVAL, "mbm_update: bad argument");
  CK(cudaSetDevice(c->device));
  c->hcase->dt = dt;
  c->hcase->t = t;
  c->hcase->done = 0;
  int st = push_case(c);
  if (st) return st;
  return run_stage(c, out_layer, in_layer, data0_layer, heun, cfl);
}

extern "C" int mbm_time_update(mbm_ctx* c, double dt, double t, double* cfl) {
  if (!c) return fail(c, MBM_EINVAL, "mbm_time_update: null context");
  std::vector<double> v(c->nblk);
  double c1 = 0.0, c2 = 0.0;
  int st = mbm_update(c, MBM_L_TMP, MBM_L_DATA, MBM_L_DATA, dt, t, 0, v.data());
  if (st) return st;
  for (double x : v) if (x > c1) c1 = x;
  if ((st = mbm_set_boundary(c, MBM_L_TMP, t + dt))) return st;
  st = run_stage(c, MBM_L_NEW, MBM_L_TMP, MBM_L_DATA, 1, v.data());
  if (st) return st;
  for (double x : v) if (x > c2) c2 = x;
  if ((st = mbm_set_boundary(c, MBM_L_NEW, t + dt))) return st;
  if (cfl) *cfl = c1 > (c2 > 0.0 ? c2 : 0.0) ? c1 : (c2 > 0.0 ? c2 : 0.0);
  return MBM_OK;
}

extern "C" int mbm_steps_capped(mbm_ctx* c, double* t, double tend, double CFLmax, double CFLreg,
                                int max_steps, int* nsteps, int* nrej) {
  if (!c || !t || max_steps < 0) return fail(c, MBM_EINVAL, "mbm_steps: bad argument");
  CK(cudaSetDevice(c->device));
  CaseDev& h = *c->hcase;
  h.t = *t;
  h.tend = tend;
  h.dt = 0.0001;                 // DT_INITIAL, reset on every call (src/Main.c:28,193)
  h.CFLmax = CFLmax;
  h.CFLreg = CFLreg;
  h.nstep = h.nrej = h.attempts = 0;
  h.step_cap = max_steps;
  h.status = 0;
  h.trace_n = 0;
  h.show_every = c->prm.show_every;
  h.max_attempts = c->prm.max_attempts;
  h.done = (*t < tend) ? 0 : 1;
  int st = push_case(c);
  if (st) return st;
  if (!h.done) CK(cudaGraphLaunch(c->gexec, c->stream));
  CK(cudaMemcpyAsync(c->hcase, c->dcase, sizeof(CaseDev), cudaMemcpyDeviceToHost, c->stream));
  if ((st = wait_stream(c))) return st;
  *t = h.t;
  if (nsteps) *nsteps = h.nstep;
  if (nrej) *nrej = h.nrej;
  if (h.status == 2) return fail(c, MBM_ENONFINITE, "CFL or dt became non-finite");
  if (h.status == 5) return fail(c, MBM_ESTEPLIMIT, "step attempts exceeded max_attempts");
  return MBM_OK;
}

extern "C" int mbm_steps(mbm_ctx* c, double* t, double tend, double CFLmax, double CFLreg, int* nsteps,
                         int* nrej) {
  return mbm_steps_capped(c, t, tend, CFLmax, CFLreg, 0, nsteps, nrej);
}

extern "C" int mbm_attempts(mbm_ctx* c, int* attempts) {
  if (!c || !attempts) return fail(c, MBM_EINVAL, "mbm_attempts: bad argument");
  *attempts = c->hcase->attempts;
  return MBM_OK;
}

extern "C" int mbm_time_stage(mbm_ctx* c, int heun, double dt, int reps, double* ms) {
  if (!c || !ms || reps < 1 || (heun != 0 && heun != 1)) return fail(c, MBM_EINVAL, "mbm_time_stage: bad argument");
  CK(cudaSetDevice(c->device));
  c->hcase->dt = dt;
  c->hcase->done = 0;
  int st = push_case(c);
  if (st) return st;
  StageArgs a{};
  a.blk = c->dblk; a.work = c->dwork; a.nwork = c->nwork; a.cases = c->dcase;
  for (int l = 0; l < 3; l++) a.buf[l] = c->buf[l];
  a.lam = c->dlam;
  a.heun = heun;
  if (heun == 0) { a.sel_in = SEL_CUR; a.sel_d0 = SEL_CUR; a.sel_out = SEL_TMP; }
  else { a.sel_in = SEL_TMP; a.sel_d0 = SEL_CUR; a.sel_out = SEL_OTHER; }
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(launch_stage(c->prm.limiter, a, c->grid, c->stream));      // warm-up launch
  CK(cudaEventRecord(e0, c->stream));
  for (int r = 0; r < reps; r++) CK(launch_stage(c->prm.limiter, a, c->grid, c->stream));
  CK(cudaEventRecord(e1, c->stream));
  CK(launch_stage_cfl(c->dblk, c->nblk, c->dcase, c->dlam, heun, c->dcfl, c->stream));
  st = wait_stream(c);
  float el = 0.f;
  if (!st) CK(cudaEventElapsedTime(&el, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st) return st;
  *ms = el / reps;
  return MBM_OK;
}

extern "C" int mbm_trace(mbm_ctx* c, double* rec, int cap, int* n) {
  if (!c || (cap > 0 && !rec)) return fail(c, MBM_EINVAL, "mbm_trace: bad argument");
  const int k = std::min(cap, c->hcase->trace_n);
  if (k > 0) {
    CK(cudaSetDevice(c->device));
    CK(cudaMemcpy(rec, c->dtrace, sizeof(double) * 4 * k, cudaMemcpyDeviceToHost));
  }
  if (n) *n = k;
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
    case MBM_ENONFINITE: return "non-finite CFL or time step";
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
