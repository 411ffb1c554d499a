/*
 * mbm_b200.h -- C ABI of the B200 (sm_100a) implementation of MultiBlockMomentsFV's
 * explicit Heun time-stepping path.
 *
 * The reference has no plugin layer: its hot path is the C function
 *     int Steps(DB_Block *B, int bMax, double *t, double tend, double CFLmax, double CFLreg)
 * (src/Main.c:31,189-244) with TimeUpdate (src/Main.c:253-284), Update
 * (src/Main.c:297-396) and SetBoundary (src/Boundary.c:173-193) below it, reading
 * the globals Kn, F (src/Scenario.c:22-23) and Limiter (src/Limiter.c:20).  The
 * entry points below replace those functions one for one; the host keeps its own
 * DB_Block arrays (array of structs, 9 doubles per cell, x fastest, ghosts
 * included) and passes them as plain pointers.
 *
 * Every call returns an int status (MBM_OK = 0).  No exception crosses the ABI.
 * A context is not thread-safe; use one host thread per context.
 */
#ifndef MBM_B200_H
#define MBM_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MBM_OK          0
#define MBM_EINVAL      1   /* bad argument or block table                       */
#define MBM_ENONFINITE  2   /* CFL or dt became non-finite / non-positive         */
#define MBM_ETIMEOUT    3   /* a bounded host wait on the device ran out          */
#define MBM_ECUDA       4   /* a CUDA runtime call failed (see mbm_last_error)   */
#define MBM_ENOMEM      5   /* device allocation failed                          */
#define MBM_ESTEPLIMIT  6   /* step attempts exceeded max_attempts               */
#define MBM_ENODEV      7   /* no CUDA device                                    */

/* layers, as the reference's layer enum (src/defs.h:21-24) */
#define MBM_L_DATA 0
#define MBM_L_TMP  1
#define MBM_L_NEW  2

/* limiters, as src/Limiter.h:9-15 */
#define MBM_LIM_NONE     0
#define MBM_LIM_AVERAGE  1
#define MBM_LIM_MINMOD   2
#define MBM_LIM_SUPERBEE 3
#define MBM_LIM_HARMONIC 4

/* arithmetic modes */
#define MBM_MODE_EXACT 0   /* operation-for-operation the reference: bitwise-equal results */
#define MBM_MODE_FAST  1   /* multiply-add contraction and reciprocal-multiply quotients in the
                              stage kernel: within 1e-10 relative per field of the reference
                              after one step and 1e-8 at the end time (not bitwise) */

/* One block: the DB_Block fields the path reads (src/defs.h:59-68). */
typedef struct {
  int nx, ny;          /* interior cells; the block holds (nx+6)*(ny+6) cells       */
  double x0, y0;       /* centre of padded cell (0,0): B.x, B.y (src/Mesh.c:364-365) */
  double dx, dy;       /* cell sizes, in (1e-100, 1e100)                           */
  int bc[4];           /* left, right, bottom, top: >0 sync with block code,
                          0 open, -1 wall, -2 Dirichlet (src/defs.h:26-31)          */
} mbm_block_desc;

typedef struct {
  double Kn;           /* Knudsen number (collision frequency rho*sqrt(theta)/Kn), in (1e-100, 1e100) */
  double F;            /* body force in x                                          */
  int limiter;         /* MBM_LIM_*                                                */
  int mode;            /* MBM_MODE_*                                               */
  int device;          /* CUDA device ordinal                                      */
  int show_every;      /* progress record every n accepted steps (reference: 20); 0 = none */
  int max_attempts;    /* bound on step attempts per mbm_steps call; 0 = 10,000,000 */
  int segment_rows;    /* rows per warp work item; 0 = tuned default               */
  void *stream;        /* cudaStream_t to launch on; NULL = a stream the context owns */
  int adjoint;         /* 1: the step loop records dt and checkpoints for mbm_adjoint_run */
} mbm_params;

/* One independent case of a batch: a contiguous run of blocks of the block array,
 * with its own physics parameters.  Sync codes of its blocks count from 1 within
 * the case. */
typedef struct {
  int first_block;
  int nblocks;
  double Kn, F;
  int limiter;
} mbm_case_desc;

typedef struct mbm_ctx mbm_ctx;

/* Allocate device state for a block table.  Replaces the allocation in main()
 * (src/Main.c:113-123).  Sync partners must have equal tangential extents
 * (src/Boundary.c:101-103) and codes must name existing blocks. */
int mbm_create(const mbm_block_desc *blocks, int nblocks, const mbm_params *params, mbm_ctx **ctx);
int mbm_destroy(mbm_ctx *ctx);

/* Many independent cases in one context (no counterpart in the reference, which
 * runs one case per process): every Heun stage of every case is one persistent
 * launch per limiter in use, and mbm_steps_batch advances all cases together in
 * one CUDA-graph loop, each with its own dt, t and step count.  Blocks are indexed
 * globally in the transfer calls. */
int mbm_create_batch(const mbm_block_desc *blocks, int nblocks, const mbm_case_desc *cases,
                     int ncases, const mbm_params *params, mbm_ctx **ctx);
/* t[c], tend[c], nsteps[c], nrej[c] per case; max_steps > 0 caps accepted steps */
int mbm_steps_batch(mbm_ctx *ctx, double *t, const double *tend, double CFLmax, double CFLreg,
                    int max_steps, int *nsteps, int *nrej);
/* The same in two halves, no counterpart in the reference: _async launches the step
 * loop of every case and returns; _wait waits for it and returns t, nsteps, nrej as
 * above.  In between the host may do its own work (write the previous output) and
 * call mbm_output_fields_async/mbm_output_wait; no other call on the context. */
int mbm_steps_batch_async(mbm_ctx *ctx, const double *t, const double *tend, double CFLmax, double CFLreg,
                          int max_steps);
int mbm_steps_batch_wait(mbm_ctx *ctx, double *t, int *nsteps, int *nrej);

/* Copy one block of a layer between the host (array of structs, (nx+6)*(ny+6)*9
 * doubles, the reference's CVector layer, src/defs.h:42-44) and the device. */
int mbm_upload(mbm_ctx *ctx, int layer, int block, const double *cells);
int mbm_download(mbm_ctx *ctx, int layer, int block, double *cells);

/* Output's payload of one block of DATA computed on the device (src/Output.c:195-243):
 * the fields rho vx vy T p Pxx Pxy Pyy qx qy over the interior plus one ghost ring,
 * x outer, y inner, variables fastest; (nx+2)*(ny+2)*10 floats (single = 1) or
 * doubles, the bytes the reference writes to its .dat file. */
int mbm_output_fields(mbm_ctx *ctx, int block, int single, void *out);

/* LoadData (src/Mesh.c:198-283) for one block, on the device: `payload` (host) is the
 * block's zone of a result file as stored -- (nx+2)*(ny+2) points of the interior plus
 * one ghost ring, x outer / y inner, the 10 fields rho vx vy T p Pxx Pxy Pyy qx qy
 * fastest, float (single = 1) or double -- and becomes the moments of L_DATA; every other
 * cell of the block becomes zero, as in the reference's main before its SetBoundary
 * (call mbm_set_boundary next).  faithful = 0 keeps the reference's mapping (the stored
 * p goes where theta belongs, P_ij where T_ij belongs), bit for bit; faithful = 1 maps
 * the fields to the state they were written from (theta = T, T_ij = P_ij / rho).  Only
 * the payload crosses to the device. */
int mbm_load_fields(mbm_ctx *ctx, int block, int single, const void *payload, int faithful);

/* The same payload formed now (from DATA as it is) into device memory the context
 * keeps per block, and copied to `host` (page-locked, e.g. from mbm_host_alloc) on a
 * stream of its own, so that the copy runs beside the next step loop; mbm_output_wait
 * returns once every such copy has landed.  No counterpart in the reference, whose
 * Output runs between intervals. */
int mbm_output_fields_async(mbm_ctx *ctx, int block, int single, void *host);
int mbm_output_wait(mbm_ctx *ctx);

/* Page-locked host memory for mbm_output_fields_async (cudaMallocHost / cudaFreeHost). */
int mbm_host_alloc(size_t bytes, void **p);
int mbm_host_free(void *p);

/* Dirichlet ghost values of one edge (code -2), in FillEdge's order: tangential
 * index over the full edge, corners included, outer; ghost layer n = 1..3 inner
 * (src/Boundary.c:105-129); 9 doubles each.  The host evaluates its SetInitial
 * at each ghost centre (src/Boundary.c:127-129); the values hold until set again. */
int mbm_set_dirichlet(mbm_ctx *ctx, int block, int side, const double *values);

/* SetBoundary (src/Boundary.c:173-193) on one layer. */
int mbm_set_boundary(mbm_ctx *ctx, int layer, double t);

/* Update (src/Main.c:297-396) of every block: out_layer <- stage(in_layer),
 * Data0 = data0_layer, Heun flag heun; cfl[b] receives each block's return value
 * (may be NULL). */
int mbm_update(mbm_ctx *ctx, int out_layer, int in_layer, int data0_layer, double dt, double t,
               int heun, double *cfl);

/* TimeUpdate (src/Main.c:253-284): both Heun stages with a boundary fill after
 * each; *cfl receives max over stages and blocks. */
int mbm_time_update(mbm_ctx *ctx, double dt, double t, double *cfl);

/* Steps (src/Main.c:189-244): advance DATA from *t to tend with the a-posteriori
 * CFL control (reject if CFL > CFLmax, next dt = dt*CFLreg/CFL, dt restarts at
 * 1e-4 on every call).  The step loop runs on the device (a CUDA graph with a
 * conditional while node); the host waits once.  *nsteps = accepted steps,
 * *nrej = rejected attempts (either may be NULL). */
int mbm_steps(mbm_ctx *ctx, double *t, double tend, double CFLmax, double CFLreg, int *nsteps,
              int *nrej);

/* mbm_steps with a cap on accepted steps (max_steps > 0); the loop also ends at
 * tend.  Used for fixed-length runs (benchmarks, the many-case workloads). */
int mbm_steps_capped(mbm_ctx *ctx, double *t, double tend, double CFLmax, double CFLreg,
                     int max_steps, int *nsteps, int *nrej);

/* Device time of the stage kernel alone: `reps` launches of Heun stage `heun` on
 * the current layers (TMP <- DATA, or NEW <- TMP with Data0 = DATA) at step dt,
 * bracketed by CUDA events on the context's stream.  *ms = mean per launch. */
int mbm_time_stage(mbm_ctx *ctx, int heun, double dt, int reps, double *ms);

/* Progress records of the last mbm_steps call, one per show_every accepted steps:
 * {step, CFL, t, next dt}, the values the reference prints (src/Main.c:218-230). */
int mbm_trace(mbm_ctx *ctx, double *records, int cap, int *n);
/* the same for case c of a batch */
int mbm_trace_case(mbm_ctx *ctx, int c, double *records, int cap, int *n);

/* Step attempts (accepted + rejected) of the last mbm_steps call; each attempt
 * runs five kernels (two stages, two ghost fills, the controller). */
int mbm_attempts(mbm_ctx *ctx, int *attempts);

/* Status of each of the first n cases after the last step-loop call: MBM_OK, or
 * MBM_ENONFINITE (the case stopped at the attempt that produced a NaN or infinity;
 * its state is the last accepted one) or MBM_ESTEPLIMIT.  The call itself returned
 * the worst of them; the other cases ran to the end.  No counterpart in the
 * reference, whose loop runs on through non-finite values. */
int mbm_case_status(mbm_ctx *ctx, int *status, int n);

/* Diagnostic, no counterpart in the reference: the fast-arithmetic reciprocal and
 * square root (MBM_MODE_FAST) of n values in device memory x; out (device, 2n
 * doubles) receives 1/x and sqrt(x) interleaved, for comparison with correctly
 * rounded results.  Normal positive operands. */
int mbm_fastmath_check(const double *x, int n, double *out);

/* ---- One case split over ranks by block (one process per GPU) ----------------
 * No counterpart in the reference, which runs every block in one process.  Each
 * rank owns whole blocks (owner[b] = rank of block b, the same table on every
 * rank).  A ghost cell whose source cell is on another rank is filled from a
 * receive buffer; the caller moves the send buffers' segments to the peers'
 * receive buffers (e.g. NCCL send/recv) between mbm_shard_pack and mbm_shard_fill,
 * ordered after the pack on the context's stream, and replaces the CFL scalar by
 * its maximum over the ranks between mbm_shard_cfl and mbm_shard_control.  The
 * Steps loop of one call, every rank in lockstep:
 *   mbm_shard_begin; while (!done) { stage(0); pack(TMP); exchange; fill(TMP);
 *   stage(1); pack(NEW); exchange; fill(NEW); cfl; max-reduce; control(&done) }
 *   mbm_shard_end.
 * Results equal the unsplit context's bit for bit (same map, same arithmetic;
 * the maximum is order-free).  The initial ghost fill is pack(DATA), exchange,
 * fill(DATA).  The single-context calls (mbm_steps, mbm_update, mbm_set_boundary,
 * mbm_time_update, the adjoint) refuse a sharded context. */

/* The exchange plan of one rank, on the host (no device needed): cells sent to and
 * received from each rank (send_counts, recv_counts: nranks entries each); up to
 * cap entries of send_cells (global block, cell J*(nx+6)+I) and recv_cells (global
 * destination block, destination cell, wall flips: 1 = x, 2 = y), peers in rank
 * order. */
int mbm_shard_plan(const mbm_block_desc *blocks, int nblocks, const int *owner, int nranks, int rank,
                   int *send_counts, int *recv_counts, int *send_cells, int *recv_cells, int cap);

/* A context holding the blocks of `rank` (numbered in their global order). */
int mbm_create_sharded(const mbm_block_desc *blocks, int nblocks, const int *owner, int nranks, int rank,
                       const mbm_params *params, mbm_ctx **ctx);

/* Cells per peer and the device buffers: send and receive (9 doubles per cell,
 * peers in rank order) and the CFL scalar (1 double). */
int mbm_shard_buffers(mbm_ctx *ctx, int *send_counts, int *recv_counts, int nranks, double **send,
                      double **recv, double **cfl);

/* Dirichlet ghost values (as mbm_set_dirichlet) of edge `side` of global block
 * `block`: every rank sets those of all blocks, since a corner ghost cell can take
 * its value from another rank's Dirichlet edge. */
int mbm_shard_set_dirichlet(mbm_ctx *ctx, int block, int side, const double *values);

int mbm_shard_begin(mbm_ctx *ctx, double t, double tend, double CFLmax, double CFLreg, int max_steps);
int mbm_shard_stage(mbm_ctx *ctx, int heun);          /* Heun stage 1 (DATA -> TMP) or 2 (-> NEW) */
int mbm_shard_pack(mbm_ctx *ctx, int layer);          /* this rank's cells other ranks need */
int mbm_shard_fill(mbm_ctx *ctx, int layer);          /* SetBoundary of the layer, remote cells received */
int mbm_shard_cfl(mbm_ctx *ctx);                      /* this rank's CFL of the attempt -> the scalar */
/* accept/reject with the scalar.  done non-NULL: waits for the stream and reports
 * whether the step loop has finished; NULL: enqueues the controller and returns at
 * once -- the stage, fill and controller kernels of a finished case return at once,
 * so a caller may enqueue several attempts (every rank the same number) and read
 * `done` once per batch. */
int mbm_shard_control(mbm_ctx *ctx, int *done);
int mbm_shard_end(mbm_ctx *ctx, double *t, int *nsteps, int *nrej);

/* No counterpart in the reference.  *on = 1 when the fast stage kernel's second Heun
 * stage fills its shared-memory rows by bulk tensor copies (TMA: 3-D tensor maps over
 * the context's TMP and relaxation layers, one copy of 32 columns x 9 moment planes per
 * row, completion on mbarriers with bounded waits; a wait that runs out stops the case
 * with MBM_ETIMEOUT); 0 when it uses per-lane asynchronous copies, the default (the
 * environment variable MBM_TMA=1 at context creation selects the bulk copies, which
 * measured slower on this kernel; bitwise mode and a driver without the tensor-map
 * encoder always use the per-lane copies; the reason is then in mbm_last_error). */
int mbm_bulk_copies(mbm_ctx *ctx, int *on);

/* Launch configuration in use, of Heun stage 1: rows per warp work item (picked by
 * the autotuner when mbm_params.segment_rows is 0; the tuner's length may be
 * fractional -- a strip of n face rows gets ceil(n / length) equal segments -- and is
 * reported rounded), work items, CTAs of the persistent stage grid. */
int mbm_config(mbm_ctx *ctx, int *segment_rows, int *work_items, int *ctas);

/* The same for either Heun stage (heun 0 or 1; each has its own work table, the
 * tuner picking each stage's length), the length unrounded.  No counterpart in the
 * reference. */
int mbm_config_stage(mbm_ctx *ctx, int heun, double *segment_rows, int *work_items, int *ctas);

/* *on = 1 when the step loop's ghost fills (SetBoundary after each stage,
 * src/Boundary.c:173-193) are done inside the stage kernels, each work item writing the
 * ghost cells whose source cells it stored (for a Dirichlet ghost: whose nearest
 * interior cell it stored) -- opt-in, MBM_GHOST_SCATTER=1 at context creation; 0 when a
 * separate gather launch fills them (the default; always in sharded contexts).  Both
 * give the same layers bit for bit. */
int mbm_ghost_scatter(mbm_ctx *ctx, int *on);

/* *on = 1 when the step loop's kernels (stages, ghost fills, controller) are launched
 * with programmatic dependent launch: each may be scheduled while the one before it
 * finishes and waits on the device for its results, which takes the launch gaps out
 * of the step.  Off with MBM_PDL=0 at context creation, when a stage runs as several
 * limiter groups on forked streams, and when the step graph cannot be built with it.
 * No counterpart in the reference. */
int mbm_dependent_launch(mbm_ctx *ctx, int *on);

/* Host-only: the resolved ghost-cell sources of a block table, 4 ints per ghost
 * cell {dst_block, dst_cell, src, src_block | flags<<16}; cells are J*(nx+6)+I,
 * src < 0 is Dirichlet row -(src+1), flags bit 0/1 = x/y wall sign.  Needs no GPU. */
int mbm_ghost_map(const mbm_block_desc *blocks, int nblocks, int *entries, int cap, int *n);

/* One Heun stage -- Update (src/Main.c:297-396) of every block -- on device buffers
 * the caller owns, allocating no device memory: no cudaMalloc, cudaFree or
 * allocating library routine is called.  No counterpart in the reference (its
 * Update allocates nothing on a GPU because it has none); it exists for callers
 * that cannot allocate: a framework whose memory pool owns the GPU, real-time
 * loops that fix every allocation at start-up.
 *
 * in, data0 and out are device arrays in this library's plane layout: blocks one
 * after another; block b has 9 planes (one per moment) of (ny+6) rows x pitch
 * doubles, pitch = ((nx+6) + 1 + 3) & ~3, plane = (pitch*(ny+6) + 31) & ~31
 * elements, moment m of padded cell (I, J) at offset_b + m*plane + J*pitch + I + 1,
 * offset_0 = 0, offset_{b+1} = offset_b + 9*plane_b.  Stage 1 (heun 0) reads `in`
 * (DATA with filled ghosts); stage 2 (heun 1) reads `in` (TMP) and `data0` (DATA).
 * Interior cells of `out` are written; its ghost cells are left as they are (fill
 * them with SetBoundary semantics before the next stage).  Sync codes are ignored
 * here.  out must share no element with in or data0 (an in-place stage is
 * refused with MBM_EINVAL: the kernel reads neighbours that other warps would have
 * overwritten).  dt must be positive and finite.  cfl[b] (host, may be NULL)
 * receives each block's Update return value.  A stage that writes a NaN or an
 * infinity into out returns MBM_ENONFINITE (out and cfl are still written; a NaN
 * never enters the CFL maxima, so cfl alone does not show it).  Launches on
 * `stream` (a cudaStream_t, NULL = the legacy default stream) and waits for that
 * stream before it returns.
 *
 * Scratch: one file-scope device array of 320 KB (held by every GPU that loads
 * the library until the process exits): at most 64 blocks and 20,064 warp work
 * items (28-column strips x 32-row segments, e.g. 16 blocks of 1024^2); larger
 * inputs return MBM_EINVAL.  Its device address is looked up by the first call on
 * each device, with that device current -- make that first call before any stream
 * capture.  Every call shares the array and clears what must start at zero; calls
 * that overlap on the GPU race.  Errors: mbm_last_error(NULL). */
int mbm_stage_noalloc(const mbm_block_desc *blocks, int nblocks, const double *in,
                      const double *data0, double *out, double Kn, double F, int limiter,
                      double dt, int heun, double *cfl, void *stream);

/* The scalar functional of the final state the adjoint differentiates, summed over
 * interior cells (unweighted): the heat flux q1^2 + q2^2 (the default), the temperature
 * theta, or the deviatoric temperature tensor (T11 - theta)^2 + 2 T12^2 + (T22 - theta)^2.
 * No counterpart in the reference. */
enum { MBM_J_HEAT_FLUX = 0, MBM_J_TEMPERATURE = 1, MBM_J_DEVIATORIC = 2 };
int mbm_set_functional(mbm_ctx *ctx, int kind);

/* Discrete adjoint (no counterpart in the reference): from the current DATA (the
 * initial state u0), run Steps for `nsteps` accepted steps (dt restarts at 1e-4,
 * CFLmax 1, CFLreg as given) recording every dt and a checkpoint every `every`
 * steps; evaluate J (mbm_set_functional; by default the sum over interior cells of
 * qx^2 + qy^2) of the final state;
 * then sweep back through the steps with dt frozen, recomputing each segment from
 * its checkpoint (the last segment's states are kept by the forward run instead;
 * MBM_ADJ_TAIL=0 recomputes it too), through the hand-written reverse of Update (relaxation, HLL
 * fluxes, limiters with one-sided derivatives at kinks) and of SetBoundary.
 * grad (host, may be NULL) receives dJ/du0 in the layer layout of mbm_upload
 * (ghost cells zero), *grad_Kn = dJ/dKn, dts[nsteps] (may be NULL) the frozen dt
 * sequence, ms[0..1] (may be NULL) the forward and the adjoint device times.  *t
 * advances to the forward run's end.  Needs a single-case context created with
 * mbm_params.adjoint = 1.  Device memory it holds after the first call: 8 layers
 * of work space, nsteps/every + 1 checkpoints and two segments of 2*every + 1 layers
 * (the next segment is recomputed beside the reversal of the current one), i.e.
 * about (nsteps/every + 4*every + 11) layers of the context's size. */
int mbm_adjoint_run(mbm_ctx *ctx, double *t, int nsteps, int every, double CFLreg, double *J,
                    double *grad, double *grad_Kn, double *dts, double *ms);

/* Frozen-dt forward: n Heun steps of DATA with the given dt values (no controller,
 * as the adjoint sees the run); *J (may be NULL) = the functional above. */
int mbm_replay(mbm_ctx *ctx, const double *dts, int n, double *J);

/* Kn and body force F of every case (the reference's globals Kn, F). */
int mbm_set_physics(mbm_ctx *ctx, double Kn, double F);

const char *mbm_strerror(int status);
/* last CUDA / validation message of a context (or the last mbm_create failure when ctx is NULL) */
const char *mbm_last_error(mbm_ctx *ctx);
int mbm_version(void);

#ifdef __cplusplus
}
#endif
#endif
