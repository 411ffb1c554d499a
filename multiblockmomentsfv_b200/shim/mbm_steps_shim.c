/*
 * mbm_steps_shim.c -- Steps() for the reference's C host, running on the GPU.
 *
 * The reference calls  int Steps(DB_Block *B, int bMax, double *t, double tend,
 * double CFLmax, double CFLreg)  once per output interval (src/Main.c:149-154) and
 * reads B[nb].layer[L_DATA] in Output afterwards.  This file defines that function
 * on top of the C ABI of include/mbm_b200.h:
 *
 *   first call   create a context from the block table, the globals Kn, F and
 *                Limiter, evaluate the scenario's SetInitial at every Dirichlet
 *                ghost centre (src/Boundary.c:127-129) and upload L_DATA;
 *   every call   mbm_steps on the device (dt restarts at 1e-4 as in the
 *                reference), print the reference's progress lines, download
 *                L_DATA (interior and ghost cells) for Output.
 *
 * It compiles against the reference's headers (DB_Block, src/defs.h:59-68) and is
 * linked in place of the reference's own Steps.  MBM_DEVICE selects the GPU
 * (default 0).  A failing call prints the library's message and exits with
 * status 2: the reference's Steps has no error return.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>

#include "database_range.h"
#include "defs.h"
#include "tools.h"
#include "Scenario.h"
#include "Limiter.h"
#include "mbm_b200.h"

static mbm_ctx *g_ctx;

static void die(int st, const char *what)
{
  fprintf(stderr, "mbm: %s failed: %s (%s)\n", what, mbm_strerror(st), mbm_last_error(g_ctx));
  exit(2);
}

/* ghost cell n = 1..3 of an edge at tangential index ti, global indices (src/Boundary.c:51-62) */
static void ghost_index(const DB_Range *R, int side, int ti, int n, int *i, int *j)
{
  switch (side) {
    case 0: *i = R->lfb.i + MBC - n; *j = ti; break;
    case 1: *i = R->rbt.i - MBC + n; *j = ti; break;
    case 2: *i = ti; *j = R->lfb.j + MBC - n; break;
    default: *i = ti; *j = R->rbt.j - MBC + n; break;
  }
}

static void create(DB_Block *B, int bMax)
{
  mbm_block_desc d[NB];
  mbm_params p;
  int nb, side, st;
  for (nb = 0; nb < bMax; nb++) {
    d[nb].nx = B[nb].range.rbt.i - B[nb].range.lfb.i + 1 - 2 * MBC;
    d[nb].ny = B[nb].range.rbt.j - B[nb].range.lfb.j + 1 - 2 * MBC;
    d[nb].x0 = B[nb].x;
    d[nb].y0 = B[nb].y;
    d[nb].dx = B[nb].dx;
    d[nb].dy = B[nb].dy;
    for (side = 0; side < 4; side++) d[nb].bc[side] = B[nb].boundary[side];
  }
  p.Kn = Kn;
  p.F = F;
  p.limiter = Limiter;
  /* MBM_MODE=fast selects the fast-arithmetic stage kernel (not bitwise) */
  p.mode = (getenv("MBM_MODE") && !strcmp(getenv("MBM_MODE"), "fast")) ? MBM_MODE_FAST : MBM_MODE_EXACT;
  p.device = getenv("MBM_DEVICE") ? atoi(getenv("MBM_DEVICE")) : 0;
  p.show_every = 20;
  p.max_attempts = 0;
  p.segment_rows = 0;
  p.stream = NULL;
  if ((st = mbm_create(d, bMax, &p, &g_ctx))) die(st, "mbm_create");

  for (nb = 0; nb < bMax; nb++)
    for (side = 0; side < 4; side++) {
      if (B[nb].boundary[side] > -2) continue;
      int nt = side < 2 ? B[nb].range.rbt.j - B[nb].range.lfb.j + 1
                        : B[nb].range.rbt.i - B[nb].range.lfb.i + 1;
      int t0 = side < 2 ? B[nb].range.lfb.j : B[nb].range.lfb.i;
      double *v = malloc(sizeof(double) * N * MBC * nt);
      for (int k = 0; k < nt; k++)
        for (int n = 1; n <= MBC; n++) {
          int gi, gj;
          ghost_index(&B[nb].range, side, t0 + k, n, &gi, &gj);
          SetInitial(v + (k * MBC + (n - 1)) * N, GetPoint(gi, gj, 1, B[nb]), 0.0);
        }
      if ((st = mbm_set_dirichlet(g_ctx, nb, side, v))) die(st, "mbm_set_dirichlet");
      free(v);
    }
  for (nb = 0; nb < bMax; nb++)
    if ((st = mbm_upload(g_ctx, MBM_L_DATA, nb, (const double *)B[nb].layer[L_DATA]))) die(st, "mbm_upload");
}

int Steps(DB_Block *B, int bMax, double *t, double tend, double CFLmax, double CFLreg)
{
  int nstep = 0, nrej = 0, st, nb, k, ntr = 0;
  double trace[4 * 512];
  struct timeval a, b;
  if (!g_ctx) create(B, bMax);
  gettimeofday(&a, NULL);
  if ((st = mbm_steps(g_ctx, t, tend, CFLmax, CFLreg, &nstep, &nrej))) die(st, "mbm_steps");
  gettimeofday(&b, NULL);
  double ms = 1e3 * (b.tv_sec - a.tv_sec) + 1e-3 * (b.tv_usec - a.tv_usec);
  double perf = ms / (1.0e-3 * FullGridSize(B, bMax) * (nstep + nrej));
  mbm_trace(g_ctx, trace, 512, &ntr);
  for (k = 0; k < ntr; k++)      /* the reference's progress line (src/Main.c:228-229) */
    printf(" step: %3d... done.  CFL: %lf, time: %lf, next dt: %lf, diff: %lf, perf = %.4f (gpu)\n",
           (int)trace[4 * k], trace[4 * k + 1], trace[4 * k + 2], trace[4 * k + 3], 0.0, perf);
  fflush(stdout);
  for (nb = 0; nb < bMax; nb++)
    if ((st = mbm_download(g_ctx, MBM_L_DATA, nb, (double *)B[nb].layer[L_DATA]))) die(st, "mbm_download");
  return nstep;
}
