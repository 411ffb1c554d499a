/*
 * mbm_oracle.c -- CPU restatement of the MultiBlockMomentsFV explicit Heun path
 * (Steps -> TimeUpdate -> Update / SetBoundary and the Flux.c, Limiter.c and
 * Scenario.c helpers it calls).
 *
 * TEST INFRASTRUCTURE ONLY: the parity checker for the CUDA path.  Nothing in
 * the product package loads or calls this file.
 *
 * Every floating-point expression keeps the operand order and association of
 * the reference expression it restates (cited file:line), because bitwise
 * agreement with the reference depends on it.  Build with -ffp-contract=off so
 * no multiply-add is fused.  The loop structure, data structures and naming are
 * this project's own.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "mbm_oracle.h"

#define NV ORC_NV
#define NG ORC_NG

struct orc_ctx {
  int nb;
  orc_block *blk;
  orc_params prm;
  orc_scenario scn;
  double *layer[3][64];     /* [layer][block] -> (nx+6)*(ny+6)*9 */
  double *aux[64];          /* per block: Prim, dPrimX, dPrimY   (src/defs.h:48-52) */
};

/* ---------------------------------------------------------------- helpers -- */
/* tools.h:3-17: the reference's max/min/sgn (NaN semantics matter: a > b ? a : b) */
static inline double rmax(double a, double b) { return a > b ? a : b; }
static inline double rmin(double a, double b) { return a < b ? a : b; }
static inline double rsgn(double a) { if (a == 0) return 0; return a < 0 ? -1 : 1; }

static inline int pitch(const orc_block *b) { return b->nx + 2 * NG; }
static inline int rows(const orc_block *b) { return b->ny + 2 * NG; }

/* ------------------------------------------------------------- moments ---- */
/* Primitive: U -> {rho, vx, vy, theta, T11, T12, T22, q1, q2}   src/Flux.c:30-56 */
void orc_primitive(const double *U, double *P)
{
  double rho = U[0];
  double v1 = U[1] / rho, v2 = U[2] / rho;
  double vs = v1 * v1 + v2 * v2;
  double th = (2 * U[3] / rho - vs) / 3;
  double E = U[3];
  double T11 = U[4] / rho - v1 * v1;
  double T12 = U[5] / rho - v1 * v2;
  double T22 = U[6] / rho - v2 * v2;
  P[0] = rho; P[1] = v1; P[2] = v2; P[3] = th;
  P[4] = T11; P[5] = T12; P[6] = T22;
  P[7] = U[7] - E * v1 - rho * (T11 * v1 + T12 * v2);
  P[8] = U[8] - E * v2 - rho * (T12 * v1 + T22 * v2);
}

/* moments from primitives with an explicit energy E       src/Flux.c:61-74, 255-263 */
static inline void cons_with_energy(double rho, double v1, double v2, double E,
                                    double T11, double T12, double T22,
                                    double q1, double q2, double *U)
{
  U[0] = rho;
  U[1] = rho * v1;
  U[2] = rho * v2;
  U[3] = E;
  U[4] = rho * (T11 + v1 * v1);
  U[5] = rho * (T12 + v1 * v2);
  U[6] = rho * (T22 + v2 * v2);
  U[7] = q1 + E * v1 + rho * (T11 * v1 + T12 * v2);
  U[8] = q2 + E * v2 + rho * (T12 * v1 + T22 * v2);
}

/* Conservative: primitives -> moments, E from primDef.h      src/Flux.c:61-74, src/primDef.h:9-20 */
void orc_conservative(const double *P, double *U)
{
  double rho = P[0], v1 = P[1], v2 = P[2], th = P[3];
  double vs = v1 * v1 + v2 * v2;
  double E = 0.5 * rho * vs + 1.5 * rho * th;
  cons_with_energy(rho, v1, v2, E, P[4], P[5], P[6], P[7], P[8], U);
}

/* Grad-13 flux along x of a moment vector                   src/Flux.c:79-119 */
static void grad13_flux_x(const double *U, double *F)
{
  double rho = U[0];
  double v1 = U[1] / rho, v2 = U[2] / rho;
  double vs = v1 * v1 + v2 * v2;
  double th = (2 * U[3] / rho - vs) / 3;
  double E = U[3];
  double T11 = U[4] / rho - v1 * v1;
  double T12 = U[5] / rho - v1 * v2;
  double T22 = U[6] / rho - v2 * v2;
  double q1 = U[7] - E * v1 - rho * (T11 * v1 + T12 * v2);
  double q2 = U[8] - E * v2 - rho * (T12 * v1 + T22 * v2);
  /* Grad-13 closure */
  double M111 = 1.2 * q1 / rho;
  double M121 = 0.4 * q2 / rho, M112 = M121;
  double M221 = 0.4 * q1 / rho, M122 = M221;
  double R11 = 5 * th * th + 7 * th * (T11 - th);
  double R12 = 7 * th * T12;

  F[0] = rho * v1;
  F[1] = rho * (T11 + v1 * v1);
  F[2] = rho * (T12 + v1 * v2);
  F[3] = E * v1 + rho * (T11 * v1 + T12 * v2) + q1;
  F[4] = rho * (M111 + 3 * T11 * v1 + v1 * v1 * v1);
  F[5] = rho * (M121 + T11 * v2 + 2 * T12 * v1 + v1 * v2 * v1);
  F[6] = rho * (M221 + T22 * v1 + 2 * T12 * v2 + v2 * v2 * v1);
  F[7] = 2 * (q1 + rho * (T11 * v1 + T12 * v2)) * v1 + E * v1 * v1
       + rho * (M111 * v1 + M112 * v2) + 0.5 * rho * (T11 * vs + R11);
  F[8] = q2 * v1 + q1 * v2 + rho * (v1 * v2 * (T11 + T22) + 1.5 * T12 * vs)
       + E * v1 * v2 + rho * (M121 * v1 + M122 * v2) + 0.5 * rho * R12;
}

/* flux through a face with unit normal (nx,ny): rotate, x-flux, rotate back   src/Flux.c:126-172 */
void orc_flux2d(const double *U, double *F, double nx, double ny)
{
  double tx = ny, ty = -nx, a, b;
  double W[NV], G[NV];
  W[0] = U[0];
  W[1] = U[1] * nx + U[2] * ny;
  W[2] = U[1] * tx + U[2] * ty;
  W[3] = U[3];
  a = U[4] * nx + U[5] * ny;
  b = U[5] * nx + U[6] * ny;
  W[4] = a * nx + b * ny;
  W[5] = a * tx + b * ty;
  a = U[4] * tx + U[5] * ty;
  b = U[5] * tx + U[6] * ty;
  W[6] = a * tx + b * ty;
  W[7] = U[7] * nx + U[8] * ny;
  W[8] = U[7] * tx + U[8] * ty;

  grad13_flux_x(W, G);

  F[0] = G[0];
  F[1] = G[1] * nx + G[2] * tx;
  F[2] = G[1] * ny + G[2] * ty;
  F[3] = G[3];
  a = G[4] * nx + G[5] * tx;
  b = G[5] * nx + G[6] * tx;
  F[4] = a * nx + b * tx;
  F[5] = a * ny + b * ty;
  a = G[4] * ny + G[5] * ty;
  b = G[5] * ny + G[6] * ty;
  F[6] = a * ny + b * ty;
  F[7] = G[7] * nx + G[8] * tx;
  F[8] = G[7] * ny + G[8] * ty;
}

/* ------------------------------------------------------------ relaxation -- */
/* damping factor of the direct production integration        src/Flux.c:213-223 */
static inline double rdamp(double z, int flag)
{
  switch (flag) {
    case -1:
    case 0: return (1 + 0.5 * z - 0.25 * z * z) / (1 + z + 0.25 * z * z);
    case 1: return (1 + z) / (1 + z + 0.25 * z * z);
    case 2: return (1 + 0.5 * z) / (1 + 0.5 * z);
    case 3: return 1.0 / (1 + 0.5 * z);
  }
  return 0.0;
}

/* ProductionsDirect (src/Flux.c:230-267) with CollFreq and ExternalForce of
 * src/Scenario.c:28-42 (nu0 = 1, force (F, 0)).  Returns 0.5*(1 - R(2z/3)). */
double orc_relax(const orc_params *p, const double *U, double *Out, double dt, int flag)
{
  double P[NV];
  orc_primitive(U, P);
  double rho = P[0], v1 = P[1], v2 = P[2], th = P[3];
  double T11 = P[4], T12 = P[5], T22 = P[6], q1 = P[7], q2 = P[8];
  double vs = v1 * v1 + v2 * v2;
  double E = 0.5 * rho * vs + 1.5 * rho * th;
  double nu0 = 1.0;
  double coll = (nu0 * rho * sqrt(th) / p->Kn) * dt;

  if (flag == 0 || flag == 2) {
    double g0 = p->F, g1 = 0.0;
    v1 += dt * g0;
    v2 += dt * g1;
    vs = v1 * v1 + v2 * v2;
    E = 0.5 * rho * vs + 1.5 * rho * th;
  }
  double d1 = rdamp(coll, flag);
  double d2 = rdamp(2.0 / 3 * coll, flag);
  T11 = d1 * (T11 - th) + th;
  T12 = d1 * T12;
  T22 = d1 * (T22 - th) + th;
  q1 = d2 * q1;
  q2 = d2 * q2;
  cons_with_energy(rho, v1, v2, E, T11, T12, T22, q1, q2, Out);
  return 0.5 * (1 - d2);
}

/* --------------------------------------------------------------- limiter -- */
/* Limit1 and its minmod / superbee helpers                   src/Limiter.c:22-59 */
static inline double superbee_phi(double r)
{
  if (r < 0.0) return 0.0;
  if (r < 0.5) return 2 * r;
  if (r < 1.0) return 1.0;
  if (r < 2.0) return r;
  return 2.0;
}

double orc_limit(int limiter, double d1, double d2)
{
  const double eps = 1.0e-10;
  double w1, w2;
  switch (limiter) {
    case ORC_LIM_NONE: return 0.0;
    case ORC_LIM_AVERAGE: return 0.5 * (d1 + d2);
    case ORC_LIM_MINMOD: return 0.5 * (rsgn(d1) + rsgn(d2)) * rmin(fabs(d1), fabs(d2));
    case ORC_LIM_SUPERBEE: return d1 * superbee_phi(d2 / d1);
    default:
      w1 = fabs(d1) + eps;
      w2 = fabs(d2) + eps;
      return (w1 * d2 + w2 * d1) / (w1 + w2);
  }
}

/* ------------------------------------------------------------------- HLL -- */
/* FnumHLLE with MaxSound1 and lamDiff                        src/Flux.c:308-379
 * dir 1 = x face, 2 = y face, dx the cell width normal to the face.  The
 * diffusive scales FFlux/GFlux return are 0, so lamDiff always sees 0 (or NaN)
 * and returns 1.  Returns the face signal speed cMax. */
static inline double sound_speed(const double *P) { return 2.0 * sqrt(5.0 / 3 * P[3]); }

static inline double lam_diff(double kaps)                    /* src/Flux.c:318-325 */
{
  if (kaps > 4.1422533434191076) return (10 + 4 * (kaps + sqrt(6 + 4 * kaps))) / ((1 + 2 * kaps) * (1 + 2 * kaps));
  if (kaps > 1) return 1.15 - 0.15 * kaps;
  return 1.0;
}

double orc_hll(const double *PL, const double *PR, double *flx, int dir, double dx)
{
  double UL[NV], UR[NV], fL[NV], fR[NV];
  double cR = sound_speed(PR), cL = sound_speed(PL);
  double vR, vL;
  double nx = dir == 1 ? 1.0 : 0.0, ny = dir == 1 ? 0.0 : 1.0;
  /* FFlux / GFlux: Conservative then Grad13Flux2D; their diffusive scale is 0 */
  orc_conservative(PL, UL);
  orc_flux2d(UL, fL, nx, ny);
  orc_conservative(PR, UR);
  orc_flux2d(UR, fR, nx, ny);
  double sL = 0.0, sR = 0.0;
  vR = PR[dir]; vL = PL[dir];

  double cMax = fabs(0.5 * (vL + vR)) + rmax(cR, cL);
  cMax = cMax / lam_diff(rmax(sL, sR) / (cMax * dx));

  double lamL = rmin(vL - cL, 0.0);
  double lamR = rmax(vR + cR, 0.0);
  double alph = lamR - lamL;
  /* FnumHLLE recomputes Conservative(PrimL/PrimR) into UL/UR; the values are identical */
  if (alph > 0.0)
    for (int n = 0; n < NV; n++)
      flx[n] = (lamR * fL[n] - lamL * fR[n] + lamL * lamR * (UR[n] - UL[n])) / alph;
  else
    for (int n = 0; n < NV; n++)
      flx[n] = 0.5 * (fL[n] + fR[n]);
  return cMax;
}

/* --------------------------------------------------------------- scenario - */
/* SetInitial restatement (src/Scenario.c:72-153): Riemann2D (golden cases),
 * ForwardFacingStep, and the seeded quadrant / uniform states of the
 * benchmark workloads.  Returns the moment vector of {rho, v, theta},
 * T_ij = theta delta_ij, q = 0. */
void orc_initial_state(const orc_scenario *s, double x, double y, double t, double *U)
{
  (void)t;
  double rho, v1, v2, th, T11, T12, T22, q1, q2, vs, E;
  v1 = 0.0; v2 = 0.0; T12 = 0.0; q1 = 0.0; q2 = 0.0; th = 1.0; rho = 1.0;
  switch (s->kind) {
    case ORC_SCN_RIEMANN2D:
      rho = (sqrt(x * x + y * y) < 0.4) ? 5.0 : 1.0;
      break;
    case ORC_SCN_FFS:
      rho = 1.0;
      v1 = 2.0 * sqrt(5.0 / 3.0);
      break;
    case ORC_SCN_QUADRANT:
    case ORC_SCN_UNIFORM: {
      int k = s->kind == ORC_SCN_UNIFORM ? 0 : (x >= 0.0) + 2 * (y >= 0.0);
      rho = s->q[k][0]; v1 = s->q[k][1]; v2 = s->q[k][2]; th = s->q[k][3];
      break;
    }
  }
  T11 = th;
  T22 = th;
  vs = v1 * v1 + v2 * v2;
  E = 0.5 * rho * vs + 1.5 * rho * th;
  cons_with_energy(rho, v1, v2, E, T11, T12, T22, q1, q2, U);
}

/* ------------------------------------------------------------- context ---- */
orc_ctx *orc_create(const orc_block *blocks, int nblocks, const orc_params *p,
                    const orc_scenario *s)
{
  if (nblocks < 1 || nblocks > 64) return NULL;
  orc_ctx *c = (orc_ctx *)calloc(1, sizeof(orc_ctx));
  c->nb = nblocks;
  c->blk = (orc_block *)malloc(sizeof(orc_block) * nblocks);
  memcpy(c->blk, blocks, sizeof(orc_block) * nblocks);
  c->prm = *p;
  c->scn = *s;
  for (int b = 0; b < nblocks; b++) {
    size_t n = (size_t)pitch(&blocks[b]) * rows(&blocks[b]);
    for (int l = 0; l < 3; l++) c->layer[l][b] = (double *)calloc(n * NV, sizeof(double));
    c->aux[b] = (double *)calloc(n * 3 * NV, sizeof(double));
  }
  return c;
}

void orc_destroy(orc_ctx *c)
{
  if (!c) return;
  for (int b = 0; b < c->nb; b++) {
    for (int l = 0; l < 3; l++) free(c->layer[l][b]);
    free(c->aux[b]);
  }
  free(c->blk);
  free(c);
}

void orc_set_params(orc_ctx *c, const orc_params *p) { c->prm = *p; }

void orc_set_layer(orc_ctx *c, int layer, int b, const double *cells)
{
  size_t n = (size_t)pitch(&c->blk[b]) * rows(&c->blk[b]) * NV;
  memcpy(c->layer[layer][b], cells, n * sizeof(double));
}

void orc_get_layer(const orc_ctx *c, int layer, int b, double *cells)
{
  size_t n = (size_t)pitch(&c->blk[b]) * rows(&c->blk[b]) * NV;
  memcpy(cells, c->layer[layer][b], n * sizeof(double));
}

/* ------------------------------------------------------------ boundary ---- */
/* ghost / interior cell of an edge in local indices            src/Boundary.c:51-81 */
static inline void ghost_cell(const orc_block *b, int side, int ti, int n, int *I, int *J)
{
  switch (side) {
    case 0: *I = NG - n; *J = ti; break;
    case 1: *I = pitch(b) - 1 - NG + n; *J = ti; break;
    case 2: *I = ti; *J = NG - n; break;
    default: *I = ti; *J = rows(b) - 1 - NG + n; break;
  }
}

static inline void inner_cell(const orc_block *b, int side, int ti, int s, int *I, int *J)
{
  switch (side) {
    case 0: *I = NG - 1 + s; *J = ti; break;
    case 1: *I = pitch(b) - NG - s; *J = ti; break;
    case 2: *I = ti; *J = NG - 1 + s; break;
    default: *I = ti; *J = rows(b) - NG - s; break;
  }
}

/* specular-wall sign table                                   src/Scenario.c:57-63 */
static const double wall_sign[4][NV] = {
  { +1, -1, +1, +1, +1, -1, +1, -1, +1 },
  { +1, -1, +1, +1, +1, -1, +1, -1, +1 },
  { +1, +1, -1, +1, +1, -1, +1, +1, -1 },
  { +1, +1, -1, +1, +1, -1, +1, +1, -1 },
};

enum { K_SYNC, K_OPEN, K_WALL, K_DIRICHLET };
static inline int kind_of(int code)                          /* src/Boundary.c:137-143 */
{
  if (code > 0) return K_SYNC;
  if (code == 0) return K_OPEN;
  if (code == -1) return K_WALL;
  return K_DIRICHLET;
}

/* FillEdge (src/Boundary.c:88-132): the NG ghost layers of one edge, full tangential
 * range, tangential index outer, layer inner. */
static void fill_edge(orc_ctx *c, int d, int s, int layer, int side, int kind, double t)
{
  const orc_block *D = &c->blk[d], *S = &c->blk[s];
  double *dst = c->layer[layer][d];
  const double *src = c->layer[layer][s];
  int nt = side < 2 ? rows(D) : pitch(D);
  static const int opposite[4] = { 1, 0, 3, 2 };
  for (int ti = 0; ti < nt; ti++)
    for (int n = 1; n <= NG; n++) {
      int gi, gj, si, sj;
      ghost_cell(D, side, ti, n, &gi, &gj);
      double *g = dst + ((size_t)gj * pitch(D) + gi) * NV;
      if (kind == K_SYNC) {
        inner_cell(S, opposite[side], ti, n, &si, &sj);
        memcpy(g, src + ((size_t)sj * pitch(S) + si) * NV, NV * sizeof(double));
      } else if (kind == K_OPEN) {
        inner_cell(D, side, ti, 1, &si, &sj);
        memcpy(g, dst + ((size_t)sj * pitch(D) + si) * NV, NV * sizeof(double));
      } else if (kind == K_WALL) {
        inner_cell(D, side, ti, n, &si, &sj);
        const double *q = dst + ((size_t)sj * pitch(D) + si) * NV;
        for (int m = 0; m < NV; m++) g[m] = wall_sign[side][m] * q[m];
      } else {
        double x = D->x0 + gi * D->dx, y = D->y0 + gj * D->dy;   /* GetPoint, src/tools.c:97-104 */
        orc_initial_state(&c->scn, x, y, t, g);
      }
    }
}

/* SetBoundary: sweep 1 every edge by its kind, sweep 2 sync edges again (src/Boundary.c:173-193) */
void orc_set_boundary(orc_ctx *c, int layer, double t)
{
  for (int b = 0; b < c->nb; b++)
    for (int side = 0; side < 4; side++) {
      int code = c->blk[b].bc[side], k = kind_of(code);
      fill_edge(c, b, k == K_SYNC ? code - 1 : b, layer, side, k, t);
    }
  for (int b = 0; b < c->nb; b++)
    for (int side = 0; side < 4; side++) {
      int code = c->blk[b].bc[side];
      if (code > 0) fill_edge(c, b, code - 1, layer, side, K_SYNC, t);
    }
}

/* main(): SetInitial on interior cells, zero elsewhere, then SetBoundary (src/Main.c:113-138) */
void orc_initialise(orc_ctx *c)
{
  for (int b = 0; b < c->nb; b++) {
    const orc_block *B = &c->blk[b];
    double *d = c->layer[ORC_DATA][b];
    memset(d, 0, (size_t)pitch(B) * rows(B) * NV * sizeof(double));
    for (int I = NG; I < pitch(B) - NG; I++)
      for (int J = NG; J < rows(B) - NG; J++)
        orc_initial_state(&c->scn, B->x0 + I * B->dx, B->y0 + J * B->dy, 0.0,
                          d + ((size_t)J * pitch(B) + I) * NV);
  }
  orc_set_boundary(c, ORC_DATA, 0.0);
}

/* --------------------------------------------------------------- stage ---- */
/* Update (src/Main.c:297-396): one Heun stage of one block.  Returns
 * dt*max(lambda_x)/dx + dt*max(lambda_y)/dy + max(CFL_prod). */
double orc_update(orc_ctx *c, int b, int out_layer, int in_layer, int data0_layer,
                  double dt, double t, int heun)
{
  (void)t;   /* ExternalForce ignores position and time (src/Scenario.c:36-42) */
  const orc_block *B = &c->blk[b];
  const int nxp = pitch(B), nyp = rows(B);
  double *New = c->layer[out_layer][b];
  const double *Dat = c->layer[in_layer][b];
  const double *Dat0 = c->layer[data0_layer][b];
  double *aux = c->aux[b];
  double cfl_x = 0, cfl_y = 0, cfl_prod = 0;
  double dtdx = dt / B->dx, dtdy = dt / B->dy;
#define CELL(I, J) ((size_t)(J) * nxp + (I))
#define PRIM(k) (aux + (k) * 3 * NV)
#define DPX(k) (aux + (k) * 3 * NV + NV)
#define DPY(k) (aux + (k) * 3 * NV + 2 * NV)

  /* 1: primitives of every cell, outermost ring included       src/Main.c:314-318 */
  for (int I = 0; I < nxp; I++)
    for (int J = 0; J < nyp; J++)
      orc_primitive(Dat + CELL(I, J) * NV, PRIM(CELL(I, J)));

  /* 2: relaxation and projected primitives                     src/Main.c:320-336 */
  for (int I = 1; I <= nxp - 2; I++)
    for (int J = 1; J <= nyp - 2; J++) {
      size_t k = CELL(I, J);
      double U0[NV];
      orc_relax(&c->prm, Dat + k * NV, U0, dt, 2 * heun + 1);
      orc_primitive(U0, PRIM(k));
      cfl_prod = rmax(cfl_prod, orc_relax(&c->prm, Dat + k * NV, New + k * NV, dt, 2 * heun));
      if (heun == 1) {
        orc_relax(&c->prm, Dat0 + k * NV, U0, dt, -1);
        for (int n = 0; n < NV; n++) New[k * NV + n] += U0[n];
      }
      for (int n = 0; n < NV; n++) { DPX(k)[n] = 0.0; DPY(k)[n] = 0.0; }
    }

  /* 3: limited slopes                                          src/Main.c:338-351 */
  for (int I = 1; I <= nxp - 2; I++)
    for (int J = 1; J <= nyp - 2; J++) {
      size_t k = CELL(I, J);
      for (int n = 0; n < NV; n++) {
        DPX(k)[n] = orc_limit(c->prm.limiter, PRIM(k)[n] - PRIM(k - 1)[n],
                              PRIM(k + 1)[n] - PRIM(k)[n]) / B->dx;
        DPY(k)[n] = orc_limit(c->prm.limiter, PRIM(k)[n] - PRIM(k - nxp)[n],
                              PRIM(k + nxp)[n] - PRIM(k)[n]) / B->dy;
      }
    }

  /* 4: faces, x index outer, y index inner; y face first      src/Main.c:353-384 */
  for (int I = 1; I <= nxp - 3; I++)
    for (int J = 1; J <= nyp - 3; J++) {
      size_t k = CELL(I, J), kx = k + 1, ky = k + nxp;
      double lo[NV], hi[NV], G[NV], Fx[NV], lam;
      for (int n = 0; n < NV; n++) {
        lo[n] = PRIM(k)[n] + 0.5 * B->dy * DPY(k)[n];
        hi[n] = PRIM(ky)[n] - 0.5 * B->dy * DPY(ky)[n];
      }
      lam = orc_hll(lo, hi, G, 2, B->dy);
      cfl_y = rmax(lam, cfl_y);
      for (int n = 0; n < NV; n++) {
        New[k * NV + n] -= dtdy * G[n];
        New[ky * NV + n] += dtdy * G[n];
      }
      for (int n = 0; n < NV; n++) {
        lo[n] = PRIM(k)[n] + 0.5 * B->dx * DPX(k)[n];
        hi[n] = PRIM(kx)[n] - 0.5 * B->dx * DPX(kx)[n];
      }
      lam = orc_hll(lo, hi, Fx, 1, B->dx);
      cfl_x = rmax(lam, cfl_x);
      for (int n = 0; n < NV; n++) {
        New[k * NV + n] -= dtdx * Fx[n];
        New[kx * NV + n] += dtdx * Fx[n];
      }
    }

  /* 5: Heun average                                            src/Main.c:390-393 */
  if (heun == 1)
    for (size_t k = 0; k < (size_t)nxp * nyp * NV; k++) New[k] = 0.5 * New[k];
#undef CELL
#undef PRIM
#undef DPX
#undef DPY
  return dt * cfl_x / B->dx + dt * cfl_y / B->dy + cfl_prod;
}

/* TimeUpdate: two Heun stages with a boundary fill after each  src/Main.c:253-284 */
double orc_time_update(orc_ctx *c, double dt, double t)
{
  double cfl1 = 0.0, cfl2 = 0.0, cflmax = 0.0;
  for (int b = 0; b < c->nb; b++) {
    double v = orc_update(c, b, ORC_TMP, ORC_DATA, ORC_DATA, dt, t, 0);
    if (v > cfl1) cfl1 = v;
  }
  orc_set_boundary(c, ORC_TMP, t + dt);
  for (int b = 0; b < c->nb; b++) {
    double v = orc_update(c, b, ORC_NEW, ORC_TMP, ORC_DATA, dt, t + dt, 1);
    if (v > cfl2) cfl2 = v;
  }
  orc_set_boundary(c, ORC_NEW, t + dt);
  return rmax(cfl1, rmax(cfl2, cflmax));
}

/* Steps: a-posteriori CFL control with step rejection          src/Main.c:189-244 */
int orc_steps(orc_ctx *c, double *t, double tend, double CFLmax, double CFLreg,
              int max_steps, int *nrej, int show_every,
              double *trace, int trace_cap, int *ntrace)
{
  int nstep = 0, rej = 0, nt = 0;
  long attempts = 0;
  double dt = 0.0001, cfl;
  while (*t < tend) {
    if (max_steps > 0 && nstep >= max_steps) break;
    nstep++;
    do {
      /* the reference loops forever when CFLreg >= CFLmax keeps every retry above
       * CFLmax; the checker gives up after 10^6 attempts instead (returns -1) */
      if (++attempts > 1000000L) { if (nrej) *nrej = rej; if (ntrace) *ntrace = nt; return -1; }
      cfl = orc_time_update(c, dt, *t);
      if (cfl > CFLmax) {
        dt = dt * CFLreg / cfl;
        rej++;
      } else {
        *t += dt;
        dt = dt * CFLreg / cfl;
        if (*t + dt > tend) dt = tend - (*t);
      }
    } while (cfl > CFLmax);
    if (show_every > 0 && !(nstep % show_every) && trace && nt < trace_cap) {
      trace[4 * nt + 0] = nstep;
      trace[4 * nt + 1] = cfl;
      trace[4 * nt + 2] = *t;
      trace[4 * nt + 3] = dt;
      nt++;
    }
    for (int b = 0; b < c->nb; b++) {
      size_t n = (size_t)pitch(&c->blk[b]) * rows(&c->blk[b]) * NV;
      memcpy(c->layer[ORC_DATA][b], c->layer[ORC_NEW][b], n * sizeof(double));
    }
  }
  if (nrej) *nrej = rej;
  if (ntrace) *ntrace = nt;
  return nstep;
}
