/*
 * mbm_oracle.h -- CPU restatement of the MultiBlockMomentsFV explicit Heun path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the CUDA
 * path: tests/, __graft_entry__.smoke() and the cpu_baseline / reference legs of
 * bench.py may load it; the product (multiblockmomentsfv_b200) never does.
 *
 * Parity status: pinned.  The restatement reproduces the reference goldens
 * reference/squareSmall.ref.{hdr,dat} and reference/square4.ref.{hdr,dat}
 * bit-for-bit (tests/test_oracle_golden.py), and agrees bit-for-bit with the
 * reference C sources compiled under oracle/_ref on seeded random inputs
 * (tests/test_oracle_vs_ref.py, run where the reference sources exist).
 *
 * Layout: every block holds three layers (DATA, TMP, NEW) of (nx+6)*(ny+6)
 * cells, 9 doubles per cell (array-of-structs, x fastest), exactly the
 * reference's CVector layer layout (src/defs.h:42-68, src/database_range.c:22-27),
 * with local indices I = i - lfb.i, J = j - lfb.j (lfb = (1,1)).
 */
#ifndef MBM_ORACLE_H
#define MBM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_NV 9      /* moments per cell                      (src/defs.h:11) */
#define ORC_NG 3      /* ghost layers per edge                  (src/defs.h:14) */

enum { ORC_DATA = 0, ORC_TMP = 1, ORC_NEW = 2 };          /* src/defs.h:21-24 */
enum { ORC_LIM_NONE = 0, ORC_LIM_AVERAGE, ORC_LIM_MINMOD,
       ORC_LIM_SUPERBEE, ORC_LIM_HARMONIC };               /* src/Limiter.h:9-15 */
enum { ORC_SCN_RIEMANN2D = 0, ORC_SCN_FFS = 1, ORC_SCN_QUADRANT = 2,
       ORC_SCN_UNIFORM = 3 };

typedef struct {
  int nx, ny;        /* interior cells (after refinement)           */
  double x0, y0;     /* centre of padded cell (0,0): B.x, B.y       (src/Mesh.c:364-365) */
  double dx, dy;
  int bc[4];         /* left, right, bottom, top codes: >0 sync, 0 open, -1 wall, -2 Dirichlet */
} orc_block;

typedef struct {
  double Kn;         /* Knudsen number  (src/Scenario.c:22) */
  double F;          /* body force in x (src/Scenario.c:23) */
  int limiter;       /* ORC_LIM_*       (src/Limiter.c:20)  */
} orc_params;

/* Initial / Dirichlet state.  kind ORC_SCN_QUADRANT uses q[k] = {rho, vx, vy, theta}
 * for the quadrants k = (x>=0) + 2*(y>=0); ORC_SCN_UNIFORM uses q[0]. */
typedef struct {
  int kind;
  double q[4][4];
} orc_scenario;

typedef struct orc_ctx orc_ctx;

orc_ctx *orc_create(const orc_block *blocks, int nblocks, const orc_params *p,
                    const orc_scenario *s);
void     orc_destroy(orc_ctx *c);
void     orc_set_params(orc_ctx *c, const orc_params *p);

/* cells = (nx+6)*(ny+6)*9 doubles, x fastest, 9 moments per cell */
void     orc_set_layer(orc_ctx *c, int layer, int block, const double *cells);
void     orc_get_layer(const orc_ctx *c, int layer, int block, double *cells);

/* SetInitial on the interior of L_DATA, then SetBoundary(L_DATA, 0)  (src/Main.c:124-138) */
void     orc_initialise(orc_ctx *c);
/* scenario state at a point, the SetInitial(U, P, t) restatement (src/Scenario.c:72-153) */
void     orc_initial_state(const orc_scenario *s, double x, double y, double t, double *U);

void     orc_set_boundary(orc_ctx *c, int layer, double t);                  /* src/Boundary.c:173 */
double   orc_update(orc_ctx *c, int block, int out_layer, int in_layer, int data0_layer,
                    double dt, double t, int heun);                          /* src/Main.c:297 */
double   orc_time_update(orc_ctx *c, double dt, double t);                   /* src/Main.c:253 */

/* Steps (src/Main.c:189-244).  max_steps > 0 caps the accepted steps (test hook; 0 =
 * no cap).  Every `show_every`-th step appends {step, CFL, t, dt} to trace (if not NULL,
 * up to trace_cap records).  Returns the accepted step count, or -1 after 10^6
 * attempts (the reference would loop on forever). */
int      orc_steps(orc_ctx *c, double *t, double tend, double CFLmax, double CFLreg,
                   int max_steps, int *nrej, int show_every,
                   double *trace, int trace_cap, int *ntrace);

/* single-cell kernels, exported for unit tests */
void     orc_primitive(const double *U, double *P);
void     orc_conservative(const double *P, double *U);
void     orc_flux2d(const double *U, double *F, double nx, double ny);
double   orc_relax(const orc_params *p, const double *U, double *Out, double dt, int flag);
double   orc_limit(int limiter, double d1, double d2);
double   orc_hll(const double *PL, const double *PR, double *flx, int dir, double dx);

#ifdef __cplusplus
}
#endif
#endif
