/*
 * ref_scenario.c -- problem definition linked into the reference build under
 * oracle/_ref in place of the reference's own src/Scenario.c.
 *
 * TEST INFRASTRUCTURE ONLY.  It provides the interface src/Scenario.h declares
 * (Type, Kn, F, R13, CollFreq, ExternalForce, WallSign, SetInitial) so that the
 * unmodified reference sources build and run the scenarios the parity tests and
 * the CPU baseline need.  The reference ships with its ForwardFacingStep state
 * active, while its goldens were made with the Riemann2D state
 * (reference/squareSmall.ref.hdr: Type = Riemann2D); the scenario is therefore
 * chosen at run time from the environment:
 *
 *   MBM_SCENARIO unset or "riemann2d"     rho = 5 for r < 0.4, else 1 (src/Scenario.c:79-98)
 *   MBM_SCENARIO = "ffs"                  uniform Mach-2 stream         (src/Scenario.c:125-138)
 *   MBM_SCENARIO = "quadrant:r,u,v,th;..." four states for (x<0,y<0), (x>=0,y<0),
 *                                         (x<0,y>=0), (x>=0,y>=0)
 *   MBM_SCENARIO = "uniform:r,u,v,th"     one state everywhere
 *
 * The collision frequency, body force, wall sign table and the moment formula are
 * the reference's (src/Scenario.c:28-63, 140-152); every expression keeps its
 * operand order.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "database_range.h"
#include "defs.h"
#include "Scenario.h"

char Type[200];

double Kn = 0.001;
double F = 0.0;
double R13 = 0.0;

double CollFreq(double rho, double theta)
{
  double nu0 = 1.0;
  return nu0 * rho * sqrt(theta) / Kn;
}

void ExternalForce(Vector P, double t, double *g)
{
  (void)P; (void)t;
  g[0] = F;
  g[1] = 0.0;
}

const double WallSign[4][N] = {
  { +1, -1, +1, +1, +1, -1, +1, -1, +1 },
  { +1, -1, +1, +1, +1, -1, +1, -1, +1 },
  { +1, +1, -1, +1, +1, -1, +1, +1, -1 },
  { +1, +1, -1, +1, +1, -1, +1, +1, -1 },
};

static int scn_kind = -1;          /* 0 riemann2d, 1 ffs, 2 quadrant, 3 uniform */
static double scn_q[4][4];

static void scn_load(void)
{
  const char *s = getenv("MBM_SCENARIO");
  scn_kind = 0;
  if (!s || !*s || !strcmp(s, "riemann2d")) return;
  if (!strcmp(s, "ffs")) { scn_kind = 1; return; }
  int nq = 0;
  if (!strncmp(s, "quadrant:", 9)) { scn_kind = 2; nq = 4; s += 9; }
  else if (!strncmp(s, "uniform:", 8)) { scn_kind = 3; nq = 1; s += 8; }
  else { fprintf(stderr, "MBM_SCENARIO: unknown scenario '%s'\n", s); exit(2); }
  char *end;
  for (int k = 0; k < nq; k++)
    for (int m = 0; m < 4; m++) {
      scn_q[k][m] = strtod(s, &end);
      if (end == s) { fprintf(stderr, "MBM_SCENARIO: bad number list\n"); exit(2); }
      s = end;
      while (*s == ',' || *s == ';' || *s == ' ') s++;
    }
}

void SetInitial(double *U, Vector P, double t)
{
  (void)t;
  double rho, v1, v2, theta, T11, T12, T22, q1, q2, vs, E;
  double x = P.x, y = P.y;
  if (scn_kind < 0) scn_load();
  v1 = 0.0; v2 = 0.0; T12 = 0.0; q1 = 0.0; q2 = 0.0; theta = 1.0; rho = 1.0;
  switch (scn_kind) {
    case 0:
      sprintf(Type, "Riemann2D");
      rho = (sqrt(x * x + y * y) < 0.4) ? 5.0 : 1.0;
      break;
    case 1:
      sprintf(Type, "ForwardFacingStep");
      v1 = 2.0 * sqrt(5.0 / 3.0);
      break;
    default: {
      int k = scn_kind == 3 ? 0 : (x >= 0.0) + 2 * (y >= 0.0);
      sprintf(Type, scn_kind == 3 ? "Uniform" : "Quadrant");
      rho = scn_q[k][0]; v1 = scn_q[k][1]; v2 = scn_q[k][2]; theta = scn_q[k][3];
      break;
    }
  }
  T11 = theta;
  T22 = theta;
  vs = v1 * v1 + v2 * v2;
  E = 0.5 * rho * vs + 1.5 * rho * theta;
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
