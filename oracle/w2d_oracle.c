/*
 * w2d_oracle.c -- CPU oracle, hot path (TEST INFRASTRUCTURE ONLY).
 *
 * Plain-C restatement of the reference's per-step block update.  Every
 * routine cites the Fortran it follows (paths relative to the reference
 * project).  See w2d_oracle.h for the precision and parity notes; this file
 * is never linked into the library under walicxe2d_b200/.
 */
#include "w2d_oracle_int.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ======================================================================
 * point thermodynamics
 * ==================================================================== */

/* src/uprim.f90:5-63 */
void orc_uprim(const W2dParams* p, double* prim, const double* uu, double* T)
{
  const int neq = p->neq;
  double r = uu[0] > 1e-15 ? uu[0] : 1e-15;              /* max(uu(1),1e-15) */
  prim[0] = r;
  prim[1] = uu[1] / r;
  prim[2] = uu[2] / r;
  for (int k = 4; k < neq; ++k) prim[k] = uu[k];          /* passives */
  prim[3] = (uu[3] - 0.5 * r * (prim[1] * prim[1] + prim[2] * prim[2])) / p->cv;
  prim[3] = fmax_f(prim[3], 1e-15);
  if (p->cooling == W2D_ADIABATIC) {
    *T = prim[3] / r;
  } else if (p->cooling == W2D_COOLINGH) {               /* uprim.f90:38-45 */
    double dentot = (2. * r - prim[4]);
    dentot = fmax_f(dentot, 1e-15);
    *T = fmax_f(1., (prim[3] / dentot) * p->tempsc);
    prim[3] = dentot * (*T) / p->tempsc;
  } else {                                               /* uprim.f90:47-53 */
    r = fmax_f(r, 1e-15);
    *T = fmax_f(1., (prim[3] / (r)) * p->tempsc);
    prim[3] = r * (*T) / p->tempsc;
  }
}

/* src/primu.f90:4-19 */
static void primu(const W2dParams* p, const double* prim, double* uu)
{
  uu[0] = prim[0];
  uu[1] = prim[0] * prim[1];
  uu[2] = prim[0] * prim[2];
  uu[3] = 0.5 * prim[0] * (prim[1] * prim[1] + prim[2] * prim[2]) + p->cv * prim[3];
  for (int k = 4; k < p->neq; ++k) uu[k] = prim[k];
}

/* src/primf.f90:5-23 */
static void primf(const W2dParams* p, const double* prim, double* ff)
{
  double etot = 0.5 * prim[0] * (prim[1] * prim[1] + prim[2] * prim[2]) + p->cv * prim[3];
  ff[0] = prim[0] * prim[1];
  ff[1] = prim[0] * prim[1] * prim[1] + prim[3];
  ff[2] = prim[0] * prim[1] * prim[2];
  ff[3] = prim[1] * (etot + prim[3]);
  for (int k = 4; k < p->neq; ++k) ff[k] = prim[k] * prim[1];
}

/* src/sound.f90:4-13 */
static double sound(const W2dParams* p, double pr, double d)
{
  return sqrt(p->gamma * pr / d);
}

/* src/swapy.f90:4-13 */
static void swapy(double* prim)
{
  double aux = prim[1];
  prim[1] = prim[2];
  prim[2] = aux;
}

/* ======================================================================
 * Riemann solvers
 * ==================================================================== */

/* src/hllcfluxes.f90:98-173 (primfhllc).  Returns 1 on the "Error in hllc"
 * stop (NaN contact speed). */
static int primfhllc(const W2dParams* p, const double* priml, const double* primr,
                     double* ff)
{
  const int neq = p->neq;
  double uu[W2D_MAXEQ], uuk[W2D_MAXEQ];
  double csl = sound(p, priml[3], priml[0]);
  double csr = sound(p, primr[3], primr[0]);
  double sr = fmax_f(priml[1] + csl, primr[1] + csr);
  double sl = fmin_f(priml[1] - csl, primr[1] - csr);
  if (sl > 0) { primf(p, priml, ff); return 0; }
  if (sr < 0) { primf(p, primr, ff); return 0; }
  double slmul = sl - priml[1];
  double srmur = sr - primr[1];
  double rholul = priml[0] * priml[1];
  double rhorur = primr[0] * primr[1];
  double sst = (srmur * rhorur - slmul * rholul - primr[3] + priml[3])
             / (srmur * primr[0] - slmul * priml[0]);
  if (sst >= 0.) {
    double rhost = priml[0] * (slmul) / (sl - sst);
    double ek = 0.5 * priml[0] * (priml[1] * priml[1] + priml[2] * priml[2]) + p->cv * priml[3];
    uuk[0] = rhost;
    uuk[1] = rhost * sst;
    uuk[2] = rhost * priml[2];
    uuk[3] = rhost * (ek / priml[0] + (sst - priml[1]) * (sst + priml[3] / (priml[0] * slmul)));
    for (int k = 4; k < neq; ++k) uuk[k] = rhost * priml[k] / priml[0];
    primf(p, priml, ff);
    primu(p, priml, uu);
    for (int k = 0; k < neq; ++k) ff[k] = ff[k] + sl * (uuk[k] - uu[k]);
    return 0;
  }
  if (sst <= 0.) {
    double rhost = primr[0] * (srmur) / (sr - sst);
    double ek = 0.5 * primr[0] * (primr[1] * primr[1] + primr[2] * primr[2]) + p->cv * primr[3];
    /* hllcfluxes.f90:157 divides by primr(4)*srmur (compat) */
    double den = (p->compat & W2D_COMPAT_HLLC_STAR) ? primr[3] : primr[0];
    uuk[0] = rhost;
    uuk[1] = rhost * sst;
    uuk[2] = rhost * primr[2];
    uuk[3] = rhost * (ek / primr[0] + (sst - primr[1]) * (sst + primr[3] / (den * srmur)));
    for (int k = 4; k < neq; ++k) uuk[k] = rhost * primr[k] / primr[0];
    primf(p, primr, ff);
    primu(p, primr, uu);
    for (int k = 0; k < neq; ++k) ff[k] = ff[k] + sr * (uuk[k] - uu[k]);
    return 0;
  }
  return 1;
}

/* src/hllfluxes.f90:98-132 (primfhll) */
static int primfhll(const W2dParams* p, const double* priml, const double* primr,
                    double* ff)
{
  const int neq = p->neq;
  double fl[W2D_MAXEQ], fr[W2D_MAXEQ], ul[W2D_MAXEQ], ur[W2D_MAXEQ];
  double csl = sound(p, priml[3], priml[0]);
  double csr = sound(p, primr[3], primr[0]);
  double sr = fmax_f(priml[1] + csl, primr[1] + csr);
  double sl = fmin_f(priml[1] - csl, primr[1] - csr);
  if (sl > 0) { primf(p, priml, ff); return 0; }
  if (sr < 0) { primf(p, primr, ff); return 0; }
  primf(p, priml, fl);
  primf(p, primr, fr);
  primu(p, priml, ul);
  primu(p, primr, ur);
  for (int k = 0; k < neq; ++k)
    ff[k] = (sr * fl[k] - sl * fr[k] + sl * sr * (ur[k] - ul[k])) / (sr - sl);
  return 0;
}

/* src/hll_hllcfluxes.f90:98-210 (primfhll_hllc) */
static int primfhll_hllc(const W2dParams* p, const double* priml, const double* primr,
                         double* ff)
{
  const int neq = p->neq;
  double uu[W2D_MAXEQ], uuk[W2D_MAXEQ], fl[W2D_MAXEQ], fr[W2D_MAXEQ];
  double ul[W2D_MAXEQ], ur[W2D_MAXEQ];
  const double eps = 1e-6;
  double beta1, beta2;
  double dq1 = primr[1] - priml[1];
  double dq2 = primr[2] - priml[2];
  double magdeltaq = sqrt(dq1 * dq1 + dq2 * dq2);
  if (magdeltaq <= eps) {
    beta1 = 1.0;
    beta2 = 0.0;
  } else {
    double alpha1 = fabs(dq1) / magdeltaq;
    beta1 = sqrt(alpha1);
    beta2 = 1. - beta1;
  }
  double csl = sound(p, priml[3], priml[0]);
  double csr = sound(p, primr[3], primr[0]);
  double sr = fmax_f(priml[1] + csl, primr[1] + csr);
  double sl = fmin_f(priml[1] - csl, primr[1] - csr);
  if (sl > 0) { primf(p, priml, ff); return 0; }
  if (sr < 0) { primf(p, primr, ff); return 0; }
  primf(p, priml, fl);
  primf(p, primr, fr);
  primu(p, priml, ul);
  primu(p, primr, ur);
  double slmul = sl - priml[1];
  double srmur = sr - primr[1];
  double rholul = priml[0] * priml[1];
  double rhorur = primr[0] * primr[1];
  double sst = (srmur * rhorur - slmul * rholul - primr[3] + priml[3])
             / (srmur * primr[0] - slmul * priml[0]);
  if (sst >= 0.) {
    double rhost = priml[0] * (slmul) / (sl - sst);
    double ek = 0.5 * priml[0] * (priml[1] * priml[1] + priml[2] * priml[2]) + p->cv * priml[3];
    uuk[0] = rhost;
    uuk[1] = rhost * sst;
    uuk[2] = rhost * priml[2];
    uuk[3] = rhost * (ek / priml[0] + (sst - priml[1]) * (sst + priml[3] / (priml[0] * slmul)));
    for (int k = 4; k < neq; ++k) uuk[k] = rhost * priml[k] / priml[0];
    primf(p, priml, ff);
    primu(p, priml, uu);
    for (int k = 0; k < neq; ++k)
      ff[k] = beta1 * (ff[k] + sl * (uuk[k] - uu[k]))
            + beta2 * ((sr * fl[k] - sl * fr[k] + sl * sr * (ur[k] - ul[k])) / (sr - sl));
    return 0;
  }
  if (sst <= 0.) {
    double rhost = primr[0] * (srmur) / (sr - sst);
    double ek = 0.5 * primr[0] * (primr[1] * primr[1] + primr[2] * primr[2]) + p->cv * primr[3];
    double den = (p->compat & W2D_COMPAT_HLLC_STAR) ? primr[3] : primr[0]; /* :192 */
    uuk[0] = rhost;
    uuk[1] = rhost * sst;
    uuk[2] = rhost * primr[2];
    uuk[3] = rhost * (ek / primr[0] + (sst - primr[1]) * (sst + primr[3] / (den * srmur)));
    for (int k = 4; k < neq; ++k) uuk[k] = rhost * primr[k] / primr[0];
    primf(p, primr, ff);
    primu(p, primr, uu);
    for (int k = 0; k < neq; ++k)
      ff[k] = beta1 * (ff[k] + sr * (uuk[k] - uu[k]))
            + beta2 * ((sr * fl[k] - sl * fr[k] + sl * sr * (ur[k] - ul[k])) / (sr - sl));
    return 0;
  }
  return 1;
}

int orc_primf_solver(const W2dParams* p, const double* priml, const double* primr,
                     double* ff)
{
  switch (p->solver) {
    case W2D_HLL:      return primfhll(p, priml, primr, ff);
    case W2D_HLL_HLLC: return primfhll_hllc(p, priml, primr, ff);
    default:           return primfhllc(p, priml, primr, ff);
  }
}

/* ======================================================================
 * slope limiter, src/limiter.f90:7-89
 * ==================================================================== */
static double average(int limiter, double a, double b)
{
  switch (limiter) {
    case -1:                                          /* :28-31 */
      return 0.;
    case 0:                                           /* :33-36 */
      return 0.5 * (a + b);
    case 1: {                                         /* :38-43 minmod */
      double s = copysign(1., a);
      return s * fmax_f(0., fmin_f(fabs(a), s * b));
    }
    case 2:                                           /* :45-52 van Leer */
      if (a * b <= 0.) return 0.;
      return a * b * (a + b) / (a * a + b * b);
    case 3: {                                         /* :54-57 van Albada */
      const double delta = 1.e-7;
      return (a * (b * b + delta) + b * (a * a + delta)) / (a * a + b * b + delta);
    }
    case 4: {                                         /* :58-65 UMIST */
      double s = copysign(1., a);
      double c = 0.25 * a + 0.75 * b;
      double d = 0.75 * a + 0.25 * b;
      double av = fmin_f(fmin_f(fmin_f(2. * fabs(a), 2. * s * b), s * c), s * d);
      return s * fmax_f(0., av);
    }
    case 5: {                                         /* :66-72 MC */
      double s = copysign(1., a);
      double c = 0.5 * (a + b);
      double av = fmin_f(fmin_f(2. * fabs(a), 2. * s * b), s * c);
      return s * fmax_f(0., av);
    }
    default: {                                        /* :73-80 superbee */
      double s = copysign(1., b);
      double av1 = fmin_f(2. * fabs(b), s * a);
      double av2 = fmin_f(fabs(b), 2. * s * a);
      return s * fmax_f(fmax_f(0., av1), av2);
    }
  }
}

void orc_limiter(const W2dParams* p, double* pll, double* pl, double* pr, double* prr)
{
  for (int k = 0; k < p->neq; ++k) {
    double dl = pl[k] - pll[k];
    double dm = pr[k] - pl[k];
    double dr = prr[k] - pr[k];
    double al = average(p->limiter, dl, dm);
    double ar = average(p->limiter, dm, dr);
    pl[k] = pl[k] + al * 0.5;
    pr[k] = pr[k] - ar * 0.5;
  }
}

/* ======================================================================
 * per-block routines
 * ==================================================================== */

/* src/calcprim.f90:5-21 on one block of arr -> prim */
static void calcprim_block(OrcSim* s, const double* ub, double* pb)
{
  const W2dParams* p = &s->p;
  const int neq = p->neq, W = s->W;
  double uu[W2D_MAXEQ], pr[W2D_MAXEQ], T;
  for (int j = 0; j < W; ++j)
    for (int i = 0; i < W; ++i) {
      for (int k = 0; k < neq; ++k) uu[k] = ub[(k * W + j) * W + i];
      orc_uprim(p, pr, uu, &T);
      for (int k = 0; k < neq; ++k) pb[(k * W + j) * W + i] = pr[k];
    }
}

/* src/hllcfluxes.f90:7-93 (and the identical drivers of hllfluxes.f90 and
 * hll_hllcfluxes.f90): fluxes f,g(neq,0:nx,0:ny) of block nb from primit.
 * f and g are [neq][ny+1][nx+1] with (i,j) -> (j*(nx+1)+i). */
static int fluxes_block(OrcSim* s, int nb, int choice, double* f, double* g,
                        int* ei, int* ej)
{
  const W2dParams* p = &s->p;
  const int neq = p->neq, nx = p->nx, ny = p->ny;
  const int F = nx + 1;
  double pl[W2D_MAXEQ], pr[W2D_MAXEQ], pll[W2D_MAXEQ], prr[W2D_MAXEQ], ff[W2D_MAXEQ];
  for (int i = 0; i <= nx; ++i)
    for (int j = 0; j <= ny; ++j) {
      for (int k = 0; k < neq; ++k) {
        pl[k] = PR(s, nb, k, i, j);
        pr[k] = PR(s, nb, k, i + 1, j);
      }
      if (choice == 2) {
        for (int k = 0; k < neq; ++k) {
          pll[k] = PR(s, nb, k, i - 1, j);
          prr[k] = PR(s, nb, k, i + 2, j);
        }
        orc_limiter(p, pll, pl, pr, prr);
      }
      if (orc_primf_solver(p, pl, pr, ff)) { *ei = i; *ej = j; return 1; }
      for (int k = 0; k < neq; ++k) f[(k * (ny + 1) + j) * F + i] = ff[k];
      /* y direction */
      for (int k = 0; k < neq; ++k) {
        pl[k] = PR(s, nb, k, i, j);
        pr[k] = PR(s, nb, k, i, j + 1);
      }
      swapy(pl);
      swapy(pr);
      if (choice == 2) {
        for (int k = 0; k < neq; ++k) {
          pll[k] = PR(s, nb, k, i, j - 1);
          prr[k] = PR(s, nb, k, i, j + 2);
        }
        swapy(pll);
        swapy(prr);
        orc_limiter(p, pll, pl, pr, prr);
      }
      if (orc_primf_solver(p, pl, pr, ff)) { *ei = i; *ej = j; return 1; }
      swapy(ff);
      for (int k = 0; k < neq; ++k) g[(k * (ny + 1) + j) * F + i] = ff[k];
    }
  return 0;
}

/* src/step.f90:46-73 (prims): geometric source terms of cylindrical
 * coordinates (y -> r, x -> z) from the global primit of cell (i,j) */
static void prims_cell(OrcSim* s, int nb, int i, int j, double* S)
{
  const W2dParams* p = &s->p;
  const int lev = LP(s, nb, 1);
  double radius = ((double)(j + IC(s, nb, 2)) - 0.5) * s->dy[lev];
  double rho = PR(s, nb, 0, i, j);
  double H = 0.5 * rho * (PR(s, nb, 1, i, j) * PR(s, nb, 1, i, j)
                          + PR(s, nb, 2, i, j) * PR(s, nb, 2, i, j))
             + (p->cv + 1.) * PR(s, nb, 3, i, j);
  S[0] = -(rho * PR(s, nb, 2, i, j) / radius);
  S[1] = -(rho * PR(s, nb, 1, i, j) * PR(s, nb, 2, i, j) / radius);
  S[2] = -(rho * PR(s, nb, 2, i, j) * PR(s, nb, 2, i, j) / radius);
  S[3] = -(H * PR(s, nb, 2, i, j) / radius);
  for (int k = 4; k < p->neq; ++k) S[k] = -(PR(s, nb, k, i, j) * PR(s, nb, 2, i, j) / radius);
}

/* src/step.f90:5-40 */
static void step_block(OrcSim* s, int nb, double dt, const double* f, const double* g)
{
  const W2dParams* p = &s->p;
  const int neq = p->neq, nx = p->nx, ny = p->ny, F = nx + 1;
  const int lev = LP(s, nb, 1);
  const int cyl = p->geometry == W2D_GEOM_CYLINDRICAL;
  double dtdx = dt / s->dx[lev];
  double dtdy = dt / s->dy[lev];
  double S[W2D_MAXEQ];
  for (int i = 1; i <= nx; ++i)
    for (int j = 1; j <= ny; ++j) {
      if (cyl) prims_cell(s, nb, i, j, S);
      int im = i - 1, jm = j - 1;
      for (int k = 0; k < neq; ++k) {
        double fi = f[(k * (ny + 1) + j) * F + i];
        double fim = f[(k * (ny + 1) + j) * F + im];
        double gj = g[(k * (ny + 1) + j) * F + i];
        double gjm = g[(k * (ny + 1) + jm) * F + i];
        UP(s, nb, k, i, j) = U(s, nb, k, i, j) - dtdx * (fi - fim) - dtdy * (gj - gjm);
        if (cyl) UP(s, nb, k, i, j) = UP(s, nb, k, i, j) + dt * S[k];
      }
    }
}

/* src/viscosity.f90:6-25 */
static void viscosity_block(OrcSim* s, int nb)
{
  const W2dParams* p = &s->p;
  const int neq = p->neq;
  for (int i = 1; i <= p->nx; ++i)
    for (int j = 1; j <= p->ny; ++j)
      for (int k = 0; k < neq; ++k)
        UP(s, nb, k, i, j) = UP(s, nb, k, i, j)
          + p->eta * (U(s, nb, k, i + 1, j) + U(s, nb, k, i - 1, j)
                    + U(s, nb, k, i, j + 1) + U(s, nb, k, i, j - 1)
                    - 4. * U(s, nb, k, i, j));
}

static void set_error(OrcSim* s, int code, int nb, int i, int j)
{
#pragma omp critical(orc_err)
  {
    if (!s->err) { s->err = code; s->err_nb = nb; s->err_i = i; s->err_j = j; }
  }
}

/* ======================================================================
 * src/tstep.f90:4-126
 * ==================================================================== */
int orc_tstep(OrcSim* s, double time, double dt)
{
  const W2dParams* p = &s->p;
  const int nb0 = 1, nb1 = s->nbmax;
  const size_t fsz = (size_t)p->neq * (p->nx + 1) * (p->ny + 1);
  if (orc_locatebounds(s)) return s->err;
  double dtm = dt / 2.;
  /* half step */
#pragma omp parallel
  {
    double* f = (double*)malloc(fsz * sizeof(double));
    double* g = (double*)malloc(fsz * sizeof(double));
#pragma omp for schedule(dynamic, 4)
    for (int nb = nb0; nb <= nb1; ++nb) {
      if (!s->leaf[nb]) continue;
      int ei, ej;
      if (fluxes_block(s, nb, 1, f, g, &ei, &ej)) { set_error(s, W2D_ERR_HLLC, nb, ei, ej); continue; }
      step_block(s, nb, dtm, f, g);
    }
    free(f); free(g);
  }
  if (s->err) return s->err;
  orc_boundaryII(s, time);
#pragma omp parallel
  {
    double* f = (double*)malloc(fsz * sizeof(double));
    double* g = (double*)malloc(fsz * sizeof(double));
#pragma omp for schedule(dynamic, 4)
    for (int nb = nb0; nb <= nb1; ++nb) {
      if (!s->leaf[nb]) continue;
      calcprim_block(s, &UP(s, nb, 0, -1, -1), &PR(s, nb, 0, -1, -1));
      int ei, ej;
      if (fluxes_block(s, nb, 2, f, g, &ei, &ej)) { set_error(s, W2D_ERR_HLLC, nb, ei, ej); continue; }
      step_block(s, nb, dt, f, g);
      if (LP(s, nb, 1) >= (p->nlevs - 1)) viscosity_block(s, nb);
      memcpy(&U(s, nb, 0, -1, -1), &UP(s, nb, 0, -1, -1), s->blk * sizeof(double));
    }
    free(f); free(g);
  }
  if (s->err) return s->err;
  orc_boundaryI(s, time);
  if (p->cooling == W2D_ADIABATIC) {
    orc_calcprim_all(s);
  } else if (p->cooling == W2D_COOLINGH) {
    orc_coolingh(s, dt * p->tsc);
    orc_calcprim_all(s);
  } else {
    orc_coolingdmc(s, dt * p->tsc);
  }
  return s->err;
}

int orc_calcprim_all(OrcSim* s)
{
#pragma omp parallel for schedule(dynamic, 8)
  for (int nb = 1; nb <= s->nbmax; ++nb)
    if (s->leaf[nb]) calcprim_block(s, &U(s, nb, 0, -1, -1), &PR(s, nb, 0, -1, -1));
  return 0;
}

/* ======================================================================
 * src/timestep.f90:7-61
 * ==================================================================== */
double orc_timestep(OrcSim* s)
{
  const W2dParams* p = &s->p;
  double dtp = 1.e30, dtcool = 1e30;
#pragma omp parallel
  {
    double dtp_l = 1.e30, dtc_l = 1e30;
#pragma omp for schedule(dynamic, 8)
    for (int nb = 1; nb <= s->nbmax; ++nb) {
      if (!s->leaf[nb]) continue;
      int lev = LP(s, nb, 1);
      for (int i = 1; i <= p->nx; ++i)
        for (int j = 1; j <= p->ny; ++j) {
          double cs = sound(p, PR(s, nb, 3, i, j), PR(s, nb, 0, i, j));
          dtp_l = fmin_f(dtp_l, s->dx[lev] / (fabs(PR(s, nb, 1, i, j)) + cs));
          dtp_l = fmin_f(dtp_l, s->dy[lev] / (fabs(PR(s, nb, 2, i, j)) + cs));
          if (p->cooling == W2D_COOLINGDMC) {                  /* :34-41 */
            double T = (PR(s, nb, 3, i, j) / PR(s, nb, 0, i, j)) * p->tempsc;
            if (T > 1e4) {
              double aloss = orc_cooldmc(s, T) * (PR(s, nb, 0, i, j) * PR(s, nb, 0, i, j));
              dtc_l = fmin_f(dtc_l, p->cv * PR(s, nb, 3, i, j) / aloss);
            }
          }
        }
    }
#pragma omp critical(orc_dt)
    {
      dtp = fmin_f(dtp, dtp_l);
      dtcool = fmin_f(dtcool, dtc_l);
    }
  }
  return fmin_f(p->cfl * dtp, 0.4 * dtcool * p->psc / p->tsc);
}

/* ======================================================================
 * user boundary: src/jet.f90:41-78 (impose_jet), called per list entry
 * through impose_user_bc (src/user_mod.f90:74-83)
 * ==================================================================== */
static void impose_jet(OrcSim* s, double* ub, int nb, double time)
{
  const W2dParams* p = &s->p;
  const int W = s->W, neq = p->neq;
  const double pi = acos(-1.);
  int lev = LP(s, nb, 1);
  double vjet = p->jet_v0 + p->jet_dv * sin(2. * pi * time / p->jet_tau);
  for (int i = -1; i <= p->nx + 2; ++i)
    for (int j = -1; j <= p->ny + 2; ++j) {
      double x = ((double)(i + IC(s, nb, 1)) - 0.5) * s->dx[lev];
      double y = ((double)(j + IC(s, nb, 2)) - 0.5) * s->dy[lev];
      if ((fabs(x - p->jet_posx) <= p->jet_lj) && (fabs(y - p->jet_posy) <= p->jet_rj)) {
        double* c = ub + (j + 1) * W + (i + 1);
        const size_t pl = (size_t)W * W;
        c[0] = p->jet_den;
        c[pl] = p->jet_den * vjet;
        c[2 * pl] = 0.;
        c[3 * pl] = 0.5 * p->jet_den * (vjet * vjet) + p->cv * p->jet_den * 1.0001 * p->jet_temp;
        if (neq > 4) c[4 * pl] = p->jet_den * 0.9999;
        if (neq > 5) c[5 * pl] = p->jet_den;
      }
    }
}

/* ======================================================================
 * ghost fills: sequential walks of innerbounds
 * ==================================================================== */

/* 0.25*sum(a(i1:i2,j1:j2)) over a 2x2 section, Fortran column-major order */
static inline double sum4(OrcSim* s, double* arr, int nb, int k, int i1, int j1)
{
  double t = 0.;
  t += ARR(s, arr, nb, k, i1, j1);
  t += ARR(s, arr, nb, k, i1 + 1, j1);
  t += ARR(s, arr, nb, k, i1, j1 + 1);
  t += ARR(s, arr, nb, k, i1 + 1, j1 + 1);
  return 0.25 * t;
}

/* src/boundaryI.f90:34-396 (internal list, serial build) on u */
int orc_boundaryI(OrcSim* s, double time)
{
  const W2dParams* p = &s->p;
  const int neq = p->neq, nx = p->nx, ny = p->ny;
  const int nxp1 = nx + 1, nyp1 = ny + 1, nxm1 = nx - 1, nym1 = ny - 1;
  const int nx2 = nx / 2, ny2 = ny / 2, nxmax = nx + 2, nymax = ny + 2;
  double* u = s->u;
  for (int e = 1; e <= s->nib; ++e) {
    const int nbs = IB(s, e, 1), n1 = IB(s, e, 2), t = IB(s, e, 3);
    int n2;
    switch (t) {
      case -1:
        if (p->bc_left == W2D_BC_REFLECTIVE) {
          for (int j = 0; j <= nyp1; ++j)
            for (int k = 0; k < neq; ++k)
              ARR(s, u, nbs, k, 0, j) = (k == 1 ? -1. : 1.) * ARR(s, u, nbs, k, 1, j);
        } else {
          for (int j = 0; j <= nyp1; ++j)
            for (int k = 0; k < neq; ++k) ARR(s, u, nbs, k, 0, j) = ARR(s, u, nbs, k, 1, j);
        }
        break;
      case -2:
        if (p->bc_right == W2D_BC_REFLECTIVE) {
          for (int j = 0; j <= nyp1; ++j)
            for (int k = 0; k < neq; ++k)
              ARR(s, u, nbs, k, nxp1, j) = (k == 1 ? -1. : 1.) * ARR(s, u, nbs, k, nx, j);
        } else {
          for (int j = 0; j <= nyp1; ++j)
            for (int k = 0; k < neq; ++k) ARR(s, u, nbs, k, nxp1, j) = ARR(s, u, nbs, k, nx, j);
        }
        break;
      case -3:
        if (p->bc_bottom == W2D_BC_REFLECTIVE) {
          for (int i = 0; i <= nxp1; ++i)
            for (int k = 0; k < neq; ++k)
              ARR(s, u, nbs, k, i, 0) = (k == 2 ? -1. : 1.) * ARR(s, u, nbs, k, i, 1);
        } else {
          /* boundaryI.f90:87 writes block "nb", the list index */
          int tb = (p->compat & W2D_COMPAT_OUTFYB) ? e : nbs;
          if (tb >= 1 && tb <= s->cap)
            for (int i = 0; i <= nxp1; ++i)
              for (int k = 0; k < neq; ++k) ARR(s, u, tb, k, i, 0) = ARR(s, u, tb, k, i, 1);
        }
        break;
      case -4:
        if (p->bc_top == W2D_BC_REFLECTIVE) {
          for (int i = 0; i <= nxp1; ++i)
            for (int k = 0; k < neq; ++k)
              ARR(s, u, nbs, k, i, nyp1) = (k == 2 ? -1. : 1.) * ARR(s, u, nbs, k, i, ny);
        } else {
          for (int i = 0; i <= nxp1; ++i)
            for (int k = 0; k < neq; ++k) ARR(s, u, nbs, k, i, nyp1) = ARR(s, u, nbs, k, i, ny);
        }
        break;
      case 1:
        for (int j = 0; j <= nyp1; ++j)
          for (int k = 0; k < neq; ++k) ARR(s, u, nbs, k, 0, j) = ARR(s, u, n1, k, nx, j);
        for (int j = 0; j <= nyp1; ++j)
          for (int k = 0; k < neq; ++k) ARR(s, u, n1, k, nxp1, j) = ARR(s, u, nbs, k, 1, j);
        break;
      case 2:
        n2 = n1 + 2;
        for (int j = 1; j <= ny2; ++j) {
          int j1 = 2 * j - 1, ny2j = ny2 + j;
          for (int k = 0; k < neq; ++k) {
            ARR(s, u, nbs, k, 0, j) = sum4(s, u, n1, k, nxm1, j1);
            ARR(s, u, nbs, k, 0, ny2j) = sum4(s, u, n2, k, nxm1, j1);
          }
        }
        for (int k = 0; k < neq; ++k) {
          ARR(s, u, nbs, k, 0, 0) = sum4(s, u, n1, k, nxm1, -1);
          ARR(s, u, nbs, k, 0, nyp1) = sum4(s, u, n2, k, nxm1, nyp1);
        }
        for (int j = 0; j <= nyp1; ++j)
          for (int k = 0; k < neq; ++k) {
            ARR(s, u, n1, k, nxp1, j) = ARR(s, u, nbs, k, 1, (j + 1) / 2);
            ARR(s, u, n2, k, nxp1, j) = ARR(s, u, nbs, k, 1, (j + 1) / 2 + ny2);
          }
        break;
      case 4:
        for (int j = 0; j <= nyp1; ++j)
          for (int k = 0; k < neq; ++k) ARR(s, u, nbs, k, nxp1, j) = ARR(s, u, n1, k, 1, j);
        for (int j = 0; j <= nyp1; ++j)
          for (int k = 0; k < neq; ++k) ARR(s, u, n1, k, 0, j) = ARR(s, u, nbs, k, nx, j);
        break;
      case 5:
        n2 = n1 + 2;
        for (int j = 1; j <= ny2; ++j) {
          int j1 = 2 * j - 1, ny2j = ny2 + j;
          for (int k = 0; k < neq; ++k) {
            ARR(s, u, nbs, k, nxp1, j) = sum4(s, u, n1, k, 1, j1);
            ARR(s, u, nbs, k, nxp1, ny2j) = sum4(s, u, n2, k, 1, j1);
          }
        }
        for (int k = 0; k < neq; ++k) {
          ARR(s, u, nbs, k, nxp1, 0) = sum4(s, u, n1, k, 1, -1);
          ARR(s, u, nbs, k, nxp1, nyp1) = sum4(s, u, n2, k, 1, nyp1);
        }
        for (int j = 0; j <= nyp1; ++j)
          for (int k = 0; k < neq; ++k) {
            ARR(s, u, n1, k, 0, j) = ARR(s, u, nbs, k, nx, (j + 1) / 2);
            ARR(s, u, n2, k, 0, j) = ARR(s, u, nbs, k, nx, (j + 1) / 2 + ny2);
          }
        break;
      case 7:
        for (int i = 0; i <= nxp1; ++i)
          for (int k = 0; k < neq; ++k) ARR(s, u, nbs, k, i, 0) = ARR(s, u, n1, k, i, ny);
        for (int i = 0; i <= nxp1; ++i)
          for (int k = 0; k < neq; ++k) ARR(s, u, n1, k, i, nyp1) = ARR(s, u, nbs, k, i, 1);
        break;
      case 8:
        n2 = n1 + 1;
        for (int i = 1; i <= nx2; ++i) {
          int i1 = 2 * i - 1, nx2i = nx2 + i;
          for (int k = 0; k < neq; ++k) {
            ARR(s, u, nbs, k, i, 0) = sum4(s, u, n1, k, i1, nym1);
            ARR(s, u, nbs, k, nx2i, 0) = sum4(s, u, n2, k, i1, nym1);
          }
        }
        for (int k = 0; k < neq; ++k) {
          ARR(s, u, nbs, k, 0, 0) = sum4(s, u, n1, k, -1, nym1);
          ARR(s, u, nbs, k, nxp1, 0) = sum4(s, u, n2, k, nxp1, nym1);
        }
        for (int i = 0; i <= nxp1; ++i)
          for (int k = 0; k < neq; ++k) {
            ARR(s, u, n1, k, i, nyp1) = ARR(s, u, nbs, k, (i + 1) / 2, 1);
            ARR(s, u, n2, k, i, nyp1) = ARR(s, u, nbs, k, (i + 1) / 2 + nx2, 1);
          }
        break;
      case 10:
        for (int i = 0; i <= nxp1; ++i)
          for (int k = 0; k < neq; ++k) ARR(s, u, nbs, k, i, nyp1) = ARR(s, u, n1, k, i, 1);
        for (int i = 0; i <= nxp1; ++i)
          for (int k = 0; k < neq; ++k) ARR(s, u, n1, k, i, 0) = ARR(s, u, nbs, k, i, ny);
        break;
      case 11:
        n2 = n1 + 1;
        for (int i = 1; i <= nx2; ++i) {
          int i1 = 2 * i - 1, nx2i = nx2 + i;
          for (int k = 0; k < neq; ++k) {
            ARR(s, u, nbs, k, i, nyp1) = sum4(s, u, n1, k, i1, 1);
            ARR(s, u, nbs, k, nx2i, nyp1) = sum4(s, u, n2, k, i1, 1);
          }
        }
        for (int k = 0; k < neq; ++k) {
          ARR(s, u, nbs, k, 0, nyp1) = sum4(s, u, n1, k, -1, 1);
          ARR(s, u, nbs, k, nxp1, nyp1) = sum4(s, u, n2, k, nxp1, 1);
        }
        for (int i = 0; i <= nxp1; ++i)
          for (int k = 0; k < neq; ++k) {
            ARR(s, u, n1, k, i, 0) = ARR(s, u, nbs, k, (i + 1) / 2, ny);
            ARR(s, u, n2, k, i, 0) = ARR(s, u, nbs, k, (i + 1) / 2 + nx2, ny);
          }
        break;
      default:
        break;
    }
    (void)nxmax; (void)nymax;
    if (p->otherb == W2D_USERBC_JET) impose_jet(s, &ARR(s, u, nbs, 0, -1, -1), nbs, time);
  }
  return 0;
}

/* src/boundaryII.f90:35-514 (internal list, serial build) on up */
int orc_boundaryII(OrcSim* s, double time)
{
  const W2dParams* p = &s->p;
  const int neq = p->neq, nx = p->nx, ny = p->ny;
  const int nxp1 = nx + 1, nyp1 = ny + 1, nxm1 = nx - 1, nym1 = ny - 1;
  const int nx2 = nx / 2, ny2 = ny / 2, nxmax = nx + 2, nymax = ny + 2;
  double* up = s->up;
#define A(nb, k, i, j) ARR(s, up, nb, k, i, j)
  for (int e = 1; e <= s->nib; ++e) {
    const int nbs = IB(s, e, 1), n1 = IB(s, e, 2), t = IB(s, e, 3);
    int n2;
    switch (t) {
      case -1: {                                   /* :38-56 */
        int jj = 2;
        for (int i = -1; i <= 0; ++i) {
          for (int j = -1; j <= nymax; ++j)
            for (int k = 0; k < neq; ++k)
              A(nbs, k, i, j) = ((p->bc_left == W2D_BC_REFLECTIVE && k == 1) ? -1. : 1.) * A(nbs, k, jj, j);
          jj = jj - 1;
        }
        break;
      }
      case -2: {                                   /* :60-78 */
        int jj = nx;
        for (int i = nxp1; i <= nxmax; ++i) {
          for (int j = -1; j <= nymax; ++j)
            for (int k = 0; k < neq; ++k)
              A(nbs, k, i, j) = ((p->bc_right == W2D_BC_REFLECTIVE && k == 1) ? -1. : 1.) * A(nbs, k, jj, j);
          jj = jj - 1;
        }
        break;
      }
      case -3: {                                   /* :92-110 */
        int jj = 2;
        for (int i = -1; i <= 0; ++i) {
          for (int ii = -1; ii <= nxmax; ++ii)
            for (int k = 0; k < neq; ++k)
              A(nbs, k, ii, i) = ((p->bc_bottom == W2D_BC_REFLECTIVE && k == 2) ? -1. : 1.) * A(nbs, k, ii, jj);
          jj = jj - 1;
        }
        break;
      }
      case -4: {                                   /* :114-132 */
        int jj = ny;
        for (int i = nyp1; i <= nymax; ++i) {
          for (int ii = -1; ii <= nxmax; ++ii)
            for (int k = 0; k < neq; ++k)
              A(nbs, k, ii, i) = ((p->bc_top == W2D_BC_REFLECTIVE && k == 2) ? -1. : 1.) * A(nbs, k, ii, jj);
          jj = jj - 1;
        }
        break;
      }
      case 1:                                      /* :141-147 */
        for (int j = -1; j <= nymax; ++j)
          for (int k = 0; k < neq; ++k) {
            A(nbs, k, -1, j) = A(n1, k, nxm1, j);
            A(nbs, k, 0, j) = A(n1, k, nx, j);
          }
        for (int j = -1; j <= nymax; ++j)
          for (int k = 0; k < neq; ++k) {
            A(n1, k, nxp1, j) = A(nbs, k, 1, j);
            A(n1, k, nxmax, j) = A(nbs, k, 2, j);
          }
        break;
      case 2:                                      /* :149-197 */
        n2 = n1 + 2;
        for (int j = 1; j <= ny2; ++j) {
          int ny2j = ny2 + j;
          for (int i = -1; i <= 0; ++i) {
            int i1 = 2 * i - 1 + nx, j1 = 2 * j - 1;
            for (int k = 0; k < neq; ++k) {
              A(nbs, k, i, j) = sum4(s, up, n1, k, i1, j1);
              A(nbs, k, i, ny2j) = sum4(s, up, n2, k, i1, j1);
            }
          }
        }
        for (int k = 0; k < neq; ++k) {
          A(nbs, k, 0, 0) = sum4(s, up, n1, k, nxm1, -1);
          A(nbs, k, -1, 0) = sum4(s, up, n1, k, nx - 3, -1);
          A(nbs, k, 0, -1) = A(nbs, k, 0, 0);
          A(nbs, k, -1, -1) = A(nbs, k, -1, 0);
          A(nbs, k, 0, nyp1) = sum4(s, up, n2, k, nxm1, nyp1);
          A(nbs, k, -1, nyp1) = sum4(s, up, n2, k, nx - 3, nyp1);
          A(nbs, k, 0, nymax) = A(nbs, k, 0, nyp1);
          A(nbs, k, -1, nymax) = A(nbs, k, -1, nyp1);
        }
        for (int i = 1; i <= 2; ++i)
          for (int j = -1; j <= nymax; ++j)
            for (int k = 0; k < neq; ++k) {
              A(n1, k, i + nx, j) = A(nbs, k, (i + 1) / 2, (j + 1) / 2);
              A(n2, k, i + nx, j) = A(nbs, k, (i + 1) / 2, (j + 1) / 2 + ny2);
            }
        break;
      case 4:                                      /* :225-231 */
        for (int j = -1; j <= nymax; ++j)
          for (int k = 0; k < neq; ++k) {
            A(nbs, k, nxp1, j) = A(n1, k, 1, j);
            A(nbs, k, nxmax, j) = A(n1, k, 2, j);
          }
        for (int j = -1; j <= nymax; ++j)
          for (int k = 0; k < neq; ++k) {
            A(n1, k, -1, j) = A(nbs, k, nxm1, j);
            A(n1, k, 0, j) = A(nbs, k, nx, j);
          }
        break;
      case 5:                                      /* :233-281 */
        n2 = n1 + 2;
        for (int i = nxp1; i <= nxmax; ++i)
          for (int j = 1; j <= ny2; ++j) {
            int i1 = 2 * (i - nx) - 1, j1 = 2 * j - 1, ny2j = ny2 + j;
            for (int k = 0; k < neq; ++k) {
              A(nbs, k, i, j) = sum4(s, up, n1, k, i1, j1);
              A(nbs, k, i, ny2j) = sum4(s, up, n2, k, i1, j1);
            }
          }
        for (int k = 0; k < neq; ++k) {
          A(nbs, k, nxp1, 0) = sum4(s, up, n1, k, 1, -1);
          A(nbs, k, nxmax, 0) = sum4(s, up, n1, k, 3, -1);
          A(nbs, k, nxp1, -1) = A(nbs, k, nxp1, 0);
          A(nbs, k, nxmax, -1) = A(nbs, k, nxmax, 0);
          A(nbs, k, nxp1, nyp1) = sum4(s, up, n2, k, 1, nyp1);
          A(nbs, k, nxmax, nyp1) = sum4(s, up, n2, k, 3, nyp1);
          A(nbs, k, nxp1, nymax) = A(nbs, k, nxp1, nyp1);
          A(nbs, k, nxmax, nymax) = A(nbs, k, nxmax, nyp1);
        }
        for (int i = 1; i <= 2; ++i)
          for (int j = -1; j <= nymax; ++j)
            for (int k = 0; k < neq; ++k) {
              A(n1, k, i - 2, j) = A(nbs, k, (i + 1) / 2 + nxm1, (j + 1) / 2);
              A(n2, k, i - 2, j) = A(nbs, k, (i + 1) / 2 + nxm1, (j + 1) / 2 + ny2);
            }
        break;
      case 7:                                      /* :309-315 */
        for (int i = -1; i <= nxmax; ++i)
          for (int k = 0; k < neq; ++k) {
            A(nbs, k, i, -1) = A(n1, k, i, nym1);
            A(nbs, k, i, 0) = A(n1, k, i, ny);
          }
        for (int i = -1; i <= nxmax; ++i)
          for (int k = 0; k < neq; ++k) {
            A(n1, k, i, nyp1) = A(nbs, k, i, 1);
            A(n1, k, i, nymax) = A(nbs, k, i, 2);
          }
        break;
      case 8:                                      /* :317-365 */
        n2 = n1 + 1;
        for (int i = 1; i <= nx2; ++i) {
          int nx2i = nx2 + i;
          for (int j = -1; j <= 0; ++j) {
            int i1 = 2 * i - 1, j1 = 2 * j - 1 + ny;
            for (int k = 0; k < neq; ++k) {
              A(nbs, k, i, j) = sum4(s, up, n1, k, i1, j1);
              A(nbs, k, nx2i, j) = sum4(s, up, n2, k, i1, j1);
            }
          }
        }
        for (int k = 0; k < neq; ++k) {
          A(nbs, k, 0, 0) = sum4(s, up, n1, k, -1, nym1);
          A(nbs, k, 0, -1) = sum4(s, up, n1, k, -1, ny - 3);
          A(nbs, k, -1, 0) = A(nbs, k, 0, 0);
          A(nbs, k, -1, -1) = A(nbs, k, -1, 0);
          A(nbs, k, nxp1, 0) = sum4(s, up, n2, k, nxp1, nym1);
          A(nbs, k, nxp1, -1) = sum4(s, up, n2, k, nxp1, ny - 3);
          A(nbs, k, nxmax, 0) = A(nbs, k, nxp1, 0);
          A(nbs, k, nxmax, -1) = A(nbs, k, nxp1, -1);
        }
        for (int i = -1; i <= nxmax; ++i)
          for (int j = 1; j <= 2; ++j)
            for (int k = 0; k < neq; ++k) {
              A(n1, k, i, j + ny) = A(nbs, k, (i + 1) / 2, (j + 1) / 2);
              A(n2, k, i, j + ny) = A(nbs, k, (i + 1) / 2 + nx2, (j + 1) / 2);
            }
        break;
      case 10:                                     /* :393-399 */
        for (int i = -1; i <= nxmax; ++i)
          for (int k = 0; k < neq; ++k) {
            A(nbs, k, i, nyp1) = A(n1, k, i, 1);
            A(nbs, k, i, nymax) = A(n1, k, i, 2);
          }
        for (int i = -1; i <= nxmax; ++i)
          for (int k = 0; k < neq; ++k) {
            A(n1, k, i, -1) = A(nbs, k, i, nym1);
            A(n1, k, i, 0) = A(nbs, k, i, ny);
          }
        break;
      case 11:                                     /* :401-449 */
        n2 = n1 + 1;
        for (int i = 1; i <= nx2; ++i)
          for (int j = nyp1; j <= nymax; ++j) {
            int i1 = 2 * i - 1, j1 = 2 * (j - ny) - 1, nx2i = nx2 + i;
            for (int k = 0; k < neq; ++k) {
              A(nbs, k, i, j) = sum4(s, up, n1, k, i1, j1);
              A(nbs, k, nx2i, j) = sum4(s, up, n2, k, i1, j1);
            }
          }
        for (int k = 0; k < neq; ++k) {
          A(nbs, k, 0, nyp1) = sum4(s, up, n1, k, -1, 1);
          A(nbs, k, 0, nymax) = sum4(s, up, n1, k, -1, 3);
          A(nbs, k, -1, nyp1) = A(nbs, k, 0, nyp1);
          A(nbs, k, -1, nymax) = A(nbs, k, 0, nymax);
          A(nbs, k, nxp1, nyp1) = sum4(s, up, n2, k, nxp1, 1);
          A(nbs, k, nxp1, nymax) = sum4(s, up, n2, k, nxp1, 3);
          A(nbs, k, nxmax, nyp1) = A(nbs, k, nxp1, nyp1);
          A(nbs, k, nxmax, nymax) = A(nbs, k, nxp1, nymax);
        }
        for (int i = -1; i <= nxmax; ++i)
          for (int j = 1; j <= 2; ++j)
            for (int k = 0; k < neq; ++k) {
              A(n1, k, i, j - 2) = A(nbs, k, (i + 1) / 2, (j + 1) / 2 + nym1);
              A(n2, k, i, j - 2) = A(nbs, k, (i + 1) / 2 + nx2, (j + 1) / 2 + nym1);
            }
        break;
      default:
        break;
    }
    if (p->otherb == W2D_USERBC_JET) impose_jet(s, &ARR(s, up, nbs, 0, -1, -1), nbs, time);
  }
#undef A
  return 0;
}

/* ======================================================================
 * cooling
 * ==================================================================== */

/* src/coolingh.f90:41-48 */
static double alpha_rec(double T) { return 2.55e-13 * pow((1.e4 / T), 0.79); }
/* src/coolingh.f90:59-66 */
static double colf(double T) { return 5.83e-11 * sqrt(T) * exp(-157828. / T); }
/* src/coolingh.f90:68-76 */
static double betah(double T)
{
  double a = 157890. / T;
  return 1.133e-24 / sqrt(a) * (-0.0713 + 0.5 * log(a) + 0.640 * pow(a, (-0.33333)));
}

/* src/coolingh.f90:88-165 (ALOSS) */
double orc_aloss(double x1, double x2, double dt, double den, double dh0, double te0)
{
  (void)x2; (void)dt;
  const double XO = 1.e-3, XION = 2.179e-11;
  const double C0 = 0.5732, C1 = 1.8288e-5, C2 = -1.15822e-10, C3 = 9.4288e-16;
  const double D0 = 0.5856, D1 = 1.55083e-5, D2 = -9.669e-12, D3 = 5.716e-19;
  const double ENK = 118409., EN = 1.634E-11;
  double te = fmax_f(te0, 1000.);
  double dh = den;
  double dhp = (1. - x1) * dh;
  double de = dhp + 1.E-4 * dh;
  double doi = XO * dh0;
  double doii = XO * dhp;
  double omega = 0.;
  if (te <= 55000.) omega = C0 + te * (C1 + te * (C2 + te * C3));
  if (te >= 72000.) omega = D0 + te * (D1 + te * (D2 + te * D3));
  if (te > 55000. && te < 72000.) {
    double omegal = C0 + te * (C1 + te * (C2 + te * C3));
    double omegah = D0 + te * (D1 + te * (D2 + te * D3));
    double frac = (te - 55000.) / 17000.;
    omega = (1. - frac) * omegal + frac * omegah;
  }
  double qla = 8.6287E-6 / (2. * sqrt(te)) * omega * exp(-ENK / te);
  double ecoll = de * dh0 * qla * EN;
  ecoll = fmax_f(ecoll, 0.);
  double cion = 5.834E-11 * sqrt(te) * exp(-1.579E5 / te);
  double eion = de * dh0 * cion * XION;
  double erec = de * dhp * (betah(te));
  erec = fmax_f(erec, 0.);
  double tm = 1. / te;
  double t2 = tm * tm;
  double eoi = de * doi * pow(10., (1381465. * t2 - 12328.69 * tm - 19.82621));
  double eoii = de * doii * pow(10., (-2061075. * t2 - 14596.24 * tm - 19.01402));
  eoi = fmax_f(eoi, 0.);
  eoii = fmax_f(eoii, 0.);
  double betaf = 1.3 * 1.42E-27 * pow(te, 0.5);
  double hiicool = de * dhp * betaf;
  double equil = (1.0455E-18 / pow(te, 0.63)) * (1. - exp(-pow((te * 1.E-5), 1.63))) * de * den + hiicool;
  double fr = 0.;
  if (te <= 44770.) fr = 0.;
  if (te >= 54770.) fr = 1.;
  if (te > 44770. && te < 54770.) {
    double ex2 = exp(-2. * (te - 49770.) / 500.);
    double tanh_ = (1. - ex2) / (1. + ex2);
    fr = 0.5 * (1. + tanh_);
  }
  return ecoll + eion + (erec + 7.033 * (eoi + eoii)) * (1. - fr) + equil * fr;
}

/* src/coolingh.f90:171-259 (atomic) */
void orc_atomic(const W2dParams* p, double dt, double* uu)
{
  const double xi = 1.e-4, boltzm = 1.3807e-16;
  double prim[W2D_MAXEQ], T;
  orc_uprim(p, prim, uu, &T);
  double col = colf(T);
  double rec = alpha_rec(T);
  double y0 = uu[4] / uu[0];
  double dh = uu[0];
  double a = rec + col;
  double b = -((2. + xi) * rec + (1. + xi) * col);
  double c = (1. + xi) * rec;
  double d = sqrt(b * b - 4. * a * c);
  double g0 = (2. * a * y0 + b + d) / (2. * a * y0 + b - d);
  double e = exp(-d * dh * dt);
  double y1 = (-b - d * (1. + g0 * e) / (1. - g0 * e)) / (2. * a);
  y1 = fmin_f(y1, 1.);
  y1 = fmax_f(y1, 0.0001);
  uu[4] = y1 * uu[0];
  double dh0 = uu[4];
  double al = orc_aloss(y0, y1, dt, dh, dh0, T) / (dh * dh);
  double tprime = 10.;
  double ce = (2. * dh * al) / (3. * boltzm * T);
  double t1 = tprime + (T - tprime) * exp(-ce * dt);
  t1 = fmax_f(t1, 0.1 * T);
  t1 = fmin_f(t1, 10. * T);
  t1 = fmax_f(t1, tprime);
  uu[3] = p->cv * (2. * uu[0] - uu[4]) * t1 / p->tempsc
        + 0.5 * prim[0] * (prim[1] * prim[1] + prim[2] * prim[2]);
}

/* src/coolingh.f90:5-34 */
int orc_coolingh(OrcSim* s, double dt)
{
  const W2dParams* p = &s->p;
  const int neq = p->neq;
#pragma omp parallel for schedule(dynamic, 8)
  for (int nb = 1; nb <= s->nbmax; ++nb) {
    if (!s->leaf[nb]) continue;
    double uu[W2D_MAXEQ];
    for (int i = 0; i <= p->nx + 1; ++i)
      for (int j = 0; j <= p->ny + 1; ++j) {
        for (int k = 0; k < neq; ++k) uu[k] = U(s, nb, k, i, j);
        orc_atomic(p, dt, uu);
        for (int k = 0; k < neq; ++k) U(s, nb, k, i, j) = uu[k];
      }
  }
  return 0;
}

/* src/dmc_module.f90:14-32 (cooldmc).  At T == 1e8 exactly the reference
 * reads cooltab(:,42), past the table; the index is clamped to 40 here. */
double orc_cooldmc(OrcSim* s, double T)
{
  if (T > 1e8) return 0.21e-26 * sqrt(T);
  int if1 = (int)(log10(T) * 10) - 39;
  if (if1 > 40) if1 = 40;
  if (if1 < 1) if1 = 1;
  double T0 = s->cooltab[0][if1 - 1], c0 = s->cooltab[1][if1 - 1];
  double T1 = s->cooltab[0][if1], c1 = s->cooltab[1][if1];
  return (c1 - c0) * (T - T0) / (T1 - T0) + c0;
}

/* src/coolingdmc.f90:6-54 */
int orc_coolingdmc(OrcSim* s, double dt)
{
  const W2dParams* p = &s->p;
  const int neq = p->neq;
  const double Tmin = 1.e4;
#pragma omp parallel for schedule(dynamic, 8)
  for (int nb = 1; nb <= s->nbmax; ++nb) {
    if (!s->leaf[nb]) continue;
    double uu[W2D_MAXEQ], pr[W2D_MAXEQ], T;
    for (int i = 0; i <= p->nx + 1; ++i)
      for (int j = 0; j <= p->ny + 1; ++j) {
        for (int k = 0; k < neq; ++k) uu[k] = U(s, nb, k, i, j);
        orc_uprim(p, pr, uu, &T);
        for (int k = 0; k < neq; ++k) PR(s, nb, k, i, j) = pr[k];
        if (T > Tmin) {
          double eth0 = p->cv * PR(s, nb, 3, i, j);
          double aloss = orc_cooldmc(s, T);
          double dens = PR(s, nb, 0, i, j);
          double ce = (aloss * (dens * dens)) / (eth0 * p->psc);   /* Aloss*dens**2 */
          PR(s, nb, 3, i, j) = PR(s, nb, 3, i, j) * exp(-ce * dt);
          U(s, nb, 3, i, j) = U(s, nb, 3, i, j) - eth0 + p->cv * PR(s, nb, 3, i, j);
        }
      }
  }
  return 0;
}

int orc_set_cooltab(OrcSim* s, const double* log_t, const double* neg_log_l, int n)
{
  if (n != 41) return W2D_ERR_ARG;
  for (int i = 0; i < n; ++i) {                 /* src/initmain.f90:89-93 */
    s->cooltab[0][i] = pow(10.e0, (log_t[i]));
    s->cooltab[1][i] = pow(10.e0, (-neg_log_l[i]));
  }
  s->ncool = n;
  return 0;
}
