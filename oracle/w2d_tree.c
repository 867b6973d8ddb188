/*
 * w2d_tree.c -- CPU oracle, host block tree and set-up (TEST INFRASTRUCTURE
 * ONLY).  Restates the reference's integer AMR logic (serial build) and the
 * data motion of refine/coarse; used as the checker of the library's C++
 * host tree and of its device kernels.
 */
#include "w2d_oracle_int.h"

#include <math.h>
#include <stdlib.h>
#include <stdio.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ---------------------------------------------------------------------- */
OrcSim* orc_create(const W2dParams* p, const W2dInit* ic)
{
  if (p->neq < 4 || p->neq > W2D_MAXEQ || p->nx < 4 || p->nx != p->ny || p->nlevs < 1)
    return NULL;
  OrcSim* s = (OrcSim*)calloc(1, sizeof(OrcSim));
  s->p = *p;
  if (ic) s->ic = *ic;
  s->cap = p->nblocks;
  s->W = p->nx + 4;
  s->blk = (size_t)p->neq * s->W * s->W;
  size_t n = (size_t)(s->cap + 1) * s->blk;
  s->u = (double*)calloc(n, sizeof(double));
  s->up = (double*)calloc(n, sizeof(double));
  s->primit = (double*)calloc(n, sizeof(double));
  s->lp = (int32_t*)calloc((size_t)(s->cap + 1) * 8, sizeof(int32_t));
  s->leaf = (int32_t*)calloc((size_t)(s->cap + 1), sizeof(int32_t));
  s->icoord = (int32_t*)calloc((size_t)(s->cap + 1) * 2, sizeof(int32_t));
  s->dx = (double*)calloc((size_t)p->nlevs + 1, sizeof(double));
  s->dy = (double*)calloc((size_t)p->nlevs + 1, sizeof(double));
  if (!s->u || !s->up || !s->primit || !s->lp || !s->leaf || !s->icoord) {
    orc_destroy(s);
    return NULL;
  }
  /* src/initmain.f90:58-62, generalized to nbroot_x x nbroot_y roots */
  for (int l = 1; l <= p->nlevs; ++l) {
    s->dx[l] = p->xmax / p->nx / (pow(2., (double)(l - 1))) / (double)(p->nbroot_x);
    s->dy[l] = p->ymax / p->ny / (pow(2., (double)(l - 1))) / (double)(p->nbroot_y);
  }
  return s;
}

void orc_destroy(OrcSim* s)
{
  if (!s) return;
  free(s->u); free(s->up); free(s->primit); free(s->lp); free(s->leaf);
  free(s->icoord); free(s->dx); free(s->dy); free(s->ib);
  free(s);
}

void orc_set_threads(OrcSim* s, int n)
{
  (void)s;
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

double* orc_u(OrcSim* s) { return s->u; }
double* orc_up(OrcSim* s) { return s->up; }
double* orc_primit(OrcSim* s) { return s->primit; }
int32_t* orc_lp(OrcSim* s) { return s->lp; }
int32_t* orc_leaf(OrcSim* s) { return s->leaf; }
int32_t* orc_icoord(OrcSim* s) { return s->icoord; }
double* orc_dx(OrcSim* s) { return s->dx; }
double* orc_dy(OrcSim* s) { return s->dy; }
int32_t* orc_innerbounds(OrcSim* s, int* n) { *n = s->nib; return s->ib + 3; }
int orc_nbmax(OrcSim* s) { return s->nbmax; }
int orc_nbleafs(OrcSim* s) { return s->nbleafs; }
int orc_cap(OrcSim* s) { return s->cap; }
double orc_time(OrcSim* s) { return s->time; }
void orc_set_nbmax(OrcSim* s, int nbmax) { s->nbmax = nbmax; }
int orc_error(OrcSim* s, int* nb, int* i, int* j)
{
  *nb = s->err_nb; *i = s->err_i; *j = s->err_j;
  return s->err;
}

/* ---------------------------------------------------------------------- */
/* initial conditions of one block (src/user_mod.f90:39-62 and the project's
 * Sedov set-up), evaluated at the block's own resolution */
static void impose_jet_ic(OrcSim* s, int nb, double time)
{
  const W2dParams* p = &s->p;
  const double pi = acos(-1.);
  int lev = LP(s, nb, 1);
  double vjet = p->jet_v0 + p->jet_dv * sin(2. * pi * time / p->jet_tau);
  for (int i = -1; i <= p->nx + 2; ++i)
    for (int j = -1; j <= p->ny + 2; ++j) {
      double x = ((double)(i + IC(s, nb, 1)) - 0.5) * s->dx[lev];
      double y = ((double)(j + IC(s, nb, 2)) - 0.5) * s->dy[lev];
      if ((fabs(x - p->jet_posx) <= p->jet_lj) && (fabs(y - p->jet_posy) <= p->jet_rj)) {
        U(s, nb, 0, i, j) = p->jet_den;
        U(s, nb, 1, i, j) = p->jet_den * vjet;
        U(s, nb, 2, i, j) = 0.;
        U(s, nb, 3, i, j) = 0.5 * p->jet_den * (vjet * vjet) + p->cv * p->jet_den * 1.0001 * p->jet_temp;
        if (p->neq > 4) U(s, nb, 4, i, j) = p->jet_den * 0.9999;
        if (p->neq > 5) U(s, nb, 5, i, j) = p->jet_den;
      }
    }
}

static void initial_conditions(OrcSim* s, int nb)
{
  const W2dParams* p = &s->p;
  const W2dInit* ic = &s->ic;
  int lev = LP(s, nb, 1);
  for (int i = -1; i <= p->nx + 2; ++i)
    for (int j = -1; j <= p->ny + 2; ++j) {
      for (int k = 0; k < p->neq; ++k) U(s, nb, k, i, j) = 0.;
      if (ic->kind == W2D_IC_JET) {              /* src/user_mod.f90:49-58 */
        U(s, nb, 0, i, j) = ic->rho0;
        U(s, nb, 3, i, j) = p->cv * 1.0001 * ic->rho0 * ic->p0 / p->tempsc;
        if (p->neq > 4) U(s, nb, 4, i, j) = ic->rho0 * 0.9999;
        if (p->neq > 5) U(s, nb, 5, i, j) = -ic->rho0;
        continue;
      }
      double x = ((double)(i + IC(s, nb, 1)) - 0.5) * s->dx[lev];
      double y = ((double)(j + IC(s, nb, 2)) - 0.5) * s->dy[lev];
      if (ic->kind == W2D_IC_SNR) {              /* ambient + src/sn.f90:19-62 */
        U(s, nb, 0, i, j) = ic->rho0;
        U(s, nb, 3, i, j) = p->cv * ic->p0;
        if (p->neq > 4) U(s, nb, 4, i, j) = ic->rho0 * ic->xh0;
        if (p->neq > 5) U(s, nb, 5, i, j) = -ic->rho0;
        double rsc = ic->extra[3];
        double xs = x * rsc, ys = y * rsc;
        double R = sqrt((xs - ic->xc) * (xs - ic->xc) + (ys - ic->yc) * (ys - ic->yc) + ic->extra[4]);
        if (R <= ic->rb) {
          double dens = ic->extra[0];
          double vr = (R / ic->rb) * ic->extra[1] / ic->extra[2];
          U(s, nb, 0, i, j) = dens;
          U(s, nb, 1, i, j) = dens * vr * (xs - ic->xc) / (R);
          U(s, nb, 2, i, j) = dens * vr * (ys - ic->yc) / (R);
          U(s, nb, 3, i, j) = 0.5 * dens * (vr * vr) + ic->e_dep;
          if (p->neq > 4) U(s, nb, 4, i, j) = dens * 0.0;
          if (p->neq > 5) U(s, nb, 5, i, j) = dens;
        }
        continue;
      }
      double r2 = (x - ic->xc) * (x - ic->xc) + (y - ic->yc) * (y - ic->yc);
      U(s, nb, 0, i, j) = ic->rho0;
      U(s, nb, 3, i, j) = p->cv * ic->p0;
      if (p->neq > 4) U(s, nb, 4, i, j) = ic->xh0 * ic->rho0;
      if (r2 < ic->rb * ic->rb) U(s, nb, 3, i, j) = ic->e_dep;
    }
  if (ic->kind == W2D_IC_JET) impose_jet_ic(s, nb, 0.);
}

static void calcprim_one(OrcSim* s, int nb)
{
  double uu[W2D_MAXEQ], pr[W2D_MAXEQ], T;
  const int neq = s->p.neq;
  for (int j = -1; j <= s->p.ny + 2; ++j)
    for (int i = -1; i <= s->p.nx + 2; ++i) {
      for (int k = 0; k < neq; ++k) uu[k] = U(s, nb, k, i, j);
      orc_uprim(&s->p, pr, uu, &T);
      for (int k = 0; k < neq; ++k) PR(s, nb, k, i, j) = pr[k];
    }
}

/* ---------------------------------------------------------------------- */
/* refine data motion, src/refine.f90:30-38 and 227-258 (serial build) */
int orc_refine(OrcSim* s, int nb, int s1, int s2, int s3, int s4)
{
  const W2dParams* p = &s->p;
  const int nx2 = p->nx / 2, ny2 = p->ny / 2;
  for (int i = -1; i <= p->nx + 2; ++i)
    for (int j = -1; j <= p->ny + 2; ++j)
      for (int k = 0; k < p->neq; ++k) {
        U(s, s1, k, i, j) = U(s, nb, k, (i + 1) / 2, (j + 1) / 2);
        U(s, s2, k, i, j) = U(s, nb, k, (i + 1) / 2 + nx2, (j + 1) / 2);
        U(s, s3, k, i, j) = U(s, nb, k, (i + 1) / 2, (j + 1) / 2 + ny2);
        U(s, s4, k, i, j) = U(s, nb, k, (i + 1) / 2 + nx2, (j + 1) / 2 + ny2);
      }
  int nx0 = IC(s, nb, 1) * 2, ny0 = IC(s, nb, 2) * 2;
  calcprim_one(s, s1); IC(s, s1, 1) = nx0;         IC(s, s1, 2) = ny0;
  calcprim_one(s, s2); IC(s, s2, 1) = nx0 + p->nx; IC(s, s2, 2) = ny0;
  calcprim_one(s, s3); IC(s, s3, 1) = nx0;         IC(s, s3, 2) = ny0 + p->ny;
  calcprim_one(s, s4); IC(s, s4, 1) = nx0 + p->nx; IC(s, s4, 2) = ny0 + p->ny;
  return 0;
}

static inline double csum4(OrcSim* s, int nb, int k, int i1, int j1)
{
  double t = 0.;
  t += U(s, nb, k, i1, j1);
  t += U(s, nb, k, i1 + 1, j1);
  t += U(s, nb, k, i1, j1 + 1);
  t += U(s, nb, k, i1 + 1, j1 + 1);
  return 0.25 * t;
}

/* coarse data motion, src/coarse.f90:29-180 (serial build, nghost = 2) */
int orc_coarse(OrcSim* s, int dad, int s1, int s2, int s3, int s4)
{
  const W2dParams* p = &s->p;
  const int nx = p->nx, ny = p->ny, nx2 = nx / 2, ny2 = ny / 2;
  const int nxmax = nx + 2, nymax = ny + 2;
  (void)nxmax; (void)nymax;
  for (int i = 1; i <= nx2; ++i)                                  /* :32-51 */
    for (int j = 1; j <= ny2; ++j) {
      int i1 = 2 * i - 1, j1 = 2 * j - 1, nx2i = nx2 + i, ny2j = ny2 + j;
      for (int k = 0; k < p->neq; ++k) {
        U(s, dad, k, i, j) = csum4(s, s1, k, i1, j1);
        U(s, dad, k, nx2i, j) = csum4(s, s2, k, i1, j1);
        U(s, dad, k, i, ny2j) = csum4(s, s3, k, i1, j1);
        U(s, dad, k, nx2i, ny2j) = csum4(s, s4, k, i1, j1);
      }
    }
  for (int k = 0; k < p->neq; ++k) {                              /* :108-111 */
    U(s, dad, k, 0, 0) = csum4(s, s1, k, -1, -1);
    U(s, dad, k, 0, ny + 1) = csum4(s, s3, k, -1, ny + 1);
  }
  for (int i = -1; i <= 0; ++i)                                   /* :112-122 */
    for (int j = 1; j <= ny2; ++j) {
      int j1 = 2 * j - 1;
      for (int k = 0; k < p->neq; ++k) {
        U(s, dad, k, i, j) = csum4(s, s1, k, -1, j1);
        U(s, dad, k, i, ny2 + j) = csum4(s, s3, k, -1, j1);
      }
    }
  for (int k = 0; k < p->neq; ++k) {                              /* :124-127 */
    U(s, dad, k, nx + 1, 0) = csum4(s, s2, k, nx + 1, -1);
    U(s, dad, k, nx + 1, ny + 1) = csum4(s, s4, k, nx + 1, ny + 1);
  }
  for (int i = nx + 1; i <= nx + 2; ++i)                          /* :128-138 */
    for (int j = 1; j <= ny2; ++j) {
      int j1 = 2 * j - 1;
      for (int k = 0; k < p->neq; ++k) {
        U(s, dad, k, i, j) = csum4(s, s2, k, nx + 1, j1);
        U(s, dad, k, i, ny2 + j) = csum4(s, s4, k, nx + 1, j1);
      }
    }
  for (int k = 0; k < p->neq; ++k) {                              /* :140-143 */
    U(s, dad, k, 0, 0) = csum4(s, s1, k, -1, -1);
    U(s, dad, k, nx + 1, 0) = csum4(s, s2, k, nx + 1, -1);
  }
  for (int i = 1; i <= nx2; ++i)                                  /* :144-154 */
    for (int j = -1; j <= 0; ++j) {
      int i1 = 2 * i - 1;
      for (int k = 0; k < p->neq; ++k) {
        U(s, dad, k, i, j) = csum4(s, s1, k, i1, -1);
        U(s, dad, k, nx2 + i, j) = csum4(s, s2, k, i1, -1);
      }
    }
  for (int k = 0; k < p->neq; ++k) {                              /* :156-159 */
    U(s, dad, k, 0, ny + 1) = csum4(s, s3, k, -1, ny + 1);
    U(s, dad, k, nx + 1, ny + 1) = csum4(s, s4, k, nx + 1, ny + 1);
  }
  for (int i = 1; i <= nx2; ++i)                                  /* :160-170 */
    for (int j = ny + 1; j <= ny + 2; ++j) {
      int i1 = 2 * i - 1;
      for (int k = 0; k < p->neq; ++k) {
        U(s, dad, k, i, j) = csum4(s, s3, k, i1, ny + 1);
        U(s, dad, k, nx2 + i, j) = csum4(s, s4, k, i1, ny + 1);
      }
    }
  calcprim_one(s, dad);                                           /* :178 */
  return 0;
}

/* ---------------------------------------------------------------------- */
/* src/updatelpup.f90:4-190 (serial build) */
static void updatelpup(OrcSim* s, int nb, int s1, int s2, int s3, int s4,
                       unsigned char* irefup, unsigned char* irefdown)
{
  int nlev2 = LP(s, nb, 1) + 1, nsr;
  s->nbleafs += 3;   /* the MPI build's nbleafs bookkeeping, :16-21 */
  /* son1 */
  LP(s, s1, 1) = nlev2; LP(s, s1, 2) = nb; LP(s, s1, 4) = 1;
  LP(s, s1, 6) = s2; LP(s, s1, 8) = s3;
  if (LP(s, nb, 5) == -1 || s->leaf[LP(s, nb, 5)]) LP(s, s1, 5) = LP(s, nb, 5);
  else { nsr = LP(s, LP(s, nb, 5), 3) + 1; LP(s, s1, 5) = nsr; LP(s, nsr, 6) = s1; }
  if (LP(s, nb, 7) == -1 || s->leaf[LP(s, nb, 7)]) LP(s, s1, 7) = LP(s, nb, 7);
  else { nsr = LP(s, LP(s, nb, 7), 3) + 2; LP(s, s1, 7) = nsr; LP(s, nsr, 8) = s1; }
  /* son2 */
  LP(s, s2, 1) = nlev2; LP(s, s2, 2) = nb; LP(s, s2, 4) = 2;
  LP(s, s2, 5) = s1; LP(s, s2, 8) = s4;
  if (LP(s, nb, 6) == -1 || s->leaf[LP(s, nb, 6)]) LP(s, s2, 6) = LP(s, nb, 6);
  else { nsr = LP(s, LP(s, nb, 6), 3); LP(s, s2, 6) = nsr; LP(s, nsr, 5) = s2; }
  if (LP(s, nb, 7) == -1 || s->leaf[LP(s, nb, 7)]) LP(s, s2, 7) = LP(s, nb, 7);
  else { nsr = LP(s, LP(s, nb, 7), 3) + 3; LP(s, s2, 7) = nsr; LP(s, nsr, 8) = s2; }
  /* son3 */
  LP(s, s3, 1) = nlev2; LP(s, s3, 2) = nb; LP(s, s3, 4) = 3;
  LP(s, s3, 6) = s4; LP(s, s3, 7) = s1;
  if (LP(s, nb, 5) == -1 || s->leaf[LP(s, nb, 5)]) LP(s, s3, 5) = LP(s, nb, 5);
  else { nsr = LP(s, LP(s, nb, 5), 3) + 3; LP(s, s3, 5) = nsr; LP(s, nsr, 6) = s3; }
  if (LP(s, nb, 8) == -1 || s->leaf[LP(s, nb, 8)]) LP(s, s3, 8) = LP(s, nb, 8);
  else { nsr = LP(s, LP(s, nb, 8), 3); LP(s, s3, 8) = nsr; LP(s, nsr, 7) = s3; }
  /* son4 */
  LP(s, s4, 1) = nlev2; LP(s, s4, 2) = nb; LP(s, s4, 4) = 4;
  LP(s, s4, 5) = s3; LP(s, s4, 7) = s2;
  if (LP(s, nb, 6) == -1 || s->leaf[LP(s, nb, 6)]) LP(s, s4, 6) = LP(s, nb, 6);
  else { nsr = LP(s, LP(s, nb, 6), 3) + 2; LP(s, s4, 6) = nsr; LP(s, nsr, 5) = s4; }
  if (LP(s, nb, 8) == -1 || s->leaf[LP(s, nb, 8)]) LP(s, s4, 8) = LP(s, nb, 8);
  else { nsr = LP(s, LP(s, nb, 8), 3) + 1; LP(s, s4, 8) = nsr; LP(s, nsr, 7) = s4; }
  s->leaf[nb] = 0;
  s->leaf[s1] = s->leaf[s2] = s->leaf[s3] = s->leaf[s4] = 1;
  irefup[nb] = 0; irefdown[nb] = 0;
  irefdown[s1] = irefdown[s2] = irefdown[s3] = irefdown[s4] = 0;
}

/* src/updatelpdown.f90:4-59 (serial build) */
static void updatelpdown(OrcSim* s, int dad, int s1, int s2, int s3, int s4)
{
  int nb1;
  s->leaf[dad] = 1;
  s->leaf[s1] = s->leaf[s2] = s->leaf[s3] = s->leaf[s4] = 0;
  s->nbleafs -= 3;
  nb1 = LP(s, dad, 5);
  if (nb1 != -1 && !s->leaf[nb1]) {
    nb1 = LP(s, LP(s, nb1, 3), 6);
    LP(s, nb1, 6) = dad;
    LP(s, LP(s, nb1, 8), 6) = dad;
  }
  nb1 = LP(s, dad, 6);
  if (nb1 != -1 && !s->leaf[nb1]) {
    nb1 = LP(s, nb1, 3);
    LP(s, nb1, 5) = dad;
    LP(s, LP(s, nb1, 8), 5) = dad;
  }
  nb1 = LP(s, dad, 7);
  if (nb1 != -1 && !s->leaf[nb1]) {
    nb1 = LP(s, LP(s, nb1, 3), 8);
    LP(s, nb1, 8) = dad;
    LP(s, LP(s, nb1, 6), 8) = dad;
  }
  nb1 = LP(s, dad, 8);
  if (nb1 != -1 && !s->leaf[nb1]) {
    nb1 = LP(s, nb1, 3);
    LP(s, nb1, 7) = dad;
    LP(s, LP(s, nb1, 6), 7) = dad;
  }
}

/* src/criteria.f90:16-50: the max relative jump of p and rho of block nb */
static double criteria_grad(OrcSim* s, int nb)
{
  const double floor_ = 1e-15;
  double grad = 0.;
  for (int i = 1; i <= s->p.nx; ++i)
    for (int j = 1; j <= s->p.ny; ++j) {
      int ip = i + 1, jp = j + 1, im = i - 1, jm = j - 1;
      double am = fmax_f(floor_, fabs(PR(s, nb, 3, i, j)));
      double am2 = fmax_f(floor_, fabs(PR(s, nb, 0, i, j)));
      double c = PR(s, nb, 3, i, j);
      grad = fmax_f(grad, fabs(PR(s, nb, 3, ip, j) - c) / am);
      grad = fmax_f(grad, fabs(PR(s, nb, 3, im, j) - c) / am);
      grad = fmax_f(grad, fabs(PR(s, nb, 3, i, jp) - c) / am);
      grad = fmax_f(grad, fabs(PR(s, nb, 3, i, jm) - c) / am);
      c = PR(s, nb, 0, i, j);
      grad = fmax_f(grad, fabs(PR(s, nb, 0, ip, j) - c) / am2);
      grad = fmax_f(grad, fabs(PR(s, nb, 0, im, j) - c) / am2);
      grad = fmax_f(grad, fabs(PR(s, nb, 0, i, jp) - c) / am2);
      grad = fmax_f(grad, fabs(PR(s, nb, 0, i, jm) - c) / am2);
    }
  return grad;
}

int orc_criteria_grad(OrcSim* s, double* grad)
{
#pragma omp parallel for schedule(dynamic, 8)
  for (int nb = 1; nb <= s->nbmax; ++nb)
    grad[nb - 1] = s->leaf[nb] ? criteria_grad(s, nb) : -1.;
  return 0;
}

/* src/markref.f90:4-85 + criteria flags (src/criteria.f90:36-50).  The max
 * is order-free, so the early return of criteria.f90:45 gives the same flags
 * as testing the block's maximum. */
static void markref(OrcSim* s, unsigned char* irefup, unsigned char* irefdown)
{
  double* grad = (double*)malloc(sizeof(double) * (size_t)(s->nbmax + 1));
  memset(irefup, 0, (size_t)s->cap + 1);
  memset(irefdown, 0, (size_t)s->cap + 1);
  orc_criteria_grad(s, grad);
  for (int nb = 1; nb <= s->nbmax; ++nb) {
    if (!(s->leaf[nb] && LP(s, nb, 1) >= 1)) continue;
    double g = grad[nb - 1];
    if (g >= s->p.tol) {
      if (LP(s, nb, 1) < s->p.nlevs) { irefup[nb] = 1; irefdown[nb] = 0; }
    } else if (g <= s->p.tol2) {
      irefdown[nb] = 1;
    }
  }
  free(grad);
}

/* src/critneighup.f90:5-61 (serial build) */
static void critneighup(OrcSim* s, unsigned char* irefup)
{
  for (int nl = s->p.nlevs - 1; nl >= 1; --nl)
    for (int nb = 1; nb <= s->nbmax; ++nb)
      if (irefup[nb] && LP(s, nb, 1) == nl)
        for (int k = 5; k <= 8; ++k) {
          int n1 = LP(s, nb, k);
          if (n1 != -1 && LP(s, n1, 1) < LP(s, nb, 1)) irefup[n1] = 1;
        }
}

/* src/critneighdown.f90:5-55 (serial build) */
static void critneighdown(OrcSim* s, unsigned char* irefdown)
{
  for (int nb = 1; nb <= s->nbmax; ++nb)
    if (irefdown[nb])
      for (int k = 5; k <= 8; ++k) {
        int n1 = LP(s, nb, k);
        if (n1 != -1 && !s->leaf[n1]) irefdown[nb] = 0;
      }
}

/* src/admesh.f90:4-111 (np = 1).  The pool-overflow test uses the updated
 * count (the reference tests the stale nbmax, admesh.f90:44). */
int orc_admesh(OrcSim* s)
{
  const int nlevs = s->p.nlevs;
  unsigned char* irefup = (unsigned char*)calloc((size_t)s->cap + 1, 1);
  unsigned char* irefdown = (unsigned char*)calloc((size_t)s->cap + 1, 1);
  int nbmaxp = s->nbmax, nbmaxp1 = s->nbmax;
  markref(s, irefup, irefdown);
  critneighup(s, irefup);
  for (int nl = 1; nl <= nlevs - 1; ++nl)
    for (int nb = 1; nb <= nbmaxp1; ++nb) {
      if (!(LP(s, nb, 1) == nl && irefup[nb])) continue;
      int s1, s2, s3, s4;
      if (LP(s, nb, 3) == 0) {
        s1 = nbmaxp + 1; s2 = s1 + 1; s3 = s1 + 2; s4 = s1 + 3;
        if (s4 > s->cap) { s->err = W2D_ERR_CAPACITY; free(irefup); free(irefdown); return s->err; }
        LP(s, nb, 3) = s1;
        nbmaxp += 4;
      } else {
        s1 = LP(s, nb, 3); s2 = LP(s, s1, 6); s3 = LP(s, s1, 8); s4 = LP(s, s3, 6);
      }
      s->nbmax = nbmaxp;
      orc_refine(s, nb, s1, s2, s3, s4);
      updatelpup(s, nb, s1, s2, s3, s4, irefup, irefdown);
    }
  critneighdown(s, irefdown);
  for (int nl = nlevs; nl >= 2; --nl)
    for (int nb = 1; nb <= nbmaxp1; ++nb) {
      if (!(irefdown[nb] && LP(s, nb, 4) == 1 && LP(s, nb, 1) == nl)) continue;
      int dad = LP(s, nb, 2), s1 = nb, s2 = LP(s, nb, 6), s3 = LP(s, nb, 8);
      int s4 = LP(s, LP(s, nb, 6), 8);
      if (irefdown[s2] && irefdown[s3] && irefdown[s4]) {
        orc_coarse(s, dad, s1, s2, s3, s4);
        updatelpdown(s, dad, s1, s2, s3, s4);
      }
    }
  free(irefup);
  free(irefdown);
  return 0;
}

/* ---------------------------------------------------------------------- */
/* src/locatebounds.f90:29-540 (serial build).  The list is sized by the
 * current leaf count; the serial reference sizes it by an nbleafs that only
 * the MPI build keeps up to date. */
static void ib_push(OrcSim* s, int a, int b, int t)
{
  if (s->nib + 1 > s->ib_cap) {
    int nc = s->ib_cap ? 2 * s->ib_cap : 64;
    s->ib = (int32_t*)realloc(s->ib, sizeof(int32_t) * 3 * (size_t)(nc + 1));
    s->ib_cap = nc;
  }
  s->nib++;
  IB(s, s->nib, 1) = a; IB(s, s->nib, 2) = b; IB(s, s->nib, 3) = t;
}

int orc_locatebounds(OrcSim* s)
{
  unsigned char* bounds = (unsigned char*)calloc(((size_t)s->cap + 1) * 4, 1);
#define BND(nb, k) bounds[(size_t)(nb) * 4 + (k) - 1]
  s->nib = 0;
  for (int nb = 1; nb <= s->nbmax; ++nb) {
    if (!s->leaf[nb]) continue;
    /* left */
    if (!BND(nb, 1)) {
      if (LP(s, nb, 5) == -1) { BND(nb, 1) = 1; ib_push(s, nb, 0, -1); }
      else if (LP(s, LP(s, nb, 5), 1) >= LP(s, nb, 1)) {
        int n1 = LP(s, nb, 5);
        if (s->leaf[n1]) { ib_push(s, nb, n1, 1); BND(nb, 1) = 1; BND(n1, 2) = 1; }
        else {
          BND(nb, 1) = 1;
          n1 = LP(s, n1, 3) + 1; int n2 = n1 + 2;
          ib_push(s, nb, n1, 2); BND(n1, 2) = 1; BND(n2, 2) = 1;
        }
      }
    }
    /* right */
    if (!BND(nb, 2)) {
      if (LP(s, nb, 6) == -1) { BND(nb, 2) = 1; ib_push(s, nb, 0, -2); }
      else if (LP(s, LP(s, nb, 6), 1) >= LP(s, nb, 1)) {
        int n1 = LP(s, nb, 6);
        if (s->leaf[n1]) { ib_push(s, nb, n1, 4); BND(nb, 2) = 1; BND(n1, 1) = 1; }
        else {
          BND(nb, 2) = 1;
          n1 = LP(s, n1, 3); int n2 = n1 + 2;
          ib_push(s, nb, n1, 5); BND(n1, 1) = 1; BND(n2, 1) = 1;
        }
      }
    }
    /* bottom */
    if (!BND(nb, 3)) {
      if (LP(s, nb, 7) == -1) { BND(nb, 3) = 1; ib_push(s, nb, 0, -3); }
      else if (LP(s, LP(s, nb, 7), 1) >= LP(s, nb, 1)) {
        int n1 = LP(s, nb, 7);
        if (s->leaf[n1]) { ib_push(s, nb, n1, 7); BND(nb, 3) = 1; BND(n1, 4) = 1; }
        else {
          BND(nb, 3) = 1;
          n1 = LP(s, n1, 3) + 2; int n2 = n1 + 1;
          ib_push(s, nb, n1, 8); BND(n1, 4) = 1; BND(n2, 4) = 1;
        }
      }
    }
    /* top */
    if (!BND(nb, 4)) {
      if (LP(s, nb, 8) == -1) { BND(nb, 4) = 1; ib_push(s, nb, 0, -4); }
      else if (LP(s, LP(s, nb, 8), 1) >= LP(s, nb, 1)) {
        int n1 = LP(s, nb, 8);
        if (s->leaf[n1]) { ib_push(s, nb, n1, 10); BND(nb, 4) = 1; BND(n1, 3) = 1; }
        else {
          BND(nb, 4) = 1;
          n1 = LP(s, n1, 3); int n2 = n1 + 1;
          ib_push(s, nb, n1, 11); BND(n1, 3) = 1; BND(n2, 3) = 1;
        }
      }
    }
  }
#undef BND
  free(bounds);
  return 0;
}

int orc_set_innerbounds(OrcSim* s, const int32_t* ib, int n)
{
  s->nib = 0;
  for (int e = 0; e < n; ++e) ib_push(s, ib[3 * e], ib[3 * e + 1], ib[3 * e + 2]);
  return 0;
}

/* ---------------------------------------------------------------------- */
/* src/basegrid.f90:26-165, generalized: nbroot_x x nbroot_y roots at level
 * 1 numbered row by row (x fastest), then uniform refinement to
 * ic.init_levels with the initial conditions re-applied to the sons. */
int orc_basegrid(OrcSim* s)
{
  const W2dParams* p = &s->p;
  const int nbx = p->nbroot_x, nby = p->nbroot_y;
  if (nbx * nby > s->cap) return s->err = W2D_ERR_CAPACITY;
  for (int iy = 0; iy < nby; ++iy)
    for (int ix = 0; ix < nbx; ++ix) {
      int nb = 1 + ix + iy * nbx;
      LP(s, nb, 1) = 1; LP(s, nb, 2) = 0; LP(s, nb, 3) = 0; LP(s, nb, 4) = 1;
      LP(s, nb, 5) = ix > 0 ? nb - 1 : -1;
      LP(s, nb, 6) = ix < nbx - 1 ? nb + 1 : -1;
      LP(s, nb, 7) = iy > 0 ? nb - nbx : -1;
      LP(s, nb, 8) = iy < nby - 1 ? nb + nbx : -1;
      IC(s, nb, 1) = ix * p->nx;
      IC(s, nb, 2) = iy * p->ny;
      s->leaf[nb] = 1;
      initial_conditions(s, nb);
      calcprim_one(s, nb);
    }
  s->nbmax = nbx * nby;
  s->nbleafs = nbx * nby;
  unsigned char* irefup = (unsigned char*)calloc((size_t)s->cap + 1, 1);
  unsigned char* irefdown = (unsigned char*)calloc((size_t)s->cap + 1, 1);
  int lmax = s->ic.init_levels < p->nlevs ? s->ic.init_levels : p->nlevs;
  for (int lev = 1; lev < lmax; ++lev) {
    int nb0 = s->nbmax;
    for (int nb = 1; nb <= nb0; ++nb) {
      if (!(s->leaf[nb] && LP(s, nb, 1) == lev)) continue;
      int s1 = s->nbmax + 1;
      if (s1 + 3 > s->cap) { free(irefup); free(irefdown); return s->err = W2D_ERR_CAPACITY; }
      LP(s, nb, 3) = s1;
      orc_refine(s, nb, s1, s1 + 1, s1 + 2, s1 + 3);
      updatelpup(s, nb, s1, s1 + 1, s1 + 2, s1 + 3, irefup, irefdown);
      s->nbmax += 4;
      for (int n2 = s1; n2 <= s1 + 3; ++n2) { initial_conditions(s, n2); calcprim_one(s, n2); }
    }
  }
  free(irefup);
  free(irefdown);
  return 0;
}

int orc_startup(OrcSim* s)
{
  int rc = orc_basegrid(s);
  if (rc) return rc;
  for (int k = 0; k < s->ic.startup_admesh && s->p.nlevs > 1; ++k)
    if ((rc = orc_admesh(s))) return rc;
  return 0;
}

/* src/main.f90:69-107 without output: timestep, time+dt, tstep, admesh */
int orc_run(OrcSim* s, int nsteps, int amr, double* dt_last)
{
  for (int n = 0; n < nsteps; ++n) {
    double dt = orc_timestep(s);
    s->time = s->time + dt;
    if (dt_last) *dt_last = dt;
    int rc = orc_tstep(s, s->time, dt);
    if (rc) return rc;
    if (amr && s->p.nlevs > 1) {
      rc = orc_admesh(s);
      if (rc) return rc;
    }
    s->steps++;
  }
  return 0;
}

/* ---------------------------------------------------------------------- */
/* src/output.f90:39-67 (OUTBIN, serial build).  Both files are unformatted
 * little-endian streams.  pointers: nbmin, nbmax, nbleafs, nblocks, then
 * lp(nbmin:nbmax,1:8), leaf(nbmin:nbmax) and icoord(nbmin:nbmax,1:2), each
 * array column-major (block ID fastest) in 4-byte integers, leaf holding
 * true_value for .true. and 0 for .false.; blocks: u(nb,:,:,:) of every
 * leaf in ascending ID, the equation index fastest, then i, then j, 8-byte
 * reals (DOUBLEP).  nbmin is 1 in the serial build. */
int orc_output_bin(OrcSim* s, const char* pointers, const char* blocks, int32_t true_value)
{
  FILE* f = fopen(pointers, "wb");
  if (!f) return s->err = W2D_ERR_ARG;
  const int32_t head[4] = {1, s->nbmax, s->nbleafs, s->cap};
  fwrite(head, sizeof(int32_t), 4, f);
  for (int k = 1; k <= 8; ++k)
    for (int nb = 1; nb <= s->nbmax; ++nb) fwrite(&LP(s, nb, k), sizeof(int32_t), 1, f);
  for (int nb = 1; nb <= s->nbmax; ++nb) {
    const int32_t v = s->leaf[nb] ? true_value : 0;
    fwrite(&v, sizeof(int32_t), 1, f);
  }
  for (int k = 1; k <= 2; ++k)
    for (int nb = 1; nb <= s->nbmax; ++nb) fwrite(&IC(s, nb, k), sizeof(int32_t), 1, f);
  if (fclose(f)) return s->err = W2D_ERR_ARG;
  f = fopen(blocks, "wb");
  if (!f) return s->err = W2D_ERR_ARG;
  const int W = s->W, neq = s->p.neq;
  for (int nb = 1; nb <= s->nbmax; ++nb) {
    if (!s->leaf[nb]) continue;
    for (int j = -1; j <= W - 2; ++j)
      for (int i = -1; i <= W - 2; ++i)
        for (int k = 0; k < neq; ++k) fwrite(&U(s, nb, k, i, j), sizeof(double), 1, f);
  }
  if (fclose(f)) return s->err = W2D_ERR_ARG;
  return 0;
}

/* src/basegrid.f90:167-251, the warm start of the serial build: the tree
 * and the leaf blocks from the two files of orc_output_bin, then calcprim of
 * every leaf (src/basegrid.f90:241-247); the run time is set to `time` (the
 * reference takes itprint*dtprint, src/initmain.f90:69-73).  The pointer
 * renumbering of basegrid.f90:188-206 applies only to files of several MPI
 * ranks, whose pointers exceed nblocks; a serial file never does.  Any
 * nonzero leaf value reads as .true. */
int orc_read_bin(OrcSim* s, const char* pointers, const char* blocks, double time)
{
  FILE* f = fopen(pointers, "rb");
  if (!f) return s->err = W2D_ERR_ARG;
  int32_t head[4];
  int ok = fread(head, sizeof(int32_t), 4, f) == 4;
  const int nbmax = head[1];
  if (!ok || head[0] != 1 || nbmax < 1 || nbmax > s->cap) {
    fclose(f);
    return s->err = ok && nbmax > s->cap ? W2D_ERR_CAPACITY : W2D_ERR_ARG;
  }
  memset(s->lp, 0, sizeof(int32_t) * 8 * ((size_t)s->cap + 1));
  memset(s->leaf, 0, sizeof(int32_t) * ((size_t)s->cap + 1));
  memset(s->icoord, 0, sizeof(int32_t) * 2 * ((size_t)s->cap + 1));
  for (int k = 1; k <= 8 && ok; ++k)
    for (int nb = 1; nb <= nbmax && ok; ++nb) ok = fread(&LP(s, nb, k), sizeof(int32_t), 1, f) == 1;
  int nleaf = 0;
  for (int nb = 1; nb <= nbmax && ok; ++nb) {
    int32_t v;
    ok = fread(&v, sizeof(int32_t), 1, f) == 1;
    s->leaf[nb] = v != 0;
    nleaf += v != 0;
  }
  for (int k = 1; k <= 2 && ok; ++k)
    for (int nb = 1; nb <= nbmax && ok; ++nb) ok = fread(&IC(s, nb, k), sizeof(int32_t), 1, f) == 1;
  fclose(f);
  if (!ok || nleaf != head[2]) return s->err = W2D_ERR_ARG;
  s->nbmax = nbmax;
  s->nbleafs = head[2];
  f = fopen(blocks, "rb");
  if (!f) return s->err = W2D_ERR_ARG;
  const int W = s->W, neq = s->p.neq;
  for (int nb = 1; nb <= nbmax && ok; ++nb) {
    if (!s->leaf[nb]) continue;
    for (int j = -1; j <= W - 2 && ok; ++j)
      for (int i = -1; i <= W - 2 && ok; ++i)
        for (int k = 0; k < neq && ok; ++k) ok = fread(&U(s, nb, k, i, j), sizeof(double), 1, f) == 1;
  }
  char extra;
  if (ok) ok = fread(&extra, 1, 1, f) == 0;   /* nothing may follow the last leaf */
  fclose(f);
  if (!ok) return s->err = W2D_ERR_ARG;
  s->time = time;
  return orc_calcprim_all(s);
}
