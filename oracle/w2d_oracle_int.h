/*
 * w2d_oracle_int.h -- oracle internals (TEST INFRASTRUCTURE ONLY).
 */
#ifndef W2D_ORACLE_INT_H
#define W2D_ORACLE_INT_H

#include "w2d_oracle.h"
#include <stddef.h>

#define W2D_MAXEQ 8

struct OrcSim {
  W2dParams p;
  W2dInit ic;
  int cap;           /* largest block ID (nblocks)            */
  int W;             /* nx + 4                                */
  size_t blk;        /* doubles per block: neq*W*W            */
  int nbmax, nbleafs;
  double *u, *up, *primit;   /* [(cap+1)*blk]                 */
  int32_t *lp;               /* [(cap+1)*8], lp(nb,k)=lp[nb*8+k-1] */
  int32_t *leaf;             /* [cap+1]                       */
  int32_t *icoord;           /* [(cap+1)*2]                   */
  double *dx, *dy;           /* [nlevs+1], 1-based            */
  int32_t *ib;               /* innerbounds [(ib_cap+1)*3], 1-based rows */
  int nib, ib_cap;
  double cooltab[2][41];
  int ncool;
  int err, err_nb, err_i, err_j;
  double time;
  long steps;
};

/* Fortran MAX/MIN of two reals as a compare-and-select (no NaN inputs). */
static inline double fmax_f(double a, double b) { return (a > b) ? a : b; }
static inline double fmin_f(double a, double b) { return (a < b) ? a : b; }

/* element (nb, k, i, j) of a pool array; k is 0-based, i, j in -1..nx+2 */
#define ARR(s, arr, nb, k, i, j) \
  (arr)[(((size_t)(nb) * (s)->p.neq + (size_t)(k)) * (s)->W + (size_t)((j) + 1)) * (s)->W + (size_t)((i) + 1)]
#define U(s, nb, k, i, j)  ARR(s, (s)->u, nb, k, i, j)
#define UP(s, nb, k, i, j) ARR(s, (s)->up, nb, k, i, j)
#define PR(s, nb, k, i, j) ARR(s, (s)->primit, nb, k, i, j)
#define LP(s, nb, k) (s)->lp[(size_t)(nb) * 8 + (k) - 1]
#define IC(s, nb, k) (s)->icoord[(size_t)(nb) * 2 + (k) - 1]
#define IB(s, e, k)  (s)->ib[(size_t)(e) * 3 + (k) - 1]

#endif
