/*
 * w2d_oracle.h -- CPU oracle for the Walicxe-2D block-update path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the
 * reference's Fortran (esquivas/walicxe2d, serial build, DOUBLEP: every
 * REAL is double) used by tests/, __graft_entry__.smoke() and the CPU
 * baseline of bench.py as the checker.  The library under walicxe2d_b200/
 * never links or calls it.
 *
 * Parity status: the reference is Fortran 90 and no Fortran compiler exists
 * in this environment, so the oracle cannot be compared with the reference
 * binary.  The reference ships no tests or golden outputs; the only shipped
 * data, src/DMClib/coolingDMC.tab, pins cooldmc at its 41 nodes
 * (tests/golden).  Everything else is "parity unpinned": pinned only by this
 * line-by-line restatement and by the known-answer tests in tests/.
 *
 * Semantics kept from the reference (each routine cites file:line):
 *   - left-to-right evaluation of every expression, x**2 as x*x, no FMA
 *     (built with -ffp-contract=off), glibc exp/pow/log/log10/sqrt;
 *   - Fortran SUM over a 2x2 section as ((((0+a11)+a21)+a12)+a22);
 *   - the sequential walk of innerbounds in boundaryI/II, corners included;
 *   - the defects listed in W2D_COMPAT_* when the compat bits are set.
 */
#ifndef W2D_ORACLE_H
#define W2D_ORACLE_H

#include "../include/w2d.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OrcSim OrcSim;

OrcSim* orc_create(const W2dParams* p, const W2dInit* ic);
void    orc_destroy(OrcSim* s);
void    orc_set_threads(OrcSim* s, int nthreads);
int     orc_set_cooltab(OrcSim* s, const double* log_t, const double* neg_log_l, int n);

/* state access (all arrays are the oracle's own storage) */
double* orc_u(OrcSim* s);        /* [(cap+1)][neq][W][W], i fastest, W = nx+4 */
double* orc_up(OrcSim* s);
double* orc_primit(OrcSim* s);
int32_t* orc_lp(OrcSim* s);      /* [(cap+1)][8]  row-major: lp[nb*8 + k-1] */
int32_t* orc_leaf(OrcSim* s);    /* [cap+1]                                  */
int32_t* orc_icoord(OrcSim* s);  /* [(cap+1)][2]                             */
double* orc_dx(OrcSim* s);       /* [nlevs+1], 1-based                       */
double* orc_dy(OrcSim* s);
int32_t* orc_innerbounds(OrcSim* s, int* n);  /* [n][3] row-major           */
int     orc_nbmax(OrcSim* s);
int     orc_nbleafs(OrcSim* s);
int     orc_error(OrcSim* s, int* nb, int* i, int* j);
double  orc_time(OrcSim* s);
int     orc_cap(OrcSim* s);
void    orc_set_nbmax(OrcSim* s, int nbmax);

/* set-up: generalized basegrid (roots nbroot_x x nbroot_y) + startup admesh */
int orc_basegrid(OrcSim* s);
int orc_startup(OrcSim* s);      /* basegrid + ic.startup_admesh admesh calls */

/* routines of the step */
int    orc_locatebounds(OrcSim* s);
double orc_timestep(OrcSim* s);
int    orc_tstep(OrcSim* s, double time, double dt);
int    orc_boundaryI(OrcSim* s, double time);
int    orc_boundaryII(OrcSim* s, double time);
int    orc_calcprim_all(OrcSim* s);
int    orc_coolingh(OrcSim* s, double dt_s);
int    orc_coolingdmc(OrcSim* s, double dt_s);
int    orc_admesh(OrcSim* s);
/* grad of criteria (per block, -1 for non-leaves) into grad[nb-1] */
int    orc_criteria_grad(OrcSim* s, double* grad);
int    orc_refine(OrcSim* s, int nb, int s1, int s2, int s3, int s4);
int    orc_coarse(OrcSim* s, int dad, int s1, int s2, int s3, int s4);
/* output (OUTBIN) and warm start of the serial build: the pointers and
 * blocks files (src/output.f90:39-67, src/basegrid.f90:167-251) */
int    orc_output_bin(OrcSim* s, const char* pointers, const char* blocks, int32_t true_value);
int    orc_read_bin(OrcSim* s, const char* pointers, const char* blocks, double time);
/* main loop: nsteps x (timestep, time+=dt, tstep, admesh if amr) */
int    orc_run(OrcSim* s, int nsteps, int amr, double* dt_last);
/* the sequential walks with the given list instead of locatebounds' one */
int    orc_set_innerbounds(OrcSim* s, const int32_t* ib, int n);

/* point functions (unit tests) */
int    orc_primf_solver(const W2dParams* p, const double* priml,
                        const double* primr, double* ff);
void   orc_limiter(const W2dParams* p, double* pll, double* pl, double* pr,
                   double* prr);
void   orc_uprim(const W2dParams* p, double* prim, const double* uu, double* T);
void   orc_atomic(const W2dParams* p, double dt, double* uu);
double orc_cooldmc(OrcSim* s, double T);
double orc_aloss(double x1, double x2, double dt, double den, double dh0,
                 double te0);

#ifdef __cplusplus
}
#endif
#endif
