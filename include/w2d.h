/*
 * w2d.h -- C-ABI of the B200 block-update library for Walicxe-2D.
 *
 * The library owns a device-resident pool of blocks (conserved variables u,
 * the half-step copy up and, under DMC cooling, the primitives) indexed by
 * the reference's own block ID.  A host that keeps the reference's Fortran
 * main loop and its integer block tree (admesh, markref, locatebounds ...)
 * calls these entry points in place of the Fortran subroutines named in each
 * comment.  All entry points return an int status (W2D_OK == 0); no entry
 * point keeps a host pointer after it returns.
 *
 * Array conventions follow the reference's Fortran globals
 * (src/globals.f90:13-29):
 *   - block IDs are 1-based (nbmin..nbmax);
 *   - lp(nb,1:8), icoord(nb,1:2) and innerbounds(n,1:3) are column-major
 *     with a caller-given leading dimension;
 *   - Fortran LOGICAL arrays (leaf) are passed as 4-byte integers, any
 *     nonzero value meaning .true.;
 *   - a block's variables are u(nb, ieq, i, j) with ieq = 1..neq and
 *     i, j = -1..nx+2.  The block-major entry points (w2d_put_blocks,
 *     w2d_get_blocks) use [block][ieq][j][i] with i fastest, which is also
 *     the device pool layout; the *_fortran variants read and write the
 *     reference's own u(nbmin:nbmaxtot, neq, -1:18, -1:18) array directly.
 */
#ifndef W2D_H
#define W2D_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define W2D_OK              0
#define W2D_ERR_ARG         1  /* bad argument or unsupported parameter      */
#define W2D_ERR_CUDA        2  /* CUDA runtime error (message in last_error) */
#define W2D_ERR_HLLC        3  /* NaN contact speed: src/hllcfluxes.f90:170  */
#define W2D_ERR_CAPACITY    4  /* block pool exhausted: src/admesh.f90:44    */
#define W2D_ERR_TOPOLOGY    5  /* innerbounds leaves a leaf face unfilled    */
#define W2D_ERR_TIMEOUT     6  /* a bounded device wait gave up              */
#define W2D_ERR_STATE       7  /* call out of order (e.g. no topology yet)   */
#define W2D_ERR_NOMEM       8  /* device or host allocation failed           */

/* ---- method selectors (JET/Makefile:27-62 compile-time flags) ----------- */
#define W2D_HLLC        0   /* -DHLLC      src/hllcfluxes.f90     */
#define W2D_HLL         1   /* -DHLL       src/hllfluxes.f90      */
#define W2D_HLL_HLLC    2   /* -DHLL_HLLC  src/hll_hllcfluxes.f90 */

#define W2D_ADIABATIC   0   /* -DADIABATIC  */
#define W2D_COOLINGH    1   /* -DCOOLINGH   src/coolingh.f90  */
#define W2D_COOLINGDMC  2   /* -DCOOLINGDMC src/coolingdmc.f90 */

#define W2D_BC_OUTFLOW     0   /* -DOUTF*  */
#define W2D_BC_REFLECTIVE  1   /* -DREF*   */

#define W2D_USERBC_NONE 0
#define W2D_USERBC_JET  1   /* -DOTHERB with impose_jet, src/jet.f90:41 */

#define W2D_GEOM_CARTESIAN   0
#define W2D_GEOM_CYLINDRICAL 1  /* -DCYLINDRICAL: x -> z, y -> r, source terms of src/step.f90:42-78 */

/* Reproduce the reference's known defects (default: both on).             */
#define W2D_COMPAT_HLLC_STAR 1  /* primr(4)/(primr(4)*srmur): hllcfluxes.f90:157 */
#define W2D_COMPAT_OUTFYB    2  /* u(nb,...) with nb the list index: boundaryI.f90:87 */

/* ---- runtime parameters (src/parameters.f90 compile-time constants) ---- */
typedef struct W2dParams {
  int32_t neq;        /* equations incl. passive scalars (4..8)             */
  int32_t npas;       /* passive scalars, neq == 4 + npas                   */
  int32_t nx, ny;     /* interior cells per block side (16)                 */
  int32_t nlevs;      /* refinement levels                                  */
  int32_t nbroot_x;   /* root blocks in x                                   */
  int32_t nbroot_y;   /* root blocks in y                                   */
  int32_t nblocks;    /* pool capacity: largest block ID                    */
  int32_t solver;     /* W2D_HLLC / W2D_HLL / W2D_HLL_HLLC                   */
  int32_t limiter;    /* LIMITER, -1..6 (src/limiter.f90:30-85)              */
  int32_t cooling;    /* W2D_ADIABATIC / W2D_COOLINGH / W2D_COOLINGDMC        */
  int32_t bc_left, bc_right, bc_bottom, bc_top;  /* W2D_BC_*                 */
  int32_t otherb;     /* W2D_USERBC_*                                        */
  int32_t compat;     /* W2D_COMPAT_* bit set                                */
  int32_t precision;  /* 64 (plain FP64 path) or 32 (FP32 state and fluxes)  */
  int32_t geometry;   /* W2D_GEOM_* (JET/Makefile:39 CYLINDRICAL)             */
  double cv, gamma, cfl, eta;      /* src/parameters.f90:39,61-63           */
  double xmax, ymax;               /* box size, code units                   */
  double tempsc, psc, tsc, rsc;    /* scalings, src/parameters.f90:50-54     */
  double tol, tol2;                /* refinement tolerances, criteria.f90:11 */
  /* jet source (src/jet.f90:14-33), code units */
  double jet_rj, jet_lj, jet_posx, jet_posy;
  double jet_den, jet_temp, jet_v0, jet_dv, jet_tau;
} W2dParams;

typedef struct W2dError {
  int32_t code;       /* W2D_ERR_* of the first failure                     */
  int32_t block;      /* block ID where the device saw it (0 if none)       */
  int32_t i, j;       /* cell or interface index (reference numbering)      */
  char message[240];
} W2dError;

typedef struct W2dCtx W2dCtx;

/* ---- lifecycle ---------------------------------------------------------- */
/* Replaces the allocate() of u, up, primit in src/initmain.f90:76-81. */
int w2d_create(const W2dParams* p, W2dCtx** out);
int w2d_destroy(W2dCtx* ctx);
/* Copies the first failure seen since the last call, then clears it. */
int w2d_last_error(W2dCtx* ctx, W2dError* err);
/* DMC table as read in src/initmain.f90:83-98: n rows of (log10 T, -log10 L). */
int w2d_set_cooltab(W2dCtx* ctx, const double* log_t, const double* neg_log_l, int n);
/* Failure detection check (no counterpart in the reference): one kernel
 * waits on a barrier that nothing completes.  Every device wait of the
 * library is bounded (about a second); this one runs out, the kernel
 * reports W2D_ERR_TIMEOUT through the context's error word and ends, and
 * the call returns W2D_ERR_TIMEOUT (w2d_last_error holds the message).  The
 * context stays usable.  Takes a second or so. */
int w2d_wait_selftest(W2dCtx* ctx);
/* Library version string and the build's target architecture. */
const char* w2d_version(void);

/* ---- topology (produced on the host by basegrid/admesh/locatebounds) ---- */
/* lp(nb,1:8), leaf(nb), icoord(nb,1:2) for nb = 1..nbmax, column-major with
 * leading dimensions ld_lp / ld_icoord (rows are block IDs starting at 1).
 * Mirrors the globals lp, leaf, icoord (src/globals.f90:19-24) and dx, dy
 * (src/initmain.f90:58-62); dx and dy hold nlevs entries. */
int w2d_set_topology(W2dCtx* ctx, const int32_t* lp, int ld_lp,
                     const int32_t* leaf, const int32_t* icoord, int ld_icoord,
                     int nbmax, const double* dx, const double* dy);
/* innerbounds(1:ninternal,1:3) as built by locatebounds
 * (src/locatebounds.f90:29-540), column-major with leading dimension ld. */
int w2d_set_bounds(W2dCtx* ctx, const int32_t* innerbounds, int ld, int ninternal);

/* ---- block data (host <-> pool) ----------------------------------------- */
/* u of the n blocks ids[0..n-1], block-major [n][neq][nx+4][nx+4], i fastest.
 * put also recomputes the stored primitives and the CFL partials of those
 * blocks, as calcprim does after the reference sets u (basegrid.f90:38-41). */
int w2d_put_blocks(W2dCtx* ctx, const int32_t* ids, int n, const double* u);
int w2d_get_blocks(W2dCtx* ctx, const int32_t* ids, int n, double* u);
/* Same, on the reference's Fortran array u(nbmin:nbmaxtot,neq,-1:18,-1:18)
 * with leading dimension ld (= nbmaxtot-nbmin+1); only the listed IDs move. */
int w2d_put_u_fortran(W2dCtx* ctx, const double* u, int ld, int nbmin,
                      const int32_t* ids, int n);
int w2d_get_u_fortran(W2dCtx* ctx, double* u, int ld, int nbmin,
                      const int32_t* ids, int n);
/* primit (block-major, like w2d_get_blocks) as the reference holds it. */
int w2d_get_primit(W2dCtx* ctx, const int32_t* ids, int n, double* prim);
/* Conserved totals (no counterpart in the reference, which writes no
 * totals): tot[q] = sum over the interior cells of every leaf of u(q) dV
 * for q = 1..neq (mass, the two momenta, energy, passives), dV = dx dy of
 * the cell's level, times the radius in cylindrical geometry (volume per
 * radian).  Per-block partials are formed on the device in FP64, in a
 * fixed order, and summed on the host in leaf order, so the totals are
 * FP64 whatever the precision of the state (the FP32 path keeps them in
 * FP64) and repeat exactly for the same state. */
int w2d_totals(W2dCtx* ctx, double* tot);

/* ---- the per-step block update (src/main.f90:87-98) --------------------- */
/* timestep(dt), src/timestep.f90:7-61: CFL minimum over interior leaf cells
 * (and the DMC cooling-time limit).  Writes dt to *dt. */
int w2d_timestep(W2dCtx* ctx, double* dt);
/* tstep(time,dt), src/tstep.f90:4-126, after w2d_set_bounds has received the
 * list that locatebounds(time) builds: half step, boundaryII, full step,
 * viscosity, u=up, boundaryI, then calcprim / coolingh / coolingdmc. */
int w2d_tstep(W2dCtx* ctx, double time, double dt);
/* criteria(nb,...), src/criteria.f90:16-50: the per-leaf maximum relative
 * jump of p and rho.  grad[nb-1] for nb = 1..nbmax (non-leaves get -1). The
 * flags follow on the host: grad >= tol -> refine (level < nlevs), else
 * grad <= tol2 -> coarsen. */
int w2d_criteria(W2dCtx* ctx, double* grad);
/* The admesh flags on the device, for hosts that keep lp on the host but
 * want neither the per-block criteria download nor the flag loops over
 * nbmax.  w2d_set_links mirrors lp(nb,3:8) (first son, son position and
 * the four neighbours) of the listed rows to the device: element (nb,k) of
 * lp is
 * lp[(nb-1)*row_stride + (k-1)*col_stride] (Fortran lp(nbmin:,8) with
 * nbmin = 1: row_stride 1, col_stride = its leading dimension).  rows NULL
 * sends blocks 1..nbmax of the last w2d_set_topology; otherwise the nrows
 * IDs listed (duplicates allowed), e.g. those updatelpup/updatelpdown
 * changed (and the parent whose lp(nb,3) admesh set).  Neighbours must be
 * -1 or block IDs within the pool, lp(nb,3) 0 or the first of four IDs
 * within it. */
int w2d_set_links(W2dCtx* ctx, const int32_t* lp, int row_stride, int col_stride,
                  const int32_t* rows, int nrows);
/* markref (src/markref.f90:23-44 with criteria's flags), critneighup
 * (src/critneighup.f90:19-58) and critneighdown (src/critneighdown.f90:22-48)
 * of one admesh pass (src/admesh.f90:23-105) on the device, from the
 * criteria maxima of the last step and the tree of w2d_set_topology +
 * w2d_set_links.  refine receives the blocks the pass refines in the order
 * admesh visits them (level ascending, then ID); coarsen the first sons
 * (lp(nb,4) = 1) of the families it coarsens, in its order (level
 * descending, then ID).  The effect of the pass's refines on critneighdown
 * (updatelpup runs before it) is accounted for.  The host then applies
 * updatelpup / updatelpdown in list order and calls w2d_refine /
 * w2d_coarse.  *nrefine / *ncoarsen receive the counts; W2D_ERR_ARG if a
 * list is longer than its capacity (the counts are still set). */
int w2d_admesh_flags(W2dCtx* ctx, int32_t* refine, int cap_refine, int* nrefine,
                     int32_t* coarsen, int cap_coarsen, int* ncoarsen);
/* locatebounds (src/locatebounds.f90:29-540) and the fill plans built from
 * its list, on the device, from the tree of w2d_set_topology +
 * w2d_set_links (lp(:,3:8)): the same plans as building innerbounds on the
 * host and passing it to w2d_set_bounds, for hosts that do not need the
 * list themselves.  Queued on the context's stream (no wait). */
int w2d_locate_bounds(W2dCtx* ctx);
/* The u motion of refine (src/refine.f90:30-38, 227-258): quads[k*5+0] is
 * the parent, quads[k*5+1..4] the four sons (BL, BR, TL, TR). */
int w2d_refine(W2dCtx* ctx, const int32_t* quads, int n);
/* The u motion of coarse (src/coarse.f90:29-180): quads[k*5+0] is the new
 * leaf (dad), quads[k*5+1..4] its four sons. */
int w2d_coarse(W2dCtx* ctx, const int32_t* quads, int n);
/* Standalone ghost fills and source terms, each equal to the reference
 * routine applied to the current pool (used by hosts that split tstep). */
int w2d_boundaryI(W2dCtx* ctx, double time);    /* src/boundaryI.f90:4   */
int w2d_boundaryII(W2dCtx* ctx, double time);   /* src/boundaryII.f90:4  */
int w2d_calcprim(W2dCtx* ctx);                  /* src/calcprim.f90:5, every leaf */
int w2d_coolingh(W2dCtx* ctx, double dt_s);     /* src/coolingh.f90:5    */
int w2d_coolingdmc(W2dCtx* ctx, double dt_s);   /* src/coolingdmc.f90:6  */

/* ---- measurement --------------------------------------------------------- */
/* Turns per-kernel CUDA-event timing on (1) or off (0) and resets it. */
int w2d_profile(W2dCtx* ctx, int on);
/* Kernel timing totals since w2d_profile(ctx,1): names[k] (NUL-separated,
 * up to cap bytes), launches[k], total_ms[k]; returns the number of kernels
 * in *nk (at most maxk). */
int w2d_profile_read(W2dCtx* ctx, char* names, int cap, int32_t* launches,
                     double* total_ms, int maxk, int* nk);
/* Number of the library's own kernel launches since creation. */
int w2d_launch_count(W2dCtx* ctx, int64_t* n);
/* Blocks until all queued work of the context is done. */
int w2d_sync(W2dCtx* ctx);
/* Records CUDA event `slot` (0..63) on the context's stream. */
int w2d_event_record(W2dCtx* ctx, int slot);
/* Milliseconds between two recorded events (waits for the later one). */
int w2d_event_elapsed(W2dCtx* ctx, int slot_a, int slot_b, double* ms);
/* Overwrites a scratch buffer larger than the L2 cache on the context's
 * stream, so that the next call starts with a cold L2. */
int w2d_flush_l2(W2dCtx* ctx);

/* ---- allocation-free time step -------------------------------------------
 * No counterpart in the reference.  For hosts that cannot allocate device
 * memory: a Fortran code whose device arrays belong to an OpenACC or
 * OpenMP-offload runtime, or a code whose memory manager forbids
 * cudaMalloc/cudaFree inside its time loop.  Such a host owns its blocks on
 * the device and cannot create a context (w2d_create allocates the pool).
 *
 * Computes what w2d_timestep computes for the nblocks blocks at u (device
 * pointer, block-major [nblocks][neq][20][20], i fastest) whose levels are
 * lev (device pointer, nblocks ints, 1..nlevs); dx, dy are host arrays of
 * nlevs spacings; dt (host) receives the CFL time step.  FP64 only, not for
 * COOLINGDMC.  Nothing is allocated: the per-block partials live in a
 * file-scope device array of W2D_NOALLOC_MAX_BLOCKS doubles that every GPU
 * loading the library keeps until exit; nblocks above that is rejected with
 * W2D_ERR_CAPACITY.  Every call looks up that array's device address
 * (cudaGetSymbolAddress, which allocates nothing) in the caller's current
 * device and context, so a host that resets its device or has its context
 * rebuilt by an offload runtime still gets a valid address; the first call
 * in a context may load the library's device code, so make it before any
 * stream capture.  A block whose level lies outside 1..nlevs makes the call
 * return W2D_ERR_TOPOLOGY (dt untouched).  Cells whose values give NaN are
 * ignored, as w2d_timestep ignores them.  All calls share the array: calls
 * that overlap on the GPU race.  Work is queued on the legacy default
 * stream, which waits for the other blocking streams of the device but not
 * for streams created non-blocking: a host that wrote u or lev on such a
 * stream (an OpenACC async queue, for one) synchronises it first.  The call
 * returns once dt has been copied back. */
#define W2D_NOALLOC_MAX_BLOCKS 65536
#define W2D_MAXLEV_NOALLOC 16
int w2d_timestep_noalloc(const W2dParams* p, const double* u, const int32_t* lev, int nblocks,
                         const double* dx, const double* dy, double* dt);

/* ---- whole-run driver ----------------------------------------------------
 * A C++ restatement of the reference's host side (main.f90 loop, basegrid,
 * admesh, markref, critneighup/down, updatelpup/down, locatebounds) driving
 * the entry points above.  It exists so that the block update can be run and
 * measured without the Fortran host; it makes the same calls a Fortran host
 * would. */
typedef struct W2dInit {
  int32_t kind;          /* W2D_IC_* */
  int32_t init_levels;   /* uniform pre-refinement (1 = roots only)          */
  int32_t startup_admesh;/* admesh passes before the loop (main.f90:60-63)   */
  int32_t pad_;
  double rho0, p0;       /* ambient density and pressure (code units)       */
  double e_dep;          /* energy density in the deposit region            */
  double xc, yc, rb;     /* deposit centre and radius (code units)          */
  double xh0;            /* neutral fraction of the ambient (COOLINGH)       */
  double extra[8];       /* kind-specific (SN: rho_in, vmax, eth_in, rsn)    */
} W2dInit;

#define W2D_IC_SEDOV 0   /* uniform ambient + energy deposit (Sedov blast)  */
#define W2D_IC_SNR   1   /* impose_sn-style remnant, src/sn.f90:19-62       */
#define W2D_IC_JET   2   /* ambient + impose_jet, src/user_mod.f90:39-62     */

typedef struct W2dSim W2dSim;
int w2d_sim_create(const W2dParams* p, const W2dInit* ic, W2dSim** out);
int w2d_sim_destroy(W2dSim* sim);
/* Advances nsteps steps of the main loop: timestep, tstep, admesh. */
int w2d_sim_run(W2dSim* sim, int nsteps);
/* time, last dt, steps taken, nbmax, leaf count, zone-updates so far */
int w2d_sim_status(W2dSim* sim, double* time, double* dt, int64_t* steps,
                   int32_t* nbmax, int32_t* nleaf, int64_t* zone_updates);
/* The context the driver uses (for w2d_get_blocks, w2d_profile ...). */
W2dCtx* w2d_sim_ctx(W2dSim* sim);
/* Host block tree: copies lp (column-major, ld = nblocks), leaf, icoord and
 * the current innerbounds (column-major, ld = *ninternal) when non-NULL. */
int w2d_sim_tree(W2dSim* sim, int32_t* lp, int32_t* leaf, int32_t* icoord,
                 int32_t* innerbounds, int32_t* ninternal);
/* Enables/disables AMR (admesh after each step); on by default if nlevs>1. */
int w2d_sim_set_amr(W2dSim* sim, int on);
/* Where the block tree's per-step integer work runs.  W2D_TREE_DEVICE:
 * admesh takes its flags from w2d_admesh_flags and the fill plans come from
 * w2d_locate_bounds; W2D_TREE_HOST: flags from the w2d_criteria download
 * and the host's loops, plans from the host's locatebounds through
 * w2d_set_bounds.  Both give the same refines, coarsenings and plans, so
 * the same run.  W2D_TREE_AUTO (default): whenever the leaf count has moved
 * by half since the last choice (and at the start), the driver times four
 * steps each way (after one untimed step each) and keeps the faster; the
 * device side wins on large trees, where the host's loops no longer hide
 * behind the half step. */
#define W2D_TREE_HOST   0
#define W2D_TREE_DEVICE 1
#define W2D_TREE_AUTO   2
int w2d_sim_set_tree_mode(W2dSim* sim, int mode);
/* The mode set and the side in use now (1 device, 0 host). */
int w2d_sim_tree_mode(W2dSim* sim, int* mode, int* device);
/* Each half alone (for tests; leaves W2D_TREE_AUTO): the flags (1 device,
 * 0 host) and the plans (1 device, 0 host). */
int w2d_sim_set_device_flags(W2dSim* sim, int on);
int w2d_sim_set_device_plans(W2dSim* sim, int on);
/* DMC table for the driver's context (as w2d_set_cooltab), then the
 * primitives and per-block partials of every leaf are recomputed with it. */
int w2d_sim_set_cooltab(W2dSim* sim, const double* log_t, const double* neg_log_l, int n);
/* Host wall-clock milliseconds spent per phase of w2d_sim_run since the
 * last reset: [0] topology and leaf-list upload, [1] timestep and half-step
 * launches, [2] locatebounds + fill plans (the device meanwhile runs the
 * reduction and the half step), [3] wait for dt, [4] launches of the rest
 * of tstep, [5] the admesh flags from the device (w2d_admesh_flags, or the
 * w2d_criteria download; waits for the device), [6] admesh integer logic,
 * [7] refine/coarse calls, [8] whole steps.  ms must hold W2D_SIM_NPHASES
 * doubles; reset != 0 zeroes the counters after reading. */
#define W2D_SIM_NPHASES 9
int w2d_sim_phase_ms(W2dSim* sim, double* ms, int reset);
/* output(itprint) with OUTBIN, src/output.f90:39-67 (serial build): writes
 * the pointers file (nbmin = 1, nbmax, nbleafs, nblocks, then lp, leaf and
 * icoord of blocks 1..nbmax, column-major 4-byte integers) and the blocks
 * file (u of every leaf in ascending ID in the order of u(nb,:,:,:), 8-byte
 * reals), little-endian streams, from the device pool.  true_value encodes
 * .true. in leaf (-1 as ifort writes it and the reference's py/ reader
 * expects, 1 as gfortran writes it).  An FP32 run writes its state as
 * 8-byte reals. */
int w2d_sim_write_bin(W2dSim* sim, const char* pointers_path, const char* blocks_path,
                      int32_t true_value);
/* Warm start, src/basegrid.f90:167-251 (serial build): replaces the run's
 * tree and leaf blocks with those of the two files (any nonzero leaf value
 * is .true.; the file's nbmax must fit the run's nblocks), recomputes the
 * leaves' primitives, sets the run time to `time` (the reference uses
 * itprint*dtprint) and makes nadmesh admesh passes (src/main.f90:59-62 makes
 * 4).  A COOLINGDMC run needs its table (w2d_sim_set_cooltab) first. */
int w2d_sim_read_bin(W2dSim* sim, const char* pointers_path, const char* blocks_path,
                     double time, int nadmesh);

/* ---- Ensembles (no counterpart in the reference) ---------------------------
 * nruns independent runs of the driver above advanced together on one
 * device: p[r], ic[r] as for w2d_sim_create (physics, precision and method
 * fields equal across runs; root grid, levels, capacity and initial
 * conditions free; no user boundary).  Run r owns the pool slots
 * base+1 .. base+cap (w2d_ens_run_slots) and numbers its blocks 1..cap.
 * One w2d_ens_run step advances every run by one step of its own dt; each
 * run's results equal those of the run alone.  threads: host threads for
 * the per-run integer work (0: one per core). */
typedef struct W2dEns W2dEns;
int w2d_ens_create(const W2dParams* p, const W2dInit* ic, int nruns, int threads, W2dEns** out);
int w2d_ens_destroy(W2dEns* ens);
int w2d_ens_run(W2dEns* ens, int nsteps);
/* as w2d_sim_status for run `run`; run = -1 sums nbmax, leaves and
 * zone-updates over the runs (time and dt 0, steps = ensemble steps) */
int w2d_ens_status(W2dEns* ens, int run, double* time, double* dt, int64_t* steps,
                   int32_t* nbmax, int32_t* nleaf, int64_t* zone_updates);
W2dCtx* w2d_ens_ctx(W2dEns* ens);
int w2d_ens_run_slots(W2dEns* ens, int run, int32_t* base, int32_t* cap);
/* leaf block IDs of a run (ascending, run numbering); ids may be NULL */
int w2d_ens_leaves(W2dEns* ens, int run, int32_t* ids, int32_t* n);
/* w2d_totals of run `run` */
int w2d_ens_totals(W2dEns* ens, int run, double* tot);
/* as w2d_sim_tree (without innerbounds) for run `run`: lp (cap x 8,
 * column-major), leaf (cap) and icoord (cap x 2, column-major) of its host
 * tree, cap its capacity (w2d_ens_run_slots); arrays may be NULL */
int w2d_ens_tree(W2dEns* ens, int run, int32_t* lp, int32_t* leaf, int32_t* icoord);
int w2d_ens_set_amr(W2dEns* ens, int on);
/* Host wall-clock ms per phase of w2d_ens_run: [0] leaf lists, [1] dt and
 * half-step launches with locatebounds + fill plans of the changed runs,
 * [2] launches of the rest of tstep, [3] unused, [4] criteria (waits for
 * the device), [5] admesh integer logic, [6] refine/coarse call, [7] whole
 * steps. */
#define W2D_ENS_NPHASES 8
int w2d_ens_phase_ms(W2dEns* ens, double* ms, int reset);

/* ---- One run partitioned by blocks over several GPUs ---------------------
 * The reference's MPI build (-DMPIP): the leaves split between ranks in
 * contiguous ranges of their Hilbert order (src/loadbalance.f90:5-240), the
 * faces between ranks exchanged inside boundaryII / boundaryI
 * (src/boundaryII.f90:516-1113, src/boundaryI.f90:398-857), dt reduced with
 * mpi_allreduce(min) (src/timestep.f90:52), block data sent across ranks by
 * refine / coarse (src/refine.f90:60-120, src/coarse.f90:200-345).
 *
 * Every rank keeps the whole block tree on the host and a pool of the full
 * capacity on its GPU indexed by global block ID; its context steps only
 * its own leaves.  Before the full step and before boundaryI each rank
 * receives, whole, the neighbour blocks of its leaves that other ranks own
 * (up, then u); dt is the minimum over ranks, the criteria maxima the
 * maximum; refined sons stay with the parent's rank, a coarsened family
 * gathers at its first son's rank; when the largest leaf count exceeds the
 * mean by more than the balance tolerance (default 0.10) the leaves are
 * re-split and moving blocks take their primitives and time-step partials
 * with them.  A partitioned run equals the run on one GPU bit for bit (dt,
 * tree, every interior and edge-ghost value), for any number of ranks.
 *
 * w2d_part_create: rank `rank` of nranks, one process per GPU (the current
 * CUDA device), joined through NCCL (libnccl.so.2, loaded at run time, or
 * the library W2D_NCCL_LIB names) from the 128-byte unique id that one rank
 * obtained with w2d_part_nccl_id and passed to all.  Every wait for the
 * other ranks is bounded (W2D_PART_TIMEOUT_S seconds, default 120): past
 * it the communicator is aborted and the call returns W2D_ERR_TIMEOUT; the
 * run cannot continue after that.  W2D_ERR_STATE: NCCL not found.
 * w2d_part_create_local: all nranks ranks in this process on the current
 * device, blocks moved by device copies between the ranks' buffers, the
 * ranks stepped in lock step -- the same partition, exchanges and results,
 * for checking a partition on one GPU.  The run must keep at least one
 * leaf per rank (W2D_ERR_STATE otherwise). */
typedef struct W2dPart W2dPart;
int w2d_part_nccl_id(uint8_t* id, int bytes);
int w2d_part_create(const W2dParams* p, const W2dInit* ic, int nranks, int rank, const uint8_t* nccl_id,
                    W2dPart** out);
int w2d_part_create_local(const W2dParams* p, const W2dInit* ic, int nranks, W2dPart** out);
int w2d_part_destroy(W2dPart* part);
/* nsteps steps of the main loop (timestep, tstep, admesh) on every rank */
int w2d_part_run(W2dPart* part, int nsteps);
/* as w2d_sim_status for the whole run (zone-updates of all ranks) */
int w2d_part_status(W2dPart* part, double* time, double* dt, int64_t* steps,
                    int32_t* nbmax, int32_t* nleaf, int64_t* zone_updates);
/* ranks of the run, the first rank this object holds and how many;
 * counters[4]: blocks sent as halo, blocks migrated, re-splits, exchanges */
int w2d_part_info(W2dPart* part, int32_t* nranks, int32_t* first_rank, int32_t* nlocal, int64_t* counters);
/* the global tree, as w2d_sim_tree (lp cap x 8 and icoord cap x 2,
 * column-major; leaf cap) */
int w2d_part_tree(W2dPart* part, int32_t* lp, int32_t* leaf, int32_t* icoord);
/* owner[nb - 1]: the rank of leaf nb, -1 for other blocks (cap entries) */
int w2d_part_owner(W2dPart* part, int32_t* owner);
/* u of leaves held by this object's ranks (block-major, as w2d_get_blocks);
 * W2D_ERR_ARG for a non-leaf or a leaf of a rank in another process */
int w2d_part_get_blocks(W2dPart* part, const int32_t* ids, int n, double* u);
int w2d_part_set_balance(W2dPart* part, double tol);
/* w2d_sim_set_cooltab on every rank */
int w2d_part_set_cooltab(W2dPart* part, const double* log_t, const double* neg_log_l, int n);
/* the context of this object's k-th rank (0 .. nlocal-1) */
W2dCtx* w2d_part_ctx(W2dPart* part, int k);
/* The partition rules alone (host only, no device): w2d_part_split gives
 * the Hilbert split of the leaves of a tree (lp, leaf, icoord as
 * w2d_set_topology takes them; nx interior cells per block side) into
 * owner[nb - 1]; w2d_part_halo the halo lists of rank `rank` for an
 * innerbounds list (as w2d_set_bounds takes it) and an owner array:
 * counts[k] blocks to send to rank k, counts[nranks + k] to receive from
 * it, the IDs (ascending per peer) in ids, sends first, *nids in all
 * (ids NULL: counts only). */
int w2d_part_split(const int32_t* lp, int ld_lp, const int32_t* leaf, const int32_t* icoord, int ld_icoord,
                   int nbmax, int nbroot_x, int nbroot_y, int nlevs, int nx, int nranks, int32_t* owner);
int w2d_part_halo(const int32_t* innerbounds, int ld, int n, const int32_t* owner, int nbmax, int rank,
                  int nranks, int32_t* counts, int32_t* ids, int cap_ids, int32_t* nids);

/* ---- Launch shapes and step graphs (no counterpart in the reference) ------
 * The per-leaf kernels (half step, full step, boundaryI, cooling, block
 * statistics) run with one CTA per leaf or on a persistent grid of 2, 4 or
 * 8 CTAs per SM walking the leaves strided or in contiguous chunks.
 * w2d_autotune(ctx, reps) tries every shape for `reps` steps of the live
 * run (results do not depend on the shape) and then keeps the fastest per
 * kernel; w2d_tuning reports, per kernel (half, full, fill I, cooling,
 * statistics), {shape index, CTAs per SM, order} in shape[3k..3k+2], the
 * chosen shape's mean ms and the tuning steps left.  w2d_set_graphs(ctx, 1)
 * makes an ensemble context, or the context of a single run without the
 * jet (w2d_sim_ctx), replay each step's two launch sequences as CUDA
 * graphs (persistent shapes only; leaf count and dt are read on the
 * device, dt reaches the host with the step's synchronization).
 * w2d_set_step_kernel(ctx, 1) lets such a single adiabatic run take each
 * step -- timestep, tstep and the block statistics -- as ONE cooperative
 * persistent kernel whose phases wait on per-block flags instead of kernel
 * boundaries, once the autotuner is done and while the fill plans are
 * current (w2d_sim_set_device_plans); the results equal those of the
 * separate kernels bit for bit.  The default, 0, keeps the separate
 * kernels, which measured faster on the B200 (the FP64 phases are latency
 * bound, and a CTA waiting for its neighbours' flags idles its warps at
 * least as long as a kernel boundary does). */
int w2d_autotune(W2dCtx* ctx, int reps);
int w2d_tuning(W2dCtx* ctx, int32_t* shape, double* ms, int* tuning_left);
int w2d_set_graphs(W2dCtx* ctx, int on);
int w2d_set_step_kernel(W2dCtx* ctx, int fused);

/* ---- Learned coolingh surrogate (no counterpart in the reference) ---------
 * A 4 -> 64 -> 64 -> 2 tanh MLP with BF16 weights on the tensor cores
 * (FP32 accumulation) mapping (log n, log T, neutral fraction, log dt) to
 * the updated (T, neutral fraction) of atomic (src/coolingh.f90:171-259),
 * trained on samples that the exact routine labels on the device.
 * Parameters: a flat FP32 vector of W2D_NN_NPARAM values, W1 [64][4], b1
 * [64], W2 [64][64], b2 [64], W3 [2][64], b3 [2] (row = output unit).
 * Features are columns f[q*n + i] (q = 0..3), targets t[q*n + i] (q = 0, 1);
 * their maps are given in w2d_nn.cuh. */
#define W2D_NN_NPARAM 4610
typedef struct W2dNN W2dNN;
int w2d_nn_create(uint64_t seed, W2dNN** out);   /* Glorot weights from seed */
int w2d_nn_destroy(W2dNN* nn);
/* n training samples drawn with `seed` (n, T, dt log-uniform over [1e-2,
 * 1e4] cm^-3, [1e2, 1e8] K, [1e-2, 1e2] yr; neutral fraction uniform over
 * [1e-4, 1]) and labelled by the exact routine, kept on the device */
int w2d_nn_samples(W2dNN* nn, int64_t n, uint64_t seed);
/* the same for coolingdmc (src/coolingdmc.f90:30-40): T log-uniform over
 * [1e4, 1e8] K, labels from the 41-row table as w2d_set_cooltab takes it
 * and the context's cv, tempsc and psc; the network then serves coolingdmc
 * contexts (it learns the rate per unit density, a function of T) */
int w2d_nn_samples_dmc(W2dNN* nn, int64_t n, uint64_t seed, const double* log_t, const double* neg_log_l,
                       int rows, double cv, double tempsc, double psc);
/* W2D_COOLINGH or W2D_COOLINGDMC: the routine the samples came from */
int w2d_nn_kind(W2dNN* nn);
/* Adam over the samples in batches of `batch` (multiple of 128), learning
 * rate cosine-decayed from lr to lr_end; *last_loss: mean squared error of
 * the last batch */
int w2d_nn_train(W2dNN* nn, int epochs, int batch, float lr, float lr_end, float* last_loss);
int w2d_nn_params(W2dNN* nn, float* params, int set);   /* get (0) / set (1) */
/* loss and gradient of the mean squared error over n host samples */
int w2d_nn_grad(W2dNN* nn, const float* feat, const float* targ, int n, float* grad, float* loss);
int w2d_nn_forward(W2dNN* nn, const float* feat, int n, float* out);   /* out [2][n] */
/* The exact routine judges the surrogate on n fresh samples: [0] share
 * the surrogate serves at the serve tolerance tol (in (0, 0.1]: inputs in
 * range, predicted relative changes of T and of the thermal pressure and
 * predicted change of the neutral fraction within tol, the test of the
 * cooling kernel), [1] median, [2] 99th percentile and [3] maximum
 * relative error of T and [4] mean and [5] maximum error of the neutral
 * fraction over those, [6] share whose exact |dT/T| <= 10%.  stats holds 8
 * doubles.  coolingh networks only: W2D_ERR_STATE for a coolingdmc
 * network. */
int w2d_nn_judge(W2dNN* nn, int64_t n, uint64_t seed, double tol, double* stats);
/* coolingh of an FP32 context (or ensemble context) through the network:
 * cells whose inputs lie outside the training ranges or whose predicted
 * relative change of T or of the thermal pressure, or predicted change of
 * the neutral fraction, exceeds the serve tolerance (below) take the exact
 * routine.  The network must outlive its
 * use by the context; nn = NULL detaches it. */
int w2d_set_surrogate(W2dCtx* ctx, W2dNN* nn);
/* largest predicted relative change of T and of the thermal pressure that
 * the network serves, in (0, 0.1] (default 0.002: cells that change faster
 * are few -- on Sedov-with-coolingh runs the share served falls from 81.4%
 * at 0.01 to 80.8% -- and the exact routine keeps their evolution exact) */
int w2d_set_surrogate_tol(W2dCtx* ctx, double tol);
/* cells served by the network and by the exact routine since creation */
int w2d_surrogate_counts(W2dCtx* ctx, int64_t* served, int64_t* exact);

#ifdef __cplusplus
}
#endif
#endif /* W2D_H */
