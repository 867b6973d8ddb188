// w2d_internal.h -- entry points shared by the C-ABI layer and the
// whole-run driver; not exported through include/w2d.h.
#pragma once

#include "../../include/w2d.h"

// Split of timestep + tstep used by the whole-run driver so that the host
// builds the fill plan while the device runs the time-step reduction and
// the half step.  The sequence
//   ctx_dt_launch, ctx_half_step, (w2d_set_bounds), ctx_dt_wait, ctx_tstep_rest
// computes exactly what w2d_timestep followed by w2d_tstep computes: the
// half step reads the dt that k_dt left in device memory, the host reads
// the same value back before the full step.
int ctx_dt_launch(W2dCtx* c);                           // k_dt; dt and error word copied to pinned memory
int ctx_half_step(W2dCtx* c);                           // k_half, dt from device memory
int ctx_dt_wait(W2dCtx* c, double* dt);                 // waits for the copy, checks the error word
int ctx_tstep_rest(W2dCtx* c, double time, double dt);  // full step, boundaryI, prim/cooling

// The refines (rq, nr quads) and coarsenings (cq, nc quads) of one admesh
// pass in one launch; equal to w2d_refine(rq) followed by w2d_coarse(cq).
int ctx_amr(W2dCtx* c, const int32_t* rq, int nr, const int32_t* cq, int nc);
