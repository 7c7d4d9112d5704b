/*
 * ramses_hydro_batch.h — many independent hydro solves on one B200.
 *
 * No counterpart in the reference (RAMSES II advances one mesh per run).  A
 * batch holds uniform-grid problems of uneven sizes resident in one device
 * pool; one batch step advances every unfinished problem by one Godunov step
 * with its own CFL dt, in ONE persistent kernel launch whose CTAs pull
 * (problem, pencil) work items from an atomic counter, followed by one
 * per-problem reduction (new dt, time, conserved totals).  Steps are replayed
 * from a captured CUDA graph.  The step is the same algorithm as rh_godunov
 * (hydro/umuscl.f90 unsplit + courant_fine); problems are stored in the
 * reference's per-oct layout with octs in row-major order.
 */
#ifndef RAMSES_HYDRO_BATCH_H
#define RAMSES_HYDRO_BATCH_H

#include "ramses_hydro.h"

#ifdef __cplusplus
extern "C" {
#endif

/* One problem: a uniform box of n[0] x n[1] x n[2] cells (even, multiples of
 * 2); ndim = 3, or 2 for a plane problem embedded as one z oct layer with
 * periodic z (the CFL counts ndim directions, as cmpdt does). */
typedef struct rh_batch_problem {
    int32_t n[3];
    int32_t ndim;
    int32_t bound_type[6];   /* x-,x+,y-,y+,z-,z+: RH_BOUND_*                 */
    double  dx;              /* cell size                                      */
    double  gamma, smallr, smallc, courant_factor;
    double  t_end;           /* the problem is done at t >= t_end (> 0)       */
    int32_t max_steps;       /* ... or after max_steps steps (0: no limit)    */
} rh_batch_problem;

/* Initial state, built on the device. */
#define RH_IC_SPLIT 1   /* two primitive states split at the middle of axis      */
#define RH_IC_BLAST 2   /* uniform (rho, p) plus pressure p_in within radius     */
#define RH_IC_HOST  3   /* copied from host: uold(1:8,1:5,1:noct), row-major octs */
typedef struct rh_batch_ic {
    int32_t kind;
    int32_t axis;            /* RH_IC_SPLIT: 0,1,2                              */
    double  left[5];         /* RH_IC_SPLIT: rho,u,v,w,p for x_axis < half      */
    double  right[5];
    double  ambient[5];      /* RH_IC_BLAST: rho,u,v,w,p outside the blast      */
    double  p_in;            /* RH_IC_BLAST: pressure inside                    */
    double  radius;          /* RH_IC_BLAST: radius (length units)              */
    double  centre[3];
    const double* host_uold; /* RH_IC_HOST                                      */
} rh_batch_ic;

/* Create the batch: precision mode, slope type (0-2), Riemann solver, and a
 * pool able to hold pool_octs octs (both time levels).  One batch per process. */
int rh_batch_init(int precision, int slope, int riemann, long long pool_octs);
int rh_batch_free(void);
/* Device bytes a problem occupies in the pool (both time levels). */
long long rh_batch_footprint(const rh_batch_problem* p);
/* Add a problem; RH_ENOMEM when the pool has no room (the caller queues it). */
int rh_batch_add(const rh_batch_problem* p, const rh_batch_ic* ic, int* id);
/* Remove a problem and release its pool space. */
int rh_batch_remove(int id);
/* Advance every unfinished problem by nsteps steps (graph replays). */
int rh_batch_step(int nsteps);
/* Per-problem state: time, steps taken, done flag (0 running, 1 finished,
 * 2 stopped by the state check), current dt and the courant_fine totals
 * (mass, ekin, eint, emag, dt) of the current state. */
int rh_batch_status(int id, double* t, int* nstep, int* done, double* dt, double* totals5);
/* Status of every problem slot at once (arrays of rh_batch_capacity()). */
int rh_batch_poll(int* done, int* nstep, double* t);
int rh_batch_capacity(void);
/* Copy a problem's current state to the host, reference layout, row-major octs. */
int rh_batch_fetch(int id, double* host_uold);
/* Tile of the batch kernel (one of the compiled shapes rh_batch_list_tiles
 * returns; lz = oct layers per pencil).  rh_batch_init starts from 7x7 octs,
 * 2 CTAs per SM, 32 layers (FP32-bulk) or 8x4 / 2 / 32 (FP64). */
int rh_batch_set_tile(int txo, int tyo, int minb, int lz);
/* Compiled batch-kernel shapes of a precision: writes up to max entries,
 * returns how many exist. */
int rh_batch_list_tiles(int precision, int* txo, int* tyo, int* minb, int max);
/* Device time of nsteps batch steps (CUDA events), milliseconds per step. */
int rh_batch_bench(int nsteps, float* ms_per_step);
/* Cells updated by one batch step over the unfinished problems. */
long long rh_batch_cells(void);
/* Kernel path of 2D problems (ndim 2: one z oct layer, periodic z): 1 (the
 * default) the plane tile body, which does the x/y work once per cell and
 * writes both planes; 0 the 3D pencil body.  Both give the same result bit for
 * bit (the pencil body's z terms are exact zeros there); the choice is kept for
 * that comparison. */
int rh_batch_set_plane_path(int on);
/* on != 0: after each step every stepped problem's new state is checked as
 * rh_check_state checks a level (NaN/Inf, density <= 0, internal energy <= 0;
 * gpu/gpu_utils.cuf:90-118, hydro/godunov_utils.f90:278-287), and a problem
 * with a bad cell is stopped with done = 2 (the others go on).  Off by
 * default: one extra read of the stepped states per step. */
int rh_batch_set_state_check(int on);
/* The check's bits of a problem (1 NaN/Inf, 2 rho <= 0, 4 eint <= 0), 0 if clean. */
int rh_batch_check_mask(int id, int* mask);

#ifdef __cplusplus
}
#endif
#endif /* RAMSES_HYDRO_BATCH_H */
