/*
 * pcom_host.h -- host driver of the B200 PCOM time step.
 *
 * The reference's driver is main.f90: it reads the grid, initial state and
 * forcing (init/set_cf/calc_hpos/set_hgrid/set_vgrid/set_grid/calc_cf/inistat,
 * main.f90:252-704), then runs the time loop of main.f90:158-238 (daily
 * int_bnd + den_prho, then the per-step call block).  Its Fortran compiler is
 * not available here, so this C++ driver stands in for it: it does
 * the same setup on the host, uploads the result through include/pcom_gpu.h
 * and drives the same loop.  A Fortran driver that keeps main.f90 calls
 * pcom_gpu.h directly instead, through the interface module
 * include/pcom_gpu.f90.
 *
 * pcom_case mirrors what the reference reads from its input files for a
 * single-domain run: global interior arrays, Fortran order (i fastest).
 */
#ifndef PCOM_HOST_H
#define PCOM_HOST_H
#include <stdint.h>
#include "pcom_gpu.h"
#ifdef __cplusplus
extern "C" {
#endif

typedef struct pcom_case {
  int32_t glo_ni, glo_nj, nk;
  int32_t dtbt, dtbc;             /* namelist time_ctrl dtbt, dtbc */
  int32_t r8;                     /* 1: literals as REAL(8) (ifort -r8) */
  int32_t rst;                    /* namelist restart_run: 1 = the caller loads a restart state after create */
  int32_t year, month, day, hour; /* namelist bdate */
  const double *lon, *lat, *z, *tmn, *smn; /* initial.nc: lon (glo_ni), lat (glo_nj), z/tmn/smn (nk) */
  const int32_t *itn;                      /* initial.nc itn: glo_ni*glo_nj */
  const double *pt, *sa;                   /* initial.nc pt, sa: glo_ni*glo_nj*nk */
  const double *taux, *tauy, *bct, *bcs, *pa, *fw; /* forcing.nc: glo_ni*glo_nj*12 */
  const double *vmix;                      /* vmix.nc (cm^2/s) glo_ni*glo_nj*nk, or NULL = all missing */
} pcom_case;

typedef struct pcom_model pcom_model;

/* pcom_model_create flag: do the host setup only, create no device handle
 * (for checking the setup on a machine without a GPU). */
#define PCOM_MODEL_HOST_ONLY 0x100

/* Setup (main.f90:86-150) and the GPU handle with static data and initial
 * state uploaded.  flags: PCOM_PREC_* (PCOM_LIT_R8 is taken from case->r8). */
int pcom_model_create(const pcom_case *c, int32_t flags, pcom_model **out);
int pcom_model_destroy(pcom_model *m);
pcom_handle *pcom_model_handle(pcom_model *m);
/* n passes of the time loop body (main.f90:158-238, without output()). */
int pcom_model_run(pcom_model *m, int64_t nsteps);
/* One pass split open, for drivers that put their own work between the
 * subroutines of the step (the halo exchanges of a domain split into row
 * slabs): begin_step advances tctr%i (returned in *it) and on a new model
 * day runs int_bnd and den_prho (main.f90:158-201; *new_day = 1); the caller
 * then runs pcom_gpu_phase 0..6 with that counter and calls end_step, which
 * advances the calendar (main.f90:231-232).  pcom_model_run is exactly
 * begin_step, pcom_gpu_step, end_step. */
int pcom_model_begin_step(pcom_model *m, int64_t *it, int32_t *new_day);
int pcom_model_end_step(pcom_model *m);
/* n passes of the time loop for n models stepped together through batch b
 * (pcom_gpu_batch_create on their handles, in the same order).  The models
 * must be at the same iteration and date (same bdate and dtbc): forcing
 * (int_bnd) is interpolated per model on day changes, then den_prho and the
 * step run batched.  No counterpart in the reference. */
int pcom_model_run_batch(pcom_model *const *ms, int32_t n, pcom_batch *b, int64_t nsteps);
/* tctr%i of the last completed step, and the model date tctr%ct. */
int64_t pcom_model_iter(pcom_model *m);
int pcom_model_date(pcom_model *m, int32_t *ymdh4);
/* Host copies of the static grid data the driver computed (pointers stay
 * owned by the model); for checks against another implementation. */
int pcom_model_static(pcom_model *m, pcom_static *out);
/* int_bnd (mod_int.f90:649-691) for the current model date into host arrays
 * of ni*nj each (any may be NULL). */
int pcom_model_int_bnd(pcom_model *m, double *taux, double *tauy, double *t, double *s, double *pa, double *fw);
/* The initial state the driver set up (inistat), into host arrays. */
int pcom_model_initial_state(pcom_model *m, pcom_state *out);

#ifdef __cplusplus
}
#endif
#endif
