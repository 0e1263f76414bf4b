/*
 * pcom_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * C interface of the CPU oracle: an FP64 C++ restatement of PCOM v2.2
 * (ouyuyuan/pcom) setup and baroclinic time step, used by tests/ and by the
 * CPU-baseline leg of bench.py as the checker.  Nothing in the product
 * (pcom_b200/, include/) links, imports or calls it.
 *
 * The input struct mirrors what the reference reads from its netCDF input
 * files (main.f90:252-310, 499-512, 585-599, 675-697; mod_mympi.f90:493-560)
 * for a single-domain run (npx = npy = 1).  All arrays are Fortran order
 * (i fastest) over the GLOBAL interior grid (glo_ni x glo_nj [x nd3]).
 */
#ifndef PCOM_ORACLE_H
#define PCOM_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_inputs {
  int32_t glo_ni, glo_nj, nk;
  int32_t dtbt, dtbc;          /* namelist dtbt, dtbc (s) */
  int32_t r8;                  /* 0: gfortran default-real literals (REAL*4), 1: ifort -r8 */
  int32_t rst;                 /* namelist restart_run (only 0 is set up here) */
  int32_t year, month, day, hour; /* namelist bdate */
  const double *lon;           /* glo_ni, grid 4 longitude (deg) */
  const double *lat;           /* glo_nj, grid 4 latitude (deg) */
  const double *z;             /* nk, layer-centre depth (m) */
  const double *tmn, *smn;     /* nk, mean T/S profile */
  const int32_t *itn;          /* glo_ni*glo_nj, number of wet levels */
  const double *pt, *sa;       /* glo_ni*glo_nj*nk, initial T/S */
  const double *taux, *tauy, *bct, *bcs, *pa, *fw; /* glo_ni*glo_nj*12 monthly forcing */
  const double *vmix;          /* glo_ni*glo_nj*nk vertical mixing (cm^2/s) or NULL (all missing) */
} orc_inputs;

void *orc_create(const orc_inputs *in);
void orc_destroy(void *m);
/* one pass of the body of the time loop of main.f90:158-238 (without output) */
void orc_step(void *m);
/* individual pieces, for bisection: 0 int_bnd, 1 den_prho, 2 den_alpha,
 * 3 int_pgra, 4 int_readyc, 5 int_trop, 6 int_clin, 7 int_ssh, 8 int_ts,
 * 9 calendar advance (tctr%pt = tctr%ct; tctr%ct = ct + dtbc) */
void orc_phase(void *m, int phase);
/* set tctr%i explicitly (the step counter used by the AB3 start-up) */
void orc_set_iter(void *m, int64_t i);
int64_t orc_get_iter(void *m);
/* pointer to a named internal array and its shape (n1, n2, n3; AoS pairs are
 * exposed as two separate arrays: e.g. "prho1", "prho2").  NULL if unknown. */
double *orc_field(void *m, const char *name, int32_t *n1, int32_t *n2, int32_t *n3);
int32_t *orc_ifield(void *m, const char *name, int32_t *n1, int32_t *n2, int32_t *n3);
/* the scalar constants of mod_con.f90 as the oracle evaluated them */
double orc_const(void *m, const char *name);
/* den_rho of mod_den.f90:57-118 for a single point */
double orc_den_rho(double t, double s, double p0, int32_t r8);
void orc_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
