/*
 * pcom_gpu.h -- C ABI of the B200 (sm_100a) implementation of the PCOM v2.2
 * baroclinic time step (ouyuyuan/pcom).
 *
 * The reference has no plugin/FFI layer: its hot path is the per-step call
 * block of main.f90:205-223 (den_alpha, int_pgra, int_readyc, int_trop,
 * int_clin, int_ssh, int_ts) plus the daily den_prho (main.f90:179,200),
 * operating on module-global arrays (mod_arrays.f90:28-122).  This header is
 * the drop-in boundary for that block: a Fortran driver binds it with
 * ISO_C_BINDING (the interface module include/pcom_gpu.f90) and keeps its own
 * setup, calendar, namelist and netCDF I/O.
 *
 * Conventions
 *  - Every array is a plain host pointer in Fortran order (i fastest) over the
 *    padded local domain ni x nj [x nk | x nkp], ni = glo_ni + 2, nj = glo_nj + 2
 *    (mod_param.f90:332-342 with npx = npy = 1).  type_mat arrays are AoS
 *    pairs (x(1), x(2)) per point (mod_type.f90:75-77).
 *  - Every function returns 0 on success or a PCOM_ERR_* code; the message of
 *    the last error is available from pcom_gpu_last_error().  Nothing here
 *    calls exit(): the Fortran side turns a nonzero status into `stop`, as the
 *    reference does for its own errors (mod_io.f90:546-549).
 *  - One handle = one model domain = one CUDA stream.  Calls are synchronous
 *    at return unless the name says _async.
 */
#ifndef PCOM_GPU_H
#define PCOM_GPU_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define PCOM_OK 0
#define PCOM_ERR_ARG 1      /* bad argument, size or inconsistent static data */
#define PCOM_ERR_CUDA 2     /* a CUDA runtime call failed */
#define PCOM_ERR_STATE 3    /* call out of order (e.g. step before upload_static) */
#define PCOM_ERR_NUMERIC 4  /* the NaN/Inf watchdog tripped */
#define PCOM_ERR_TIMEOUT 5  /* a bounded device-side wait gave up */

/* pcom_dims.flags */
#define PCOM_PREC_FP64 0x0   /* FP64 everywhere: the reference's arithmetic */
/* Mixed: the 3-D fields are stored as FP32 and the advection, friction,
 * diffusion, upwelling and Smagorinsky stencils compute in FP32; alpha and
 * adp are stored as anomalies from a reference profile (fixed from the level
 * means of the first T/S given to pcom_gpu_set_state); the barotropic
 * subcycle computes velocities, fluxes and divergence in FP32 while the
 * bottom pressure ch, its gradients and its ch/mch/mch2 accumulation stay
 * FP64, as do the baroclinic pressure-gradient and AB3 updates, the tracer
 * update and the global sums.  The ABI keeps
 * FP64 host arrays: the library converts on upload and download.  No
 * counterpart in the reference. */
#define PCOM_PREC_MIXED 0x1
#define PCOM_LIT_R8 0x10     /* default-REAL literals read as REAL(8) (ifort -r8);
                                otherwise REAL(4) as gfortran compiles them */

typedef struct pcom_handle pcom_handle;

/* Sizes and time steps.  Replaces the dimension/namelist globals of
 * mod_param.f90:40-81 (glo_ni, glo_nj, nk, ni, nj, nm%bt, nm%bc, nm%rst). */
typedef struct pcom_dims {
  int32_t glo_ni, glo_nj, nk;
  int32_t ni, nj;          /* must equal glo_ni + 2, glo_nj + 2 */
  int32_t dtbt, dtbc;      /* barotropic / baroclinic step (s) */
  int32_t flags;           /* PCOM_PREC_* | PCOM_LIT_R8 */
  int32_t rst;             /* nm%rst: 1 = restart run (skips the AB3 start-up) */
  int32_t reserved[3];
} pcom_dims;

/* Static grid data, uploaded once (main.f90:105-122 computes it).
 * rh[g], tn[g]: ni*nj, dx[g]: AoS ni*nj*2 for g = grid 1..4 (type_gi,
 * mod_type.f90:97-108), in the order g1j, g2j, g3j, g4j.
 * z1/pr1/dz1/dpr1: nkp (gi1); z2/pr2/dz2/dpr2: nk (gi2) (type_gj).
 * msk_t, msk_u: ni*nj*nk int32; lev_t, lev_u: ni*nj int32; phih and prh:
 * ni*nj; suffix _t = T grid (g12), _u = U grid (g32) (type_gij).  cv1, cv2, cor, graphihx,
 * graphihy: ni*nj (U grid).  km, kh: ni*nj*nkp. */
typedef struct pcom_static {
  const double *rh[4], *tn[4], *dx[4];
  const double *z1, *pr1, *dz1, *dpr1;
  const double *z2, *pr2, *dz2, *dpr2;
  const int32_t *msk_t, *lev_t, *msk_u, *lev_u;
  const double *phih_t, *prh_t, *phih_u, *prh_u;
  const double *cv1, *cv2, *cor;
  const double *km, *kh;
  const double *graphihx, *graphihy;
} pcom_static;

/* Prognostic and carried state (mod_arrays.f90:80-116).  Any pointer may be
 * NULL to skip that field.  3D fields are ni*nj*nk except wm (ni*nj*nkp) and
 * prho (AoS ni*nj*nk*2).  chc..mch2 are the four levels of `ch`
 * (mod_arrays.f90:433-436). */
typedef struct pcom_state {
  double *tc, *sc, *tp, *sp;
  double *uc, *vc, *up, *vp;
  double *auc, *aup, *aupp, *avc, *avp, *avpp;
  double *ubc, *vbc, *ubp, *vbp;
  double *chc, *chp, *mch, *mch2;
  double *am;
  double *prho;
  double *alpha, *adp;
  double *wm;
} pcom_state;

/* Daily surface forcing after int_bnd (mod_int.f90:649-691), ni*nj each. */
typedef struct pcom_forcing {
  const double *taux, *tauy, *t, *s, *pa, *fw;
} pcom_forcing;

/* Time-mean accumulators and their record counters (eqts%act/acs/acr,
 * equv%acu/acv, eqw%acw, eqch%acch, acssh; mod_type.f90:155-205). */
typedef struct pcom_accum {
  double *act, *acs, *acr, *acu, *acv, *acw;
  double *acch, *acssh;
  int32_t n_ts, n_uv, n_w, n_ch, n_ssh;
} pcom_accum;

/* --- lifetime ------------------------------------------------------------ */
/* Replaces arrays_allocate (mod_arrays.f90:142-352) for the device mirrors. */
int pcom_gpu_create(const pcom_dims *dims, pcom_handle **out);
int pcom_gpu_destroy(pcom_handle *h);

/* --- data movement ------------------------------------------------------- */
/* Grid data computed by set_hgrid/set_vgrid/set_grid/calc_cf/inistat
 * (main.f90:408-704).  Masks must be the ones set_grid builds
 * (msk = lev >= k); any other mask is rejected with PCOM_ERR_ARG. */
int pcom_gpu_upload_static(pcom_handle *h, const pcom_static *s);
/* State in/out: at start-up (inistat, main.f90:675-704), restart read
 * (input_rst, mod_mympi.f90:460-478) and restart write (merge_out_rst,
 * mod_mympi.f90:133-176). */
int pcom_gpu_set_state(pcom_handle *h, const pcom_state *s);
int pcom_gpu_get_state(pcom_handle *h, pcom_state *s);
/* bnd%* after int_bnd or the 6-hourly file reads (main.f90:164-201). */
int pcom_gpu_set_forcing(pcom_handle *h, const pcom_forcing *f);
/* Asynchronous host transfers (no counterpart in the reference), for a
 * driver that overlaps its I/O with the steps:
 * pcom_gpu_set_forcing_async stages taux, tauy, t, s and pa (all five
 * required; fw is not used by the step) in a second set of device forcing
 * fields on the handle's upload stream and returns; the next step (or phase,
 * pcom_gpu_set_forcing, pcom_gpu_int_bnd) switches to the staged set after
 * the upload.  pcom_gpu_get_state_async snapshots the requested fields on
 * the handle's stream after the work enqueued so far and copies the
 * snapshots to the host buffers on the download stream, overlapping the
 * next steps.  Host buffers must stay valid and untouched until pcom_gpu_sync
 * (or any synchronous call) returns; pinned host memory makes the copies
 * asynchronous. */
int pcom_gpu_set_forcing_async(pcom_handle *h, const pcom_forcing *f);
int pcom_gpu_get_state_async(pcom_handle *h, pcom_state *s);
/* Accumulators for output() (main.f90:726-760) and their reset. */
int pcom_gpu_get_accum(pcom_handle *h, pcom_accum *a);
int pcom_gpu_reset_accum(pcom_handle *h);

/* --- compute ------------------------------------------------------------- */
/* den_prho (mod_den.f90:120-153): daily density derivatives. */
int pcom_gpu_den_prho(pcom_handle *h);
/* One baroclinic step: main.f90:205-223 in order.  tctr_i is tctr%i, the
 * 1-based step counter that drives the AB3 start-up (mod_int.f90:122-132). */
int pcom_gpu_step(pcom_handle *h, int64_t tctr_i);
/* The same, enqueued on the handle's stream without waiting. */
int pcom_gpu_step_async(pcom_handle *h, int64_t tctr_i);
/* One subroutine of the step, for bisection against a CPU run:
 * 0 den_alpha (main.f90:205), 1 int_pgra, 2 int_readyc, 3 int_trop,
 * 4 int_clin, 5 int_ssh, 6 int_ts (mod_int.f90:64-507). */
int pcom_gpu_phase(pcom_handle *h, int32_t phase, int64_t tctr_i);

/* --- diagnostics --------------------------------------------------------- */
/* Copy a named device array (state, intermediate or static) to host.
 * n is the capacity of `host` in doubles; returns PCOM_ERR_ARG if too small
 * or unknown.  Names: the pcom_state/pcom_accum members plus fx, fy, pax,
 * pay, ut, vt, bphi_xn/xs/ye/yw, bgraphi_xn/xs/ye/yw. */
int pcom_gpu_get_field(pcom_handle *h, const char *name, double *host, int64_t n);
/* Element count of a named array (0 if unknown). */
int64_t pcom_gpu_field_size(pcom_handle *h, const char *name);
/* Device address of a named array (the current buffer: the AB3 history and
 * the T/S pool rotate between steps, so ask again after each step), its
 * element count and element size (8, or 4 for a 3-D field of a mixed
 * handle).  For drivers that move parts of device arrays themselves, e.g.
 * the halo rows of a domain split into row slabs.  No counterpart in the
 * reference. */
int pcom_gpu_field_ptr(pcom_handle *h, const char *name, void **dev, int64_t *count, int32_t *elem_bytes);
/* Split the domain into row slabs (mod_param.f90:279-344 with npx = 1): the
 * step's 3-D kernels and den_prho compute only rows j_lo..j_hi (padded
 * 1-based index, within 1..nj; default 1..nj); the 2-D prep kernels and the
 * barotropic subcycle still cover every row.  Every kernel keeps global row
 * indexing, so a slab's rows come out exactly as in the whole-domain run
 * once the driver has supplied the rows they read outside the slab (the
 * halo rows of the 3-D fields and the other slabs' rows of the 2-D fields
 * the barotropic subcycle reads; pcom_b200/decomp.py does this with
 * torch.distributed).  Replaces the reference's y decomposition and its
 * halo exchange (mod_mympi.f90:669-861). */
int pcom_gpu_set_rows(pcom_handle *h, int32_t j_lo, int32_t j_hi);
/* Run the NaN/Inf watchdog over the prognostic fields; PCOM_ERR_NUMERIC if
 * any wet point is not finite. */
int pcom_gpu_check_finite(pcom_handle *h);
/* Daily forcing on the device (int_bnd, mod_int.f90:649-691): upload the 12
 * monthly fields once (each pointer: 12 x ni x nj doubles, month slowest,
 * the layout of frc%*%v; fw is not used by the step and may be NULL), then
 * per model day bnd = (frc(m2) - frc(m1)) f + frc(m1) with the months and
 * weight int_bnd computes from the calendar.  Replaces the daily host
 * int_bnd + pcom_gpu_set_forcing upload. */
int pcom_gpu_set_forcing_months(pcom_handle *h, const pcom_forcing *months);
int pcom_gpu_int_bnd(pcom_handle *h, int32_t m1, int32_t m2, double f);
/* Barotropic kernel choice: 0 automatic (resident when the domain's tiles
 * fit one per CTA, else multi-tile), 1 resident (one region point per
 * thread, coefficients in registers), 2 multi-tile (several tiles per CTA),
 * 3 generic (non-separable metrics).  All give the same results; the choice
 * is for tuning and tests.  No counterpart in the reference. */
int pcom_gpu_set_trop_kernel(pcom_handle *h, int32_t which);
/* Concurrent phases in pcom_gpu_step (on by default): int_readyc's 2-D prep
 * and upwelling run beside den_alpha and int_pgra, and smag beside int_ssh
 * and int_ts, on a second stream of the handle forked from and joined back
 * to the handle's stream by events within each step.  Results are the same
 * either way; 0 issues every launch on the handle's stream in phase order.
 * pcom_gpu_phase always runs serially.  No counterpart in the reference. */
int pcom_gpu_set_overlap(pcom_handle *h, int32_t enable);
/* Longest a device-side wait (a grid barrier of the barotropic kernels) may
 * take before the kernel gives up, returns early and the next synchronising
 * call reports PCOM_ERR_TIMEOUT (default 2 s; the barriers normally take
 * microseconds).  The handle stays usable after a timeout: its barrier
 * counters are reset, the state of the interrupted step is not meaningful.
 * No counterpart in the reference. */
int pcom_gpu_set_wait_limit(pcom_handle *h, double seconds);
/* Global sums over the wet T cells of the interior: out3[0] = volume (m^3),
 * out3[1] = sum of T dV (K m^3), out3[2] = sum of S dV (psu m^3), with
 * dV = a^2 rh1 dx1x dx1y dz(k); FP64, in a fixed reduction order.  No
 * counterpart in the reference. */
int pcom_gpu_global_sums(pcom_handle *h, double *out3);

/* --- streams and timing -------------------------------------------------- */
/* Use an external CUDA stream (cudaStream_t as void*) for all work. */
int pcom_gpu_set_stream(pcom_handle *h, void *stream);
int pcom_gpu_sync(pcom_handle *h);
/* Latency floor of the barotropic subcycle: one launch of the resident FP64
 * kernel's synchronisation skeleton.  It has the same grid, block and
 * shared memory, and per substep the same ring reload, the seven CTA
 * barriers, the interior stores and the grid barrier, without the
 * arithmetic.  Its device time in milliseconds for the handle's nstep
 * substeps goes to *ms (CUDA events; the call synchronises the handle's
 * stream).  The model state is unchanged: the skeleton writes only the
 * subcycle's scratch buffers.  PCOM_ERR_STATE unless the handle runs the
 * resident FP64 kernel.  No counterpart in the reference. */
int pcom_gpu_trop_floor(pcom_handle *h, double *ms);
/* Per-kernel device timing with CUDA events (off by default).  When on,
 * pcom_gpu_profile_read fills up to `cap` entries of names (64 chars each),
 * launch counts and total milliseconds and returns the entry count. */
int pcom_gpu_profile(pcom_handle *h, int32_t enable);
int pcom_gpu_profile_read(pcom_handle *h, char *names, int64_t *launches, double *ms, int32_t cap);
/* Number of this library's kernel launches issued so far on this handle. */
int64_t pcom_gpu_launch_count(pcom_handle *h);

/* --- closure coupling ----------------------------------------------------- */
/* No counterpart in the reference.  Data and corrections for the learned
 * subgrid closure (include/pcom_cnn.h) on FP64 handles. */
typedef struct {
  float in_mean[5], in_std[5];  /* u, v, T, S, alpha - alpha_ref(k) */
  float out_std[4];             /* du, dv, dT, dS tendency scales (0: output unused) */
  float out_gain[4];            /* applied fraction per output (pcom_gpu_cnn_apply) */
  float out_clip;               /* |y| limit in units of out_std (0: none) */
  double alpha_ref[64];         /* [k - 1], k = 1..nk */
} pcom_cnn_stats;
/* Set the coarse handle's state to the block means (factor x factor) of the
 * fine handle's state over wet fine cells: T-grid fields (tc, sc, tp, sp,
 * ch, mch, mch2) on T cells, U-grid fields (uc, vc, up, vp, the AB3
 * history, am, ub, vb) on U points, velocities and their history set to 0
 * where the coarse U point is land.  The grids must nest: fine glo_ni,
 * glo_nj = factor x coarse, and the coarse levels no deeper than any fine
 * column of their block. */
int pcom_gpu_coarsen(pcom_handle *fine, pcom_handle *coarse, int32_t factor);
/* Network input from the state: BF16 [nk][glo_nj][glo_ni][16] (device),
 * channels (uc, vc, tc, sc, alpha - alpha_ref) normalised by `stats`, zero
 * on land and in channels 5..15.  x_bf16 must be 16-byte aligned
 * (PCOM_ERR_ARG otherwise). */
int pcom_gpu_cnn_features(pcom_handle *h, void *x_bf16, const pcom_cnn_stats *stats);
/* Training target: (truth - pred) / dt / out_std per channel into FP32
 * [nk][glo_nj][glo_ni][4] (device), and the wet mask (U points for u, v, T
 * cells for T, S) into `mask` of the same shape (either may be NULL). */
int pcom_gpu_cnn_target(pcom_handle *pred, pcom_handle *truth, float *target, float *mask, const pcom_cnn_stats *stats,
                        double dt);
/* Apply the network's output y (FP32 [nk][glo_nj][glo_ni][4], device) as a
 * tendency over dt seconds: uc, up += dt out_gain[0] out_std[0] y0 (wet U
 * points, y clipped to +-out_clip when out_clip > 0), vc, vp likewise, tc,
 * tp, sc, sp on wet T cells.  y must be 16-byte aligned (PCOM_ERR_ARG
 * otherwise). */
int pcom_gpu_cnn_apply(pcom_handle *h, const float *y, const pcom_cnn_stats *stats, double dt);

/* --- batches -------------------------------------------------------------- */
/* No counterpart in the reference (it runs one domain per MPI job).  A batch
 * steps several handles together -- ensemble members and basins of uneven
 * size that share dtbt and dtbc -- with every kernel of the step launched
 * once for all members and the barotropic subcycles of all members in one
 * persistent cooperative launch over the work list of their tiles.  After the
 * two AB3 start-up steps the whole batched step is replayed from a captured
 * CUDA graph.  Members must be advanced only through the batch (their ring
 * buffers rotate in lock step); each member's handle still serves its state,
 * fields and accumulators. */
typedef struct pcom_batch pcom_batch;
int pcom_gpu_batch_create(pcom_handle *const *members, int32_t n, pcom_batch **out);
int pcom_gpu_batch_destroy(pcom_batch *b);
/* One baroclinic step of every member (main.f90:205-223), tctr_i as in pcom_gpu_step. */
int pcom_gpu_batch_step(pcom_batch *b, int64_t tctr_i);
int pcom_gpu_batch_step_async(pcom_batch *b, int64_t tctr_i);
/* Wait for the batch's enqueued work (on the first member's stream) and
 * report a barrier timeout; call it before reading a member after
 * pcom_gpu_batch_step_async. */
int pcom_gpu_batch_sync(pcom_batch *b);
/* den_prho of every member (mod_den.f90:120-153). */
int pcom_gpu_batch_den_prho(pcom_batch *b);
/* Replay captured CUDA graphs (default on) or launch kernel by kernel. */
int pcom_gpu_batch_use_graphs(pcom_batch *b, int32_t enable);
/* Time candidate tile shapes of the batched barotropic kernel on the
 * members' current state (which it saves and restores) and keep the fastest;
 * a one-line report of the trials goes to `report`. */
int pcom_gpu_batch_autotune(pcom_batch *b, char *report, int32_t len);
/* Set the barotropic tile shape by hand (tx, ty >= 1, (tx+4)*(ty+4) <= 640)
 * and optionally cap the tiles of one co-resident group (max_resident > 0;
 * members with more tiles use the multi-tile kernel).  0 = no cap. */
int pcom_gpu_batch_set_tiles(pcom_batch *b, int32_t tx, int32_t ty, int32_t max_resident);
/* Kernels the batch has launched (graph replays included). */
int64_t pcom_gpu_batch_launch_count(pcom_batch *b);

/* --- allocation-free barotropic subcycle -------------------------------- */
/* No counterpart in the reference.  One int_trop subcycle (the resident
 * barotropic kernel: the arithmetic of pcom_gpu_step's int_trop, with IEEE
 * divisions) over arrays the caller owns, for callers that cannot let the
 * library allocate device memory: host frameworks that own every byte of
 * the GPU and hand it out from their own pool (a coupled-model driver that
 * sizes one pool for all its components at start-up, a serving stack whose
 * caching allocator holds the device), where a cudaMalloc inside the library
 * would fail or break the framework's memory budget.  All pointers are device
 * pointers in Fortran order; FP64 fields are ni*nj (lev_* int32).  The
 * metrics are given as separate components (dxx = dx%x(1), dxy = dx%x(2)) of
 * grids 1..4.  am1 is am(:,:,1).
 * The scratch this needs (halo ping-pong buffers, 1-D metric copies and the
 * grid-barrier words, about 3.2 MB) is a fixed array inside the library that
 * every GPU which loads the library holds until the process exits; it is
 * sized for ni*nj <= PCOM_NOALLOC_MAX_POINTS and ni, nj <= PCOM_NOALLOC_MAX_DIM
 * (the 1-degree 362 x 162 domain fits); larger domains are rejected with
 * PCOM_ERR_ARG.  The first call on a device (per CUDA context) looks up that
 * array's device address, so make it before any stream capture.  The call
 * clears the array's barrier and flag words itself; everything else in it is
 * overwritten before use.  Calls share the array: calls that overlap on the
 * GPU race.  The call waits on `stream` and returns once the subcycle has
 * finished. */
#define PCOM_NOALLOC_MAX_POINTS 65536
#define PCOM_NOALLOC_MAX_DIM 1024
typedef struct pcom_trop_io {
  int32_t glo_ni, glo_nj, dtbt, dtbc, flags;   /* flags: PCOM_LIT_R8 or 0 */
  const int32_t *lev_t, *lev_u;
  const double *prh_t, *prh_u, *cor, *am1, *graphihx, *graphihy;
  const double *dxx[4], *dxy[4], *rh[4];
  const double *ut, *vt, *bphi[4], *bgraphi[4]; /* xn, xs, ye, yw */
  double *chc, *chp, *mch, *mch2, *ubc, *vbc, *ubp, *vbp, *acch;
} pcom_trop_io;
int pcom_gpu_trop_noalloc(const pcom_trop_io *io, void *stream);

/* Message of the last failed call on this thread. */
int pcom_gpu_last_error(char *buf, int32_t len);

#ifdef __cplusplus
}
#endif
#endif
