// pcom_dev.cuh -- device-side view of one PCOM domain and the helpers every
// kernel shares.
//
// Layout in HBM: every field is FP64 (the mixed path stores its 3-D fields
// as FP32), Fortran order (i fastest) over the
// padded ni x nj domain, one contiguous plane per level.  The two x-halo
// columns (1 and ni) of every stored field hold copies of columns ni-1 and 2:
// that is what the reference's halo exchange leaves behind after each
// operator with npx = 1 (mod_mympi.f90:669-746), and because every operator
// covers all interior columns, every field the reference computes is
// periodic over the glo_ni interior columns.  Kernels therefore compute the
// interior columns 2..ni-1 with ring neighbours and also store the halo twin.
// Rows 1 and nj are NOT exchanged (MPI_PROC_NULL, mod_param.f90:299-305):
// each operator's row range and default value is reproduced explicitly.
//
// Arithmetic: the FP64 path is compiled with --fmad=false and keeps the
// reference's evaluation order, so results are bitwise those of the
// reference's gfortran build on x86-64 (SSE2, no FMA).
#pragma once
#include <cstdint>
#include <type_traits>
#include <cuda/atomic>
#include <cuda_runtime.h>

#define PCOM_MAXK 64

struct DevConsts {
  double g, a, a0, rho0, pi, gamma_t, gamma_s, gamma_b, deltat, deltas, cdbot, tice, smag_c, ah_c;
  double c_tc, c_tp, c_tpp;
  double eos[42];
};

// Everything a kernel needs, passed by value as a __grid_constant__ param.
// R is the storage type of the 3-D fields: double for the FP64 path, float
// for the mixed path (whose 2-D fields, barotropic state and accumulations
// stay double).
template <typename R> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };

// Fields of every precision: sizes, constants, the static grid, the 2-D
// state and scratch (always FP64).
struct DevCommon {
  int ni, nj, nk, nkp, nim, njm, glo_ni, glo_nj;
  // rows j_lo..j_hi (padded 1-based index) the step's 3-D kernels compute:
  // 1..nj for a whole domain, this rank's slab of rows when the domain is
  // split into row slabs across ranks (the 2-D prep kernels and the
  // barotropic subcycle always cover every row)
  int j_lo, j_hi;
  int bt, bc, nstep, rst;
  long long n2, n3, n3p;
  DevConsts c;
  double pr2[PCOM_MAXK], dpr2[PCOM_MAXK], dz1[PCOM_MAXK + 1];  // 1-based: [k]
  double dz2[PCOM_MAXK];                                         // layer thickness (gi2), 1-based
  // static 2D (index 1..4 = grid g1j..g4j)
  const double *rh[5], *dxx[5], *dxy[5];
  const double *tn3;
  const int *lev_t, *lev_u;
  const double *prh_t, *phih_t, *prh_u;
  const double *cv1, *cv2, *cor, *graphihx, *graphihy;
  // forcing (bnd)
  const double *taux, *tauy, *bnd_t, *bnd_s, *bnd_pa;
  // 2-D state
  double *ubc, *vbc, *ubp, *vbp;
  double *chc, *chp, *mch, *mch2;
  // 2-D step intermediates
  double *pax, *pay, *ut, *vt;
  double *bphi[4], *bgra[4];  // xn, xs, ye, yw
  double *sch_r, *sch_w;      // readyc sch (land 1) and upwelling sqrt(ter(chp))
  double *acch, *acssh;
  // barotropic subcycle scratch
  double *tr_ch[2], *tr_ub[2], *tr_vb[2];
  double *tr_acc[6];  // mch, mch2, ub, vb accumulators; first-substep viscosity (u, v)
  unsigned *bar;   // [0] arrival count, [1] generation
  unsigned long long *tile_flag;  // per-tile progress of the barotropic kernel (monotone across launches)
  int *err;        // [0] timeout flag, [1] watchdog flag
  // longest a device-side wait (the barotropic kernels' grid barriers) may
  // take before it gives up and sets err[0] (ns of global time)
  unsigned long long wait_ns = 2000000000ULL;
  // lat-lon (separable) metrics: dx?x depends on i only, dx?y and rh? on j
  // only (set_hgrid builds them from 1-D lon/lat, main.f90:408-493); when the
  // uploaded 2-D arrays have that structure these 1-D copies are set
  int separable;
  const double *dxx1d[5], *dxy1d[5], *rh1d[5];  // [g][i-1] and [g][j-1]
  // correctly rounded reciprocals of every static divisor (see dvr below):
  // 1/dx?x (i), 1/dx?y (j), 1/rh? (j), a*rh? and 1/(a*rh?) (j),
  // (a*a)*rh3 and its reciprocal (j)
  const double *rdxx1d[5], *rdxy1d[5], *rrh1d[5], *arh1d[5], *rarh1d[5];
  const double *aarh3, *raarh3;
  double ra, rg, rbc32;                             // 1/a, 1/g, 1/(4*8*dtbc)
  double rdpr2[PCOM_MAXK], rdz1[PCOM_MAXK + 1];     // 1/dpr (gi2), 1/dz (gi1)
  // 2-D static reciprocals: bottom pressures, Coriolis-adjustment
  // denominators 1 + (0.5 cor dt)^2 for dtbc and dtbt, smag's dx and 1/dx
  const double *rprh_t, *rprh_u, *rwc, *rwt, *dxs, *rdxs;
  const double *dys1d, *rdys1d;                     // smag's dy and 1/dy (j)
  // per-step 2-D reciprocals written by the 2-D prep kernels
  double *rsch, *rsch2, *rchc, *rmch, *rgm2, *schc, *schu, *rmch2;
  // AB3 start-up control for the current step
  int ab3_mode;    // 0 normal, 1 step 1 (copy auc into aup, aupp), 2 step 2 (aupp = aup)
  // mixed path: alpha and adp are stored as anomalies from the reference
  // profile alpha_r(k) = 1/rho(T_r(k), S_r(k), pr(k)) and from its int_tobot
  // over the column's own wet levels (adp_ref below, from the suffix sums
  // adp_cum(k) = sum_{kk >= k} alpha_r(kk) dpr(kk)); 1-based.  am1 is an
  // FP64 copy of am at level 1 for the barotropic subcycle
  double alpha_r[PCOM_MAXK], adp_cum[PCOM_MAXK + 1];
  double *am1;
};

// The 3-D fields, stored as R.
template <typename R>
struct DevT : DevCommon {
  const R *km, *kh;  // nkp levels
  R *tc, *sc, *tp, *sp;
  R *uc, *vc, *up, *vp;
  R *auc, *aup, *aupp, *avc, *avp, *avpp;
  R *am, *alpha, *adp, *wm;
  typename Vec2<R>::type *prho;
  R *fx, *fy;
  R *uu, *vv;                 // unweighted velocity for smag
  R *tn_, *sn_;               // new T/S (int_ts writes here, then pointers rotate)
  R *act, *acs, *acr, *acu, *acv, *acw;  // accumulators
};

using Dev = DevT<double>;
using DevM = DevT<float>;


#define PD __device__ __forceinline__

template <typename R>
PD long long I2(const DevT<R> &P, int i, int j) { return (long long)(i - 1) + (long long)P.ni * (j - 1); }
template <typename R>
PD long long I3(const DevT<R> &P, int i, int j, int k) { return I2(P, i, j) + P.n2 * (k - 1); }
// ring neighbours of an interior column (2 <= i <= ni-1)
template <typename R>
PD int IM(const DevT<R> &P, int i) { return i == 2 ? P.ni - 1 : i - 1; }
template <typename R>
PD int IP(const DevT<R> &P, int i) { return i == P.ni - 1 ? 2 : i + 1; }

PD double ld(const double *p, long long q) { return __ldg(p + q); }
PD float ld(const float *p, long long q) { return __ldg(p + q); }

// global time in ns
PD unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// One thread's bounded wait for an arrival counter to reach `want`: gives up
// when another thread has set *err, or after limit_ns of global time (then
// it sets *err itself; an iteration cap bounds the loop as well).  Returns
// true when the counter got there.
PD bool wait_count(unsigned long long *cnt, unsigned long long want, int *err, unsigned long long limit_ns) {
  cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> c(*cnt);
  cuda::atomic_ref<int, cuda::thread_scope_device> e(*err);
  if (c.load(cuda::memory_order_acquire) >= want) return true;
  const unsigned long long t0 = global_ns();
  for (long long it = 1; it < (1LL << 28); ++it) {
    if (c.load(cuda::memory_order_acquire) >= want) return true;
    if (e.load(cuda::memory_order_relaxed) != 0) return false;
    if (global_ns() - t0 > limit_ns) break;
    if (it > 1024) __nanosleep(32);
  }
  e.store(1, cuda::memory_order_relaxed);
  return false;
}

// x / y rounded to nearest, given ry = 1/y correctly rounded: the quotient
// estimate x*ry is corrected once with its exact remainder (Markstein's
// theorem, IBM J. Res. Dev. 34(1), 1990: with a correctly rounded reciprocal
// and a quotient within one ulp, q + (x - y q) ry rounds to the correctly
// rounded x / y).  Checked bit-for-bit against IEEE division on 1.7e10
// random and adversarial operand pairs on B200.  Finite operands only.
PD double dvr(double x, double y, double ry) {
  const double q = x * ry;
  const double r = __fma_rn(-q, y, x);
  return __fma_rn(r, ry, q);
}
// mixed path: an FP32 quotient from the (rounded) reciprocal
template <typename Y, typename RY>
PD float dvr(float x, Y, RY ry) { return x * (float)ry; }

// alpha and adp as stored (anomalies on the mixed path) and as used
template <typename R>
PD R alpha_store(const DevT<R> &P, double v, int k) {
  if constexpr (std::is_same<R, float>::value) return (float)(v - P.alpha_r[k]); else return v;
}
template <typename R>
PD double alpha_full(const DevT<R> &P, R v, int k) {
  if constexpr (std::is_same<R, float>::value) return P.alpha_r[k] + (double)v; else return v;
}
// int_tobot of the reference profile over levels k..lev of a column
PD double adp_ref(const double *alpha_r, const double *dpr2, const double *cum, int k, int lev) {
  return k <= lev ? alpha_r[k] * dpr2[k] * 0.5 + (cum[k + 1] - cum[lev + 1]) : 0.0;
}
// q2: the column's 2-D index (its lev sets the reference)
template <typename R>
PD R adp_store(const DevT<R> &P, double v, int k, long long q2) {
  if constexpr (std::is_same<R, float>::value)
    return (float)(v - adp_ref(P.alpha_r, P.dpr2, P.adp_cum, k, __ldg(P.lev_t + q2)));
  else return v;
}
template <typename R>
PD double adp_full(const DevT<R> &P, R v, int k, long long q2) {
  if constexpr (std::is_same<R, float>::value)
    return adp_ref(P.alpha_r, P.dpr2, P.adp_cum, k, __ldg(P.lev_t + q2)) + (double)v;
  else return v;
}

// store to an interior column and to its halo twin
template <typename T, typename R, typename V>
PD void st2(T *p, const DevT<R> &P, int i, long long q, V v) {
  const T w = (T)v;
  p[q] = w;
  if (i == 2) p[q + (P.ni - 2)] = w;
  else if (i == P.ni - 1) p[q - (P.ni - 2)] = w;
}

// den_rho, mod_den.f90:57-118, same evaluation order as the reference.
PD double den_rho(const DevConsts &C, double t, double s, double p0) {
  const double *e = C.eos;
  double p = p0 * e[41];
  double p2 = p * p;
  double t2 = t * t;
  double t3 = t2 * t;
  double t4 = t3 * t;
  double t5 = t4 * t;
  double s32 = s * sqrt(s);
  double s2 = s * s;
  double r0 = e[0] + e[1] * t - e[2] * t2 + e[3] * t3 - e[4] * t4 + e[5] * t5;
  double a = e[6] - e[7] * t + e[8] * t2 - e[9] * t3 + e[10] * t4;
  double b = -e[11] + e[12] * t - e[13] * t2;
  double r = r0 + a * s + b * s32 + e[14] * s2;
  double k = e[15] + e[16] * t - e[17] * t2 + e[18] * t3 - e[19] * t4 +
             (e[20] - e[21] * t + e[22] * t2 - e[23] * t3) * s +
             (e[24] + e[25] * t - e[26] * t2) * s32 +
             (e[27] + e[28] * t - e[29] * t2 + e[30] * t3) * p +
             (e[31] - e[32] * t + e[33] * t2) * s * p + e[34] * s32 * p +
             (e[35] - e[36] * t + e[37] * t2) * p2 +
             (-e[38] + e[39] * t + e[40] * t2) * s * p2;
  return r / (1.0 - p / k);
}

// ---------------------------------------------------------------------------
// 2-D staggered-grid primitives.  Grids: T = g1j, E = g2j, U = g3j, N = g4j
// (mod_arrays.f90:148-166).  Each helper returns the value the reference's
// operator leaves at (i, j) after its halo exchange; i must be interior.

// ter T->U, diagonal 4-point mean (ter_r2d, hga = g1j, mod_op.f90:416-419);
// rows j = nj get the default `dft`.
template <typename R>
PD double terTU(const DevT<R> &P, const double *f, int i, int j, double dft) {
  if (j > P.njm) return dft;
  long long q = I2(P, i, j);
  return (ld(f, q) + ld(f, q + P.ni) + ld(f, q + 1) + ld(f, q + 1 + P.ni)) * 0.25;
}

// msk of the T grid (g12) and U grid (g32): set_grid builds msk = (lev >= k)
// (main.f90:605-625); pcom_gpu_upload_static checks that the given masks are
// exactly that, so kernels derive them from the 2-D lev arrays.
template <typename R>
PD double mT(const DevT<R> &P, long long q2, int k) { return (double)(__ldg(P.lev_t + q2) >= k); }
template <typename R>
PD double mU(const DevT<R> &P, long long q2, int k) { return (double)(__ldg(P.lev_u + q2) >= k); }

// launch geometry shared by the column kernels
#define COLS_X 32
#define COLS_Y 4
