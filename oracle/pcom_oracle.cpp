/*
 * pcom_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * An FP64 CPU restatement of the PCOM v2.2 baroclinic time step and of the
 * setup that feeds it, written array-op by array-op the way the reference's
 * Fortran is written, so that a reviewer can hold it against the Fortran
 * line by line.  It is the checker for the CUDA path in pcom_b200/ and the
 * CPU baseline ("port") timed by bench.py; the product never calls it.
 *
 * Parity pinning: the reference ships no field-level golden data and cannot
 * be built in this image (no gfortran/MPI/netCDF), so field-level parity is
 * UNPINNED beyond this restatement.  The only known-answer value shipped with
 * the reference -- rho(3 degC, 35.5 psu, 300e5 Pa) = 1041.83267 kg/m^3 within
 * 3.6e-7 (notes.rst:20-26) -- pins den_rho (tests/test_oracle.py).
 *
 * Semantics emulated (cited per function below):
 *  - gfortran default REAL literals are REAL(4): every unsuffixed literal is
 *    rounded to float once, then widened (L() below); expressions made only of
 *    literals and integers are evaluated in REAL(4) (mod_con.f90:27,
 *    mod_int.f90:314-316, mod_arrays.f90:298, mod_int.f90:667,675).
 *    r8 = 1 switches to the ifort "-r8" reading (all literals double).
 *  - left-to-right evaluation of + - * / chains, no FMA contraction
 *    (build with -ffp-contract=off), sequential SUM over k.
 *  - halo exchange of mod_mympi.f90:669-861 with npx = npy = 1: column 1 <-
 *    column ni-1, column ni <- column 2, rows 1 and nj untouched
 *    (MPI_PROC_NULL north/south neighbours, mod_param.f90:299-305).
 *  - Fortran locals that the reference never writes on some points
 *    (grachint/chgraint%x(1) row nj in int_trop, mod_int.f90:212-228; the
 *    land points of wk in int_ts, mod_int.f90:503-504) are taken as 0 and as
 *    "acr unchanged on land" respectively.  Both are multiplied by a zero
 *    mask (or are land-only diagnostics), so any finite value gives the same
 *    result on wet points.
 */
#include "pcom_oracle.h"
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <memory>
#include <utility>
#include <malloc.h>
#include <map>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

/* ------------------------------------------------------------------ arrays */
// Allocator whose resize leaves new doubles/ints uninitialised, so that an
// array's fill below runs in parallel instead of as a serial zero-fill.
template <class T>
struct DefaultInit : std::allocator<T> {
  template <class U>
  struct rebind { using other = DefaultInit<U>; };
  DefaultInit() = default;
  template <class U>
  DefaultInit(const DefaultInit<U> &) noexcept {}
  template <class U>
  void construct(U *p) noexcept { ::new ((void *)p) U; }
  template <class U, class... Args>
  void construct(U *p, Args &&...args) { ::new ((void *)p) U(std::forward<Args>(args)...); }
};
struct A3 {
  int n1 = 0, n2 = 0, n3 = 0;
  std::vector<double, DefaultInit<double>> v;
  A3() {}
  A3(int a, int b, int c = 1, double x = 0.0) { init(a, b, c, x); }
  void init(int a, int b, int c = 1, double x = 0.0) {
    n1 = a; n2 = b; n3 = c;
    const long long n = (long long)a * b * c;
    v.resize((size_t)n);
    _Pragma("omp parallel for schedule(static)") for (long long q = 0; q < n; ++q) v[q] = x;
  }
  inline double &operator()(int i, int j, int k = 1) {
    return v[(size_t)(i - 1) + (size_t)n1 * ((size_t)(j - 1) + (size_t)n2 * (size_t)(k - 1))];
  }
  inline double operator()(int i, int j, int k = 1) const {
    return v[(size_t)(i - 1) + (size_t)n1 * ((size_t)(j - 1) + (size_t)n2 * (size_t)(k - 1))];
  }
  void fill(double x) { std::fill(v.begin(), v.end(), x); }
};
struct I3 {
  int n1 = 0, n2 = 0, n3 = 0;
  std::vector<int32_t, DefaultInit<int32_t>> v;
  void init(int a, int b, int c = 1, int x = 0) {
    n1 = a; n2 = b; n3 = c;
    const long long n = (long long)a * b * c;
    v.resize((size_t)n);
    _Pragma("omp parallel for schedule(static)") for (long long q = 0; q < n; ++q) v[q] = x;
  }
  inline int32_t &operator()(int i, int j, int k = 1) {
    return v[(size_t)(i - 1) + (size_t)n1 * ((size_t)(j - 1) + (size_t)n2 * (size_t)(k - 1))];
  }
  inline int32_t operator()(int i, int j, int k = 1) const {
    return v[(size_t)(i - 1) + (size_t)n1 * ((size_t)(j - 1) + (size_t)n2 * (size_t)(k - 1))];
  }
};

#define PAR _Pragma("omp parallel for schedule(static)")
// level x row nests: one work item per (k, j), so 2-D fields (n3 = 1) split
// over rows too
#define PAR2 _Pragma("omp parallel for collapse(2) schedule(static)")

/* ---------------------------------------------------------------- literals */
/* A default-REAL literal: rounded once to REAL(4) (gfortran) or kept (r8). */
struct Lit {
  int r8;
  double operator()(float f, double d) const { return r8 ? d : (double)f; }
};
#define L(x) lit((float)(x##f), (double)(x))

struct Consts {
  double rho0, a0, g, a, pi, omega, torad, gamma_t, gamma_s, gamma_b, deltat,
      deltas, cdbot, tice, km_c, am_c, smag_c, ah_c;
  double c_tc, c_tp, c_tpp, alpha_land;
};

static void make_consts(Consts &C, int r8) {
  Lit lit{r8};
  /* mod_con.f90:16-36 */
  C.rho0 = L(1029.0);
  C.a0 = 1.0 / C.rho0;
  C.g = L(9.8);
  C.a = L(6370e3);
  C.pi = L(3.141592653589793);
  C.omega = C.pi / L(43082.0);
  C.torad = C.pi / L(180.0);
  C.gamma_t = C.g * L(40.0) / L(3901.0);
  /* 1.0 / (120*24*60*60): a REAL(4) / INTEGER expression */
  C.gamma_s = r8 ? 1.0 / (double)(120 * 24 * 60 * 60) : (double)(1.0f / (float)(120 * 24 * 60 * 60));
  C.gamma_b = L(0.2);
  C.deltat = L(1.0e-2);
  C.deltas = L(1.0e-3);
  C.cdbot = L(2.6);
  C.tice = L(-1.5);
  C.km_c = L(1.0e-5);
  C.am_c = L(1.0e3);
  C.smag_c = L(0.56);
  C.ah_c = L(1.0e3);
  /* mod_int.f90:314-316: 23.0/12 etc. are REAL(4) divisions */
  C.c_tc = r8 ? 23.0 / 12 : (double)(23.0f / 12);
  C.c_tp = r8 ? -16.0 / 12 : (double)(-16.0f / 12);
  C.c_tpp = r8 ? 5.0 / 12 : (double)(5.0f / 12);
  /* mod_arrays.f90:298: 1/1000.0*one */
  C.alpha_land = r8 ? 1.0 / 1000.0 : (double)(1.0f / 1000.0f);
}

/* den_rho, mod_den.f90:57-118 (UNESCO 1981 / Jackett & McDougall 1995). */
static double den_rho(double t, double s, double p0, int r8) {
  Lit lit{r8};
  double p = p0 * L(1e-5);
  double p2 = p * p;
  double t2 = t * t;
  double t3 = t2 * t;
  double t4 = t3 * t;
  double t5 = t4 * t;
  double s32 = s * std::sqrt(s);
  double s2 = s * s;
  double r0 = L(999.842594) + L(6.793952e-2) * t - L(9.095290e-3) * t2 + L(1.001685e-4) * t3 -
              L(1.120083e-6) * t4 + L(6.536336e-9) * t5;
  double a = L(8.24493e-1) - L(4.0899e-3) * t + L(7.6438e-5) * t2 - L(8.2467e-7) * t3 + L(5.3875e-9) * t4;
  double b = -L(5.72466e-3) + L(1.0227e-4) * t - L(1.6546e-6) * t2;
  double r = r0 + a * s + b * s32 + L(4.8314e-4) * s2;
  double k = L(1.965933e4) + L(1.444304e2) * t - L(1.706103) * t2 + L(9.648704e-3) * t3 - L(4.190253e-5) * t4 +
             (L(5.284855e1) - L(3.101089e-1) * t + L(6.283263e-3) * t2 - L(5.084188e-5) * t3) * s +
             (L(3.886640e-1) + L(9.085835e-3) * t - L(4.619924e-4) * t2) * s32 +
             (L(3.186519) + L(2.212276e-2) * t - L(2.984642e-4) * t2 + L(1.956415e-6) * t3) * p +
             (L(6.704388e-3) - L(1.847318e-4) * t + L(2.059331e-7) * t2) * s * p + L(1.480266e-4) * s32 * p +
             (L(2.102898e-4) - L(1.202016e-5) * t + L(1.394680e-7) * t2) * p2 +
             (-L(2.040237e-6) + L(6.128773e-8) * t + L(6.207323e-10) * t2) * s * p2;
  return r / (1.0 - p / k);
}

/* ------------------------------------------------------------------- grids */
/* type_gi (mod_type.f90:97-108): horizontal stagger grid with its index shift
 * (i, j) and its east-west / north-south / diagonal neighbours
 * (mod_arrays.f90:148-168, 554-582). */
struct HG {
  int n = 0, si = 0, sj = 0;
  A3 rh, tn, dx1, dx2;
  HG *ns = nullptr, *ew = nullptr, *di = nullptr;
};
struct VG { /* type_gj, 1-based vectors */
  int n = 0;
  std::vector<double> z, pr, dz, dpr;
  void init(int len) { z.assign(len + 1, 0.0); pr.assign(len + 1, 0.0); dz.assign(len + 1, 0.0); dpr.assign(len + 1, 0.0); }
};
struct G3 { /* type_gij */
  I3 msk, lev;
  A3 phih, prh;
};

struct Time { int y, m, d, h, mi, s, mm; };

static int days_year(int y) { /* mod_type.f90:423-438 */
  int d = 365;
  if (y % 100 == 0) { if (y % 400 == 0) d = 366; }
  else if (y % 4 == 0) d = 366;
  return d;
}
static int days_month(int y, int m) { /* mod_type.f90:403-420 */
  static const int days[12] = {31, 28, 31, 30, 31, 30, 31, 31, 30, 31, 30, 31};
  int d = days[m - 1];
  if (m == 2 && days_year(y) == 366) d = 29;
  return d;
}
static Time time_plus(Time t, int dt) { /* mod_type.f90:593-635 */
  t.s += dt;
  if (t.s >= 60) { t.mi += t.s / 60; t.s %= 60; }
  if (t.mi >= 60) { t.h += t.mi / 60; t.mi %= 60; }
  if (t.h >= 24) { t.d += t.h / 24; t.h %= 24; }
  if (t.d > t.mm) { t.m += 1; t.d = 1; }
  if (t.m > 12) { t.y += 1; t.m = 1; }
  t.mm = days_month(t.y, t.m);
  return t;
}

/* ------------------------------------------------------------------- model */
struct Model {
  Consts C;
  int r8 = 0;
  int glo_ni, glo_nj, nk, ni, nj, nim, njm, nkp;
  int bt, bc, rst = 0;
  HG g1j, g2j, g3j, g4j;
  VG gi1, gi2;
  G3 g12, g32;
  std::vector<double> lon, lat, z; /* 1-based */
  A3 hposx, hposy;
  A3 cv1, cv2, cor, km, kh, graphihx, graphihy;
  A3 frc_taux, frc_tauy, frc_t, frc_s, frc_pa, frc_fw;
  A3 bnd_taux, bnd_tauy, bnd_t, bnd_s, bnd_pa, bnd_fw;
  /* state */
  A3 tc, sc, tp, sp;               /* temp%v(:,:,:,tc/tp), salt */
  A3 uc, vc, up, vp;               /* upres/vpres */
  A3 auc, aup, aupp, avc, avp, avpp;
  A3 fx, fy, pax, pay;
  A3 ubc, vbc, ubp, vbp, ut, vt;
  A3 chc, chp, mch, mch2;
  A3 am, prho1, prho2, alpha, adp, wm;
  A3 bphi_xn, bphi_xs, bphi_ye, bphi_yw, bgra_xn, bgra_xs, bgra_ye, bgra_yw;
  A3 act, acs, acr, acu, acv, acw, acch, acssh;
  int n_ts = 0, n_uv = 0, n_w = 0, n_ch = 0, n_ssh = 0;
  /* time control */
  Time ct, pt;
  long long iter = 0; /* tctr%i */
  long long nday = 0;
  bool first = true;
  std::map<std::string, A3 *> f;
  std::map<std::string, I3 *> fi;

  /* -------------------------------------------------------- halo exchange */
  /* swpbnd_r3d/r2d (mod_mympi.f90:669-746) with px = py = 1 */
  void swp(A3 &x) const {
    for (int k = 1; k <= x.n3; ++k)
      for (int j = 1; j <= x.n2; ++j) {
        x(1, j, k) = x(ni - 1, j, k);
        x(ni, j, k) = x(2, j, k);
      }
  }
  void swpi(I3 &x) const {
    for (int k = 1; k <= x.n3; ++k)
      for (int j = 1; j <= x.n2; ++j) {
        x(1, j, k) = x(ni - 1, j, k);
        x(ni, j, k) = x(2, j, k);
      }
  }

  /* ----------------------------------------------------------- operators */
  /* ter_r3d / ter_r2d, mod_op.f90:361-427 */
  void ter(A3 &ans, const A3 &var, const HG &hga, const HG &hgb, double dft = 0.0) const {
    const int n3 = var.n3;
    ans.init(ni, nj, n3, dft);
    if (hga.n == hgb.n) { fprintf(stderr, "no need to interpolate\n"); abort(); }
    if (hga.ew == &hgb) {
      PAR2 for (int k = 1; k <= n3; ++k)
        for (int j = 1; j <= nj; ++j)
          for (int i = 1; i <= nim; ++i) ans(i + hga.si, j, k) = 0.5 * (var(i, j, k) + var(i + 1, j, k));
    } else if (hga.ns == &hgb) {
      PAR2 for (int k = 1; k <= n3; ++k)
        for (int j = 1; j <= njm; ++j)
          for (int i = 1; i <= ni; ++i) ans(i, j + hga.sj, k) = 0.5 * (var(i, j, k) + var(i, j + 1, k));
    } else if (hga.di == &hgb) {
      PAR2 for (int k = 1; k <= n3; ++k)
        for (int j = 1; j <= njm; ++j)
          for (int i = 1; i <= nim; ++i)
            ans(i + hga.si, j + hga.sj, k) =
                (var(i, j, k) + var(i, j + 1, k) + var(i + 1, j, k) + var(i + 1, j + 1, k)) * 0.25;
    } else { fprintf(stderr, "unhandled relative position in ter\n"); abort(); }
    swp(ans);
  }
  /* p1_r3d / p1_r2d / p1_r3d_b, mod_op.f90:496-527, 561-620 */
  void p1(A3 &ans, const A3 &var, const HG &ga, const HG &gb, const I3 *mask = nullptr) const {
    A3 tmp;
    const A3 *t = &var;
    if (gb.ew != &ga) { ter(tmp, var, ga, *gb.ew); t = &tmp; }
    const int n3 = var.n3;
    ans.init(ni, nj, n3, 0.0);
    PAR2 for (int k = 1; k <= n3; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= nim; ++i) {
          double d = (*t)(i + 1, j, k) - (*t)(i, j, k);
          if (mask) d = d * (*mask)(i + 1, j, k) * (*mask)(i, j, k);
          ans(i + ga.si, j, k) = d;
        }
    PAR2 for (int k = 1; k <= n3; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) ans(i, j, k) = ans(i, j, k) / gb.dx1(i, j);
    swp(ans);
  }
  /* p2_r3d / p2_r2d / p2_r3d_b, mod_op.f90:622-713 */
  void p2(A3 &ans, const A3 &var, const HG &ga, const HG &gb, const I3 *mask = nullptr) const {
    A3 tmp;
    const A3 *t = &var;
    if (gb.ns != &ga) { ter(tmp, var, ga, *gb.ns); t = &tmp; }
    const int n3 = var.n3;
    ans.init(ni, nj, n3, 0.0);
    PAR2 for (int k = 1; k <= n3; ++k)
      for (int j = 1; j <= njm; ++j)
        for (int i = 1; i <= ni; ++i) {
          double d = (*t)(i, j + 1, k) - (*t)(i, j, k);
          if (mask) d = d * (*mask)(i, j + 1, k) * (*mask)(i, j, k);
          ans(i, j + ga.sj, k) = d;
        }
    PAR2 for (int k = 1; k <= n3; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) ans(i, j, k) = ans(i, j, k) / gb.dx2(i, j);
    swp(ans);
  }
  /* px_r3d_center, mod_op.f90:529-559 (hg = guj) */
  void px_center(A3 &ans, const A3 &var, const HG &hg) const {
    ans.init(ni, nj, var.n3, 0.0);
    PAR2 for (int k = 1; k <= var.n3; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 2; i <= ni - 1; ++i) {
          double dx = C.a * hg.ew->rh(i, j) * (hg.ew->dx1(i, j) + hg.ew->dx1(i + 1, j));
          ans(i, j, k) = (var(i + 1, j, k) - var(i - 1, j, k)) / dx;
        }
    swp(ans);
  }
  /* p3_r3d, mod_op.f90:715-735: var on gi1 (nkp) -> gi2 (nk) */
  void p3(A3 &ans, const A3 &var) const {
    ans.init(ni, nj, nk, 0.0);
    PAR2 for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) ans(i, j, k) = (var(i, j, k) - var(i, j, k + 1)) / gi2.dpr[k];
  }
  /* pz_r3d, mod_op.f90:762-790: gi2 (nk) -> gi1 (nkp) */
  void pz(A3 &ans, const A3 &var, const I3 &msk) const {
    ans.init(ni, nj, nkp, 0.0);
    PAR2 for (int k = 2; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i)
          ans(i, j, k) = (var(i, j, k - 1) - var(i, j, k)) * msk(i, j, k - 1) * msk(i, j, k) / gi1.dz[k];
  }
  /* dx3_r3d_b, mod_op.f90:792-811 */
  void dx3(A3 &ans, const A3 &var) const {
    ans.init(ni, nj, nkp, 0.0);
    PAR2 for (int k = 2; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) ans(i, j, k) = var(i, j, k - 1) - var(i, j, k);
  }
  /* vter_r3d, mod_op.f90:327-359.  from_gi2: gi2 -> gi1, else gi1 -> gi2 */
  void vter(A3 &ans, const A3 &var, bool from_gi2) const {
    if (from_gi2) {
      ans.init(ni, nj, nkp, 0.0);
      PAR2 for (int k = 2; k <= nk; ++k)
        for (int j = 1; j <= nj; ++j)
          for (int i = 1; i <= ni; ++i) ans(i, j, k) = (var(i, j, k - 1) + var(i, j, k)) * 0.5;
    } else {
      ans.init(ni, nj, nk, 0.0);
      PAR2 for (int k = 1; k <= nk; ++k)
        for (int j = 1; j <= nj; ++j)
          for (int i = 1; i <= ni; ++i) ans(i, j, k) = (var(i, j, k) + var(i, j, k + 1)) * 0.5;
    }
  }
  /* div_r3d / div_r2d, mod_op.f90:813-848 */
  void div(A3 &ans, const A3 &va, const A3 &vb, const HG &ga, const HG &gb, const HG &gc) const {
    A3 wka, wkb, tmp(ni, nj, vb.n3);
    p1(wka, va, ga, gc);
    for (int k = 1; k <= vb.n3; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) tmp(i, j, k) = vb(i, j, k) * gb.rh(i, j);
    p2(wkb, tmp, gb, gc);
    ans.init(ni, nj, va.n3);
    for (int k = 1; k <= va.n3; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) ans(i, j, k) = (wka(i, j, k) + wkb(i, j, k)) / (C.a * gc.rh(i, j));
  }
  /* gra_r2d / gra_r2d_b / gra_r3d / gra_r3d_b, mod_op.f90:850-902 */
  void gra(A3 &ax, A3 &ay, const A3 &var, const HG &ga, const HG &gb, const HG &gc) const {
    p1(ax, var, ga, gb);
    for (int k = 1; k <= var.n3; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) ax(i, j, k) = ax(i, j, k) / (C.a * gb.rh(i, j));
    p2(ay, var, ga, gc);
    PAR for (long long q = 0; q < (long long)ay.v.size(); ++q) ay.v[q] = ay.v[q] / C.a;
  }
  /* op_lap, mod_op.f90:904-925 */
  void lap(A3 &ans, const A3 &var, const HG &ga, const HG &gb) const {
    A3 wka, wkb;
    p1(wka, var, ga, *gb.ew);
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni; ++i) wka(i, j) = wka(i, j) / gb.ew->rh(i, j);
    p1(wkb, wka, *gb.ew, gb);
    ans = wkb;
    p2(wka, var, ga, *gb.ns);
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni; ++i) wka(i, j) = wka(i, j) * gb.ns->rh(i, j);
    p2(wkb, wka, *gb.ns, gb);
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni; ++i) ans(i, j) = ans(i, j) + wkb(i, j);
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni; ++i) ans(i, j) = ans(i, j) / (C.a * C.a * gb.rh(i, j));
  }
  /* int_tobot, mod_op.f90:927-944 (grd = g12) */
  void int_tobot(A3 &ans, const A3 &var) const {
    A3 temp(ni, nj, nk);
    ans.init(ni, nj, nk);
    PAR for (int j = 1; j <= nj; ++j) {
      for (int k = 1; k <= nk; ++k)
        for (int i = 1; i <= ni; ++i) temp(i, j, k) = var(i, j, k) * gi2.dpr[k] * g12.msk(i, j, k);
      for (int i = 1; i <= ni; ++i) {
        for (int k = 1; k <= nk - 1; ++k) {
          double s = 0.0;
          for (int kk = k + 1; kk <= nk; ++kk) s = s + temp(i, j, kk);
          ans(i, j, k) = temp(i, j, k) * 0.5 + s;
        }
        ans(i, j, nk) = temp(i, j, nk) * 0.5;
      }
    }
  }
  /* op_vint_ns, mod_op.f90:946-962 */
  void vint_ns(const A3 &var, A3 &ren, A3 &res) const {
    ren.init(ni, nj); res.init(ni, nj);
    PAR for (int j = 1; j <= nj; ++j) {
      int js = (j == 1) ? nj : j - 1; /* cshift(-1, dim=2) */
      for (int i = 1; i <= ni; ++i) {
        double s1 = 0.0, s2 = 0.0;
        for (int k = 1; k <= nk; ++k) {
          s1 = s1 + var(i, j, k) * gi2.dpr[k] * g32.msk(i, j, k);
          s2 = s2 + var(i, j, k) * gi2.dpr[k] * g32.msk(i, js, k);
        }
        ren(i, j) = s1 / g32.prh(i, j);
        res(i, j) = s2 / g32.prh(i, js);
      }
    }
    swp(ren); swp(res);
  }
  /* op_vint_ew, mod_op.f90:964-981 */
  void vint_ew(const A3 &var, A3 &ree, A3 &rew) const {
    ree.init(ni, nj); rew.init(ni, nj);
    PAR for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni; ++i) {
        int is = (i == 1) ? ni : i - 1; /* cshift(-1, dim=1) */
        double s1 = 0.0, s2 = 0.0;
        for (int k = 1; k <= nk; ++k) {
          s1 = s1 + var(i, j, k) * gi2.dpr[k] * g32.msk(i, j, k);
          s2 = s2 + var(i, j, k) * gi2.dpr[k] * g32.msk(is, j, k);
        }
        ree(i, j) = s1 / g32.prh(i, j);
        rew(i, j) = s2 / g32.prh(is, j);
      }
    swp(ree); swp(rew);
  }
  /* vint_r3d, mod_op.f90:983-995 */
  void vint(A3 &ans, const A3 &var, const G3 &grd) const {
    ans.init(ni, nj);
    PAR for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni; ++i) {
        double s = 0.0;
        for (int k = 1; k <= nk; ++k) s = s + var(i, j, k) * gi2.dpr[k] * grd.msk(i, j, k);
        ans(i, j) = s / grd.prh(i, j);
      }
  }

  /* ---------------------------------------------------------- mod_den */
  /* den_alpha, mod_den.f90:33-55 */
  void den_alpha(A3 &alpha_, const A3 &t, const A3 &s, const A3 &ch) const {
    PAR2 for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i)
          if (g12.msk(i, j, k) == 1) alpha_(i, j, k) = 1.0 / den_rho(t(i, j, k), s(i, j, k), ch(i, j) * gi2.pr[k], r8);
  }
  /* den_prho, mod_den.f90:120-153 */
  void den_prho() {
    PAR2 for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i)
          if (g12.msk(i, j, k) > 0) {
            double t = tc(i, j, k), s = sc(i, j, k), p = chc(i, j) * gi2.pr[k];
            double ra = den_rho(t + C.deltat, s, p, r8), rb = den_rho(t - C.deltat, s, p, r8);
            prho1(i, j, k) = (ra - rb) / (2 * C.deltat);
            ra = den_rho(t, s + C.deltas, p, r8);
            rb = den_rho(t, s - C.deltas, p, r8);
            prho2(i, j, k) = (ra - rb) / (2 * C.deltas);
          }
  }

  /* ---------------------------------------------------------- mod_int */
  /* int_pgra, mod_int.f90:64-88 */
  void int_pgra() {
    int_tobot(adp, alpha);
    A3 wkb, wkc, wk(ni, nj, nk), wkx, wky;
    ter(wkb, adp, g1j, *g1j.ew);
    ter(wkc, alpha, g1j, *g1j.ew);
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) wk(i, j, k) = wkb(i, j, k) + gi2.pr[k] * wkc(i, j, k);
    vint_ns(wk, bphi_xn, bphi_xs);
    ter(wkb, adp, g1j, *g1j.ns);
    ter(wkc, alpha, g1j, *g1j.ns);
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) wk(i, j, k) = wkb(i, j, k) + gi2.pr[k] * wkc(i, j, k);
    vint_ew(wk, bphi_ye, bphi_yw);
    gra(wkx, wky, adp, g1j, *g1j.ew, *g1j.ns);
    vint_ns(wkx, bgra_xn, bgra_xs);
    vint_ew(wky, bgra_ye, bgra_yw);
  }

  /* upwelling, mod_int.f90:626-647 */
  void upwelling() {
    A3 sch, wk3d, wk2d, va(ni, nj, nk), vb(ni, nj, nk);
    ter(sch, chp, g1j, g3j); /* g32%hg = g3j */
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) {
          double s3 = std::sqrt(sch(i, j));
          va(i, j, k) = s3 * uc(i, j, k);
          vb(i, j, k) = s3 * vc(i, j, k);
        }
    div(wk3d, va, vb, g3j, g3j, g1j); /* wm%g%hg = g11%hg = g1j */
    vint(wk2d, wk3d, g12);
    PAR for (long long q = 0; q < (long long)wk2d.v.size(); ++q) { double &x = wk2d.v[q]; x = -x; }
    for (int k = 2; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) {
          wm(i, j, k) = wm(i, j, k - 1) + gi2.dpr[k - 1] * (wk2d(i, j) + wk3d(i, j, k - 1));
          wm(i, j, k) = wm(i, j, k) * g12.msk(i, j, k);
        }
  }

  /* op_adv, mod_op.f90:224-278 */
  void op_adv(A3 &ans, const A3 &var, const A3 &sch) {
    A3 wka(ni, nj, nk), u, v, w, wkap(ni, nj, nkp), wkb, wkm1(ni, nj, nk), wkm2(ni, nj, nk), wkbp(ni, nj, nkp);
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) wka(i, j, k) = uc(i, j, k) / sch(i, j);
    ter(u, wka, g3j, *g3j.ew);
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) wka(i, j, k) = vc(i, j, k) / sch(i, j) * g3j.rh(i, j);
    ter(v, wka, g3j, *g3j.ns);
    for (int k = 1; k <= nkp; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) wkap(i, j, k) = wm(i, j, k) / chc(i, j);
    ter(w, wkap, g1j, g3j);
    A3 wa, wb;
    ter(wa, var, g3j, *g3j.ew);
    ter(wb, var, g3j, *g3j.ns);
    PAR for (long long q = 0; q < (long long)wa.v.size(); ++q) { wkm1.v[q] = wa.v[q] * u.v[q]; wkm2.v[q] = wb.v[q] * v.v[q]; }
    p1(wa, wkm1, *g3j.ew, g3j);
    p2(wb, wkm2, *g3j.ns, g3j);
    ans.init(ni, nj, nk);
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) ans(i, j, k) = (wa(i, j, k) + wb(i, j, k)) / (C.a * g3j.rh(i, j));
    vter(wkap, var, true);
    PAR for (long long q = 0; q < (long long)wkap.v.size(); ++q) wkap.v[q] = wkap.v[q] * w.v[q];
    for (int k = 2; k <= nkp - 1; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) wkbp(i, j, k) = wkap(i, j, k) * g32.msk(i, j, k - 1) * g32.msk(i, j, k);
    p3(wa, wkbp);
    PAR for (long long q = 0; q < (long long)ans.v.size(); ++q) ans.v[q] = ans.v[q] + wa.v[q];
    p1(wkm1, u, *g3j.ew, g3j);
    p2(wkm2, v, *g3j.ns, g3j);
    p3(wa, w);
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i)
          ans(i, j, k) = ans(i, j, k) -
                         0.5 * var(i, j, k) * ((wkm1(i, j, k) + wkm2(i, j, k)) / (C.a * g3j.rh(i, j)) + wa(i, j, k));
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) ans(i, j, k) = ans(i, j, k) * g32.msk(i, j, k);
  }

  /* fri_r3d, mod_op.f90:103-167 */
  void fri_r3d(A3 &ans, const A3 &sch, const A3 &v, const A3 &vpv, const A3 &vcv, const A3 &tau) {
    A3 wx, wy, ch3da, ch3db, wka, wkp;
    gra(wx, wy, v, g3j, *g3j.ew, *g3j.ns);
    ter(ch3da, chc, g1j, *g3j.ew);
    ter(ch3db, chc, g1j, *g3j.ns);
    A3 va(ni, nj, nk), vb(ni, nj, nk);
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) {
          va(i, j, k) = ch3da(i, j) * wx(i, j, k);
          vb(i, j, k) = ch3db(i, j) * wy(i, j, k);
        }
    div(wka, va, vb, *g3j.ew, *g3j.ns, g3j);
    ans.init(ni, nj, nk);
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) ans(i, j, k) = am(i, j, k) / sch(i, j) * wka(i, j, k);
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) ans(i, j, k) = ans(i, j, k) + am(i, j, k) * cv1(i, j) * vpv(i, j, k);
    px_center(wka, vcv, g3j);
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i)
          ans(i, j, k) = ans(i, j, k) + am(i, j, k) * cv2(i, j) * sch(i, j) * wka(i, j, k);
    pz(wkp, vpv, g32.msk);
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i)
          wkp(i, j, k) = C.g * C.rho0 * km(i, j, k) * wkp(i, j, k) / (sch(i, j) * sch(i, j));
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni; ++i) wkp(i, j, 1) = C.g * tau(i, j) / sch(i, j);
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni; ++i) {
        int k = g32.lev(i, j);
        if (k > 0) {
          double mag = std::sqrt(v(i, j, k) * v(i, j, k) + vcv(i, j, k) * vcv(i, j, k));
          wkp(i, j, k + 1) = v(i, j, k) * C.g * C.cdbot * mag / sch(i, j);
        }
      }
    p3(wka, wkp);
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) ans(i, j, k) = ans(i, j, k) * g32.msk(i, j, k) + wka(i, j, k);
  }

  /* int_readyc, mod_int.f90:90-151; op_fri, mod_op.f90:169-184 */
  void int_readyc() {
    A3 wkx, wky, sch;
    /* gra_r2d_b(bnd%pa%v, bnd%pa%hg=g1j, wkx, wky) */
    gra(wkx, wky, bnd_pa, g1j, *g1j.ew, *g1j.ns);
    ter(pax, wkx, *g1j.ew, g3j);
    ter(pay, wky, *g1j.ns, g3j);
    ter(sch, chc, g1j, g3j, 1.0);
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni; ++i) {
        sch(i, j) = std::sqrt(sch(i, j));
        if (g32.lev(i, j) == 0) sch(i, j) = 1.0;
      }
    upwelling();
    aupp = aup; avpp = avp; aup = auc; avp = avc;
    op_adv(auc, uc, sch);
    op_adv(avc, vc, sch);
    if (rst != 1) {
      if (iter == 1) { aupp = auc; avpp = avc; aup = auc; avp = avc; }
      else if (iter == 2) { aupp = aup; avpp = avp; }
    }
    /* op_fri */
    A3 u(ni, nj, nk), v(ni, nj, nk), mv(ni, nj, nk);
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) {
          u(i, j, k) = uc(i, j, k) / sch(i, j);
          v(i, j, k) = vc(i, j, k) / sch(i, j);
          mv(i, j, k) = -v(i, j, k);
        }
    fri_r3d(fx, sch, u, uc, mv, bnd_taux);
    fri_r3d(fy, sch, v, vc, u, bnd_tauy);
    ut.init(ni, nj, 1, 0.0);
    vt.init(ni, nj, 1, 0.0);
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) {
          double wx = -auc(i, j, k) - sch(i, j) * C.a0 * pax(i, j) + fx(i, j, k);
          double wy = -avc(i, j, k) - sch(i, j) * C.a0 * pay(i, j) + fy(i, j, k);
          ut(i, j) = ut(i, j) + wx * gi2.dpr[k] * g32.msk(i, j, k);
          vt(i, j) = vt(i, j) + wy * gi2.dpr[k] * g32.msk(i, j, k);
        }
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni; ++i) {
        ut(i, j) = ut(i, j) / g32.prh(i, j);
        vt(i, j) = vt(i, j) / g32.prh(i, j);
      }
  }

  /* int_trop, mod_int.f90:153-296 */
  void int_trop() {
    A3 ua(ni, nj), va(ni, nj); /* upbaccu */
    A3 s1(ni, nj), s2(ni, nj), wk, sch(ni, nj), l1, l2, vs1(ni, nj), vs2(ni, nj), v01(ni, nj), v02(ni, nj);
    A3 gx, gy, gi1_(ni, nj), gi2_(ni, nj), cg1(ni, nj), cg2(ni, nj), pg1(ni, nj), pg2(ni, nj);
    ua = ubc; va = vbc;
    mch = chc; mch2 = chc;
    const int nstep = bc / bt * 2;
    for (int nt = 1; nt <= nstep; ++nt) {
      sch.fill(1.0);
      ter(wk, chp, g1j, g3j);
      PAR for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i)
          if (g32.lev(i, j) > 0) sch(i, j) = std::sqrt(wk(i, j));
      PAR for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) {
          s1(i, j) = g32.prh(i, j) * sch(i, j) * ubp(i, j);
          s2(i, j) = g32.prh(i, j) * sch(i, j) * vbp(i, j);
        }
      div(wk, s1, s2, g3j, g3j, g1j);
      PAR for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) {
          double w = chp(i, j) - wk(i, j) * bt * C.gamma_b / g12.prh(i, j);
          if (g12.lev(i, j) > 0) chc(i, j) = w;
        }
      ter(wk, chc, g1j, g3j);
      PAR for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i)
          if (g32.lev(i, j) > 0) sch(i, j) = std::sqrt(wk(i, j));
      lap(l1, ubp, g3j, g3j);
      lap(l2, vbp, g3j, g3j);
      PAR for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) {
          int seau = g32.msk(i, j, 1);
          vs1(i, j) = seau * am(i, j, 1) * l1(i, j);
          vs2(i, j) = seau * am(i, j, 1) * l2(i, j);
        }
      if (nt == 1) { v01 = vs1; v02 = vs2; }
      gra(gx, gy, chc, g1j, *g1j.ew, *g1j.ns);
      gi1_.fill(0.0); /* row nj never written by the reference (see header) */
      PAR for (int j = 1; j <= njm; ++j)
        for (int i = 1; i <= ni; ++i)
          gi1_(i, j) = 0.5 * (gx(i, j) * bphi_xn(i, j) + gx(i, j + 1) * bphi_xs(i, j + 1));
      PAR for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= nim; ++i)
          gi2_(i, j) = 0.5 * (gy(i, j) * bphi_ye(i, j) + gy(i + 1, j) * bphi_yw(i + 1, j));
      swp(gi1_); swp(gi2_);
      ter(wk, chc, g1j, *g1j.ew);
      cg1.fill(0.0);
      PAR for (int j = 1; j <= njm; ++j)
        for (int i = 1; i <= ni; ++i)
          cg1(i, j) = 0.5 * (wk(i, j) * bgra_xn(i, j) + wk(i, j + 1) * bgra_xs(i, j + 1));
      ter(wk, chc, g1j, *g1j.ns);
      PAR for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= nim; ++i)
          cg2(i, j) = 0.5 * (wk(i, j) * bgra_ye(i, j) + wk(i + 1, j) * bgra_yw(i + 1, j));
      swp(cg1); swp(cg2);
      PAR for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) {
          int seau = g32.msk(i, j, 1);
          pg1(i, j) = (gi1_(i, j) + cg1(i, j) + graphihx(i, j)) * seau * sch(i, j);
          pg2(i, j) = (gi2_(i, j) + cg2(i, j) + graphihy(i, j)) * seau * sch(i, j);
        }
      PAR for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) {
          int seau = g32.msk(i, j, 1);
          double p1_ = seau * (vs1(i, j) - v01(i, j) + ut(i, j) - pg1(i, j) + 0.5 * cor(i, j) * vbp(i, j));
          double p2_ = seau * (vs2(i, j) - v02(i, j) + vt(i, j) - pg2(i, j) - 0.5 * cor(i, j) * ubp(i, j));
          double w1 = p1_ * bt + ubp(i, j);
          double w2 = p2_ * bt + vbp(i, j);
          double cb = 0.5 * cor(i, j) * bt;
          double u_ = (w1 + 0.5 * cor(i, j) * bt * w2) / (1 + cb * cb);
          double v_ = (w2 - 0.5 * cor(i, j) * bt * w1) / (1 + cb * cb);
          u_ = 0.5 * (u_ + ubp(i, j));
          v_ = 0.5 * (v_ + vbp(i, j));
          p1_ = seau * (vs1(i, j) - v01(i, j) - pg1(i, j) + ut(i, j) + cor(i, j) * v_);
          p2_ = seau * (vs2(i, j) - v02(i, j) - pg2(i, j) + vt(i, j) - cor(i, j) * u_);
          ubc(i, j) = p1_ * bt + ubp(i, j);
          vbc(i, j) = p2_ * bt + vbp(i, j);
        }
      ubp = ubc; vbp = vbc;
      PAR for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) {
          s1(i, j) = g32.prh(i, j) * sch(i, j) * ubc(i, j);
          s2(i, j) = g32.prh(i, j) * sch(i, j) * vbc(i, j);
        }
      div(wk, s1, s2, g3j, g3j, g1j);
      PAR for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) chc(i, j) = chp(i, j) - g12.msk(i, j, 1) * wk(i, j) * bt / g12.prh(i, j);
      if (nt <= nstep / 2) {
        PAR for (long long q = 0; q < (long long)mch.v.size(); ++q) mch.v[q] = mch.v[q] + chc.v[q];
      }
      chp = chc;
      PAR for (long long q = 0; q < (long long)ua.v.size(); ++q) {
        ua.v[q] = ua.v[q] + ubc.v[q];
        va.v[q] = va.v[q] + vbc.v[q];
        mch2.v[q] = mch2.v[q] + chc.v[q];
      }
    }
    PAR for (long long q = 0; q < (long long)ua.v.size(); ++q) {
      ubc.v[q] = ua.v[q] / (nstep + 1);
      vbc.v[q] = va.v[q] / (nstep + 1);
      ubp.v[q] = ubc.v[q];
      vbp.v[q] = vbc.v[q];
      mch.v[q] = mch.v[q] / (nstep / 2 + 1);
      mch2.v[q] = mch2.v[q] / (nstep + 1);
      chc.v[q] = mch2.v[q];
      chp.v[q] = chc.v[q];
      acch.v[q] = acch.v[q] + chc.v[q];
    }
    n_ch += 1;
  }

  /* smag, mod_int.f90:403-440 */
  void smag(const A3 &u, const A3 &v) {
    PAR2 for (int k = 1; k <= nk; ++k)
      for (int j = 2; j <= nj - 1; ++j)
        for (int i = 2; i <= ni - 1; ++i) {
          double dx = C.a * (g4j.rh(i, j) * g4j.dx1(i, j) + g4j.rh(i + 1, j) * g4j.dx1(i + 1, j));
          double dy = C.a * (g2j.dx2(i, j) + g2j.dx2(i, j + 1));
          double dt = 4 * (u(i + 1, j, k) - u(i - 1, j, k)) / dx - 4 * (v(i, j + 1, k) - v(i, j - 1, k)) / dy +
                      v(i, j, k) * g3j.tn(i, j) / C.a;
          double ds = 4 * (v(i + 1, j, k) - v(i - 1, j, k)) / dx + 4 * (u(i, j + 1, k) - u(i, j - 1, k)) / dy -
                      u(i, j, k) * g3j.tn(i, j) / C.a;
          double cc = 0.5 * C.smag_c / C.pi * (0.5 * dx + 0.5 * dy);
          cc = cc * cc;
          double wk = cc * std::sqrt(dt * dt + ds * ds);
          double am_max = (dx * dx + dy * dy) / (4 * 8 * bc);
          am(i, j, k) = (wk < am_max) ? wk : am_max;
        }
    swp(am);
  }

  /* int_clin, mod_int.f90:298-401 */
  void int_clin() {
    A3 sch(ni, nj, 1, 1.0), wk(ni, nj), px, py, mx, my, tmp;
    ter(tmp, mch, g1j, g3j, 1.0);
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni; ++i)
        if (g32.lev(i, j) > 0) sch(i, j) = std::sqrt(tmp(i, j));
    gra(mx, my, mch, g1j, *g1j.ew, *g1j.ns); /* k-independent, same for every k */
    A3 ak(ni, nj), t1, t2;
    for (int k = 1; k <= nk; ++k) {
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) wk(i, j) = g12.phih(i, j) + mch(i, j) * adp(i, j, k);
      gra(px, py, wk, g1j, *g1j.ew, *g1j.ns);
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) ak(i, j) = alpha(i, j, k);
      ter(t1, ak, g1j, *g1j.ew);
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) px(i, j) = px(i, j) + t1(i, j) * gi2.pr[k] * mx(i, j);
      ter(t1, ak, g1j, *g1j.ns);
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) py(i, j) = py(i, j) + t1(i, j) * gi2.pr[k] * my(i, j);
      ter(t1, px, *g1j.ew, g3j);
      ter(t2, py, *g1j.ns, g3j);
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) {
          double p1_ = -(t1(i, j) + C.a0 * pax(i, j)) * sch(i, j);
          double p2_ = -(t2(i, j) + C.a0 * pay(i, j)) * sch(i, j);
          p1_ = p1_ - (C.c_tc * auc(i, j, k) + C.c_tp * aup(i, j, k) + C.c_tpp * aupp(i, j, k));
          p2_ = p2_ - (C.c_tc * avc(i, j, k) + C.c_tp * avp(i, j, k) + C.c_tpp * avpp(i, j, k));
          p1_ = p1_ + fx(i, j, k);
          p2_ = p2_ + fy(i, j, k);
          p1_ = p1_ + cor(i, j) * vc(i, j, k);
          p2_ = p2_ - cor(i, j) * uc(i, j, k);
          double w1 = p1_, w2 = p2_;
          double w = 0.5 * cor(i, j) * bc;
          p1_ = w1 + w * w2;
          p2_ = w2 - w * w1;
          w = 1 + w * w;
          p1_ = p1_ * g32.msk(i, j, k) / w;
          p2_ = p2_ * g32.msk(i, j, k) / w;
          uc(i, j, k) = up(i, j, k) + p1_ * bc;
          vc(i, j, k) = vp(i, j, k) + p2_ * bc;
        }
    }
    A3 w1, w2;
    vint(w1, uc, g32);
    vint(w2, vc, g32);
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i)
          if (g32.msk(i, j, k) > 0) {
            uc(i, j, k) = uc(i, j, k) - w1(i, j) + ubc(i, j);
            vc(i, j, k) = vc(i, j, k) - w2(i, j) + vbc(i, j);
          }
    up = uc; vp = vc;
    ter(tmp, mch2, g1j, g3j, 1.0);
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni; ++i) sch(i, j) = std::sqrt(tmp(i, j));
    A3 uu(ni, nj, nk), vv(ni, nj, nk);
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) {
          uu(i, j, k) = uc(i, j, k) * sch(i, j) / mch2(i, j);
          vv(i, j, k) = vc(i, j, k) * sch(i, j) / mch2(i, j);
        }
    PAR for (long long q = 0; q < (long long)uu.v.size(); ++q) {
      acu.v[q] = acu.v[q] + uu.v[q];
      acv.v[q] = acv.v[q] + vv.v[q];
    }
    n_uv += 1;
    smag(uu, vv);
  }

  /* int_ssh, mod_int.f90:602-624 */
  void int_ssh() {
    den_alpha(alpha, tp, sp, mch);
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni; ++i) {
        double s = 0.0;
        for (int k = 1; k <= nk; ++k) s = s + alpha(i, j, k) * gi2.dpr[k] * mch(i, j) * g12.msk(i, j, k);
        double ssh = s / C.g;
        ssh = g12.phih(i, j) / C.g + ssh;
        acssh(i, j) = acssh(i, j) + ssh;
      }
    n_ssh += 1;
  }

  /* op_adv_ts, mod_op.f90:280-325 */
  void op_adv_ts(A3 &ans, const A3 &var) {
    A3 sch, u1(ni, nj, nk), u2(ni, nj, nk), w1, w2, wa, wb, tmp(ni, nj, nk), wkp, wmp(ni, nj, nkp);
    ter(sch, chc, g1j, g3j, 1.0);
    PAR for (long long q = 0; q < (long long)sch.v.size(); ++q) { double &x = sch.v[q]; x = std::sqrt(x); }
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) {
          u1(i, j, k) = uc(i, j, k) * sch(i, j);
          u2(i, j, k) = vc(i, j, k) * sch(i, j) * g3j.rh(i, j);
        }
    p1(w1, var, g1j, *g1j.ew);
    p2(w2, var, g1j, *g1j.ns);
    ter(wa, u1, g3j, *g1j.ew);
    PAR for (long long q = 0; q < (long long)tmp.v.size(); ++q) tmp.v[q] = wa.v[q] * w1.v[q];
    ter(wb, tmp, *g1j.ew, g1j);
    ans.init(ni, nj, nk);
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) ans(i, j, k) = wb(i, j, k) / (C.a * g1j.rh(i, j));
    ter(wa, u2, g3j, *g1j.ns);
    PAR for (long long q = 0; q < (long long)tmp.v.size(); ++q) tmp.v[q] = wa.v[q] * w2.v[q];
    ter(wb, tmp, *g1j.ns, g1j);
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) ans(i, j, k) = ans(i, j, k) + wb(i, j, k) / (C.a * g1j.rh(i, j));
    dx3(wkp, var);
    PAR for (long long q = 0; q < (long long)wmp.v.size(); ++q) wmp.v[q] = wm.v[q] * wkp.v[q];
    vter(wa, wmp, false);
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) ans(i, j, k) = ans(i, j, k) + wa(i, j, k) / gi2.dpr[k];
  }

  /* op_dif, mod_op.f90:186-222 */
  void op_dif(A3 &ans, const A3 &ch, const A3 &var) {
    A3 w1, w2, c1, c2, wk, va(ni, nj, nk), vb(ni, nj, nk), wkp;
    p1(w1, var, g1j, *g1j.ew, &g12.msk);
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) w1(i, j, k) = w1(i, j, k) / (C.a * g2j.rh(i, j));
    p2(w2, var, g1j, *g1j.ns, &g12.msk);
    PAR for (long long q = 0; q < (long long)w2.v.size(); ++q) { double &x = w2.v[q]; x = x / C.a; }
    ter(c1, ch, g1j, *g1j.ew);
    ter(c2, ch, g1j, *g1j.ns);
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) {
          va(i, j, k) = c1(i, j) * w1(i, j, k);
          vb(i, j, k) = c2(i, j) * w2(i, j, k);
        }
    div(wk, va, vb, *g1j.ew, *g1j.ns, g1j);
    ans.init(ni, nj, nk);
    PAR for (long long q = 0; q < (long long)wk.v.size(); ++q) ans.v[q] = C.ah_c * wk.v[q];
    pz(wkp, var, g12.msk);
    for (int k = 1; k <= nkp; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) wkp(i, j, k) = C.g * C.rho0 * kh(i, j, k) * wkp(i, j, k);
    p3(wk, wkp);
    PAR for (long long q = 0; q < (long long)ans.v.size(); ++q) ans.v[q] = ans.v[q] + wk.v[q];
  }

  /* mix, mod_int.f90:583-600 */
  void mix(std::vector<double> &rhoa, std::vector<double> &rhob, int na, int nb, int i, int j) {
    double st = 0.0, sd = 0.0, ss = 0.0;
    for (int k = na; k <= nb; ++k) st = st + tc(i, j, k) * gi2.dpr[k];
    for (int k = na; k <= nb; ++k) sd = sd + gi2.dpr[k];
    double tn = st / sd;
    for (int k = na; k <= nb; ++k) tc(i, j, k) = tn;
    for (int k = na; k <= nb; ++k) ss = ss + sc(i, j, k) * gi2.dpr[k];
    sd = 0.0;
    for (int k = na; k <= nb; ++k) sd = sd + gi2.dpr[k];
    double sn = ss / sd;
    for (int k = na; k <= nb; ++k) sc(i, j, k) = sn;
    for (int k = na; k <= nb; ++k) rhoa[k] = prho1(i, j, k) * tc(i, j, k) + prho2(i, j, k) * sc(i, j, k);
    for (int k = na; k <= nb - 1; ++k)
      rhob[k] = prho1(i, j, k + 1) * tc(i, j, k) + prho2(i, j, k + 1) * sc(i, j, k);
    if (nb < nk) rhob[nb] = prho1(i, j, nb + 1) * tc(i, j, nb) + prho2(i, j, nb + 1) * sc(i, j, nb);
  }
  /* adjust, mod_int.f90:544-581 */
  void adjust(std::vector<double> &rhoa, std::vector<double> &rhob, int &kcnt, int nlev, int i, int j) {
    int na = kcnt, nb = kcnt + 1;
    mix(rhoa, rhob, na, nb, i, j);
    while (nb < nlev) {
      if (rhob[nb] > rhoa[nb + 1]) {
        nb = nb + 1;
        mix(rhoa, rhob, na, nb, i, j);
      } else {
        if ((na <= 1) || (rhob[na - 1] <= rhoa[na])) break;
        na = na - 1;
        mix(rhoa, rhob, na, nb, i, j);
      }
    }
    while (na > 1) {
      if (rhob[na - 1] <= rhoa[na]) break;
      na = na - 1;
      mix(rhoa, rhob, na, nb, i, j);
    }
    kcnt = nb;
  }
  /* convect, mod_int.f90:509-542 */
  void convect() {
    PAR for (int i = 1; i <= ni; ++i) {
      std::vector<double> rhoa(nk + 2), rhob(nk + 2);
      for (int j = 1; j <= nj; ++j) {
        int nlev = g12.lev(i, j);
        if (nlev > 1) {
          std::fill(rhoa.begin(), rhoa.end(), 0.0);
          std::fill(rhob.begin(), rhob.end(), 0.0);
          for (int k = 2; k <= nlev; ++k) rhoa[k] = prho1(i, j, k) * tc(i, j, k) + prho2(i, j, k) * sc(i, j, k);
          for (int k = 1; k <= nlev - 1; ++k)
            rhob[k] = prho1(i, j, k + 1) * tc(i, j, k) + prho2(i, j, k + 1) * sc(i, j, k);
          int kcnt = 1;
          while (kcnt < nlev) {
            if (rhob[kcnt] > rhoa[kcnt + 1]) adjust(rhoa, rhob, kcnt, nlev, i, j);
            else kcnt = kcnt + 1;
          }
        }
      }
    }
  }

  /* int_ts, mod_int.f90:442-507 */
  void int_ts() {
    upwelling();
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i)
          acw(i, j, k) = acw(i, j, k) + wm(i, j, k) * alpha(i, j, k) / (C.g * mch2(i, j));
    n_w += 1;
    A3 a1, a2, d1, d2;
    op_adv_ts(a1, tc);
    op_adv_ts(a2, sc);
    op_dif(d1, mch, tp);
    op_dif(d2, mch, sp);
    A3 p1_(ni, nj, nk), p2_(ni, nj, nk);
    PAR for (long long q = 0; q < (long long)p1_.v.size(); ++q) {
      p1_.v[q] = -a1.v[q];
      p2_.v[q] = -a2.v[q];
      p1_.v[q] = p1_.v[q] + d1.v[q];
      p2_.v[q] = p2_.v[q] + d2.v[q];
    }
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni; ++i) {
        double pb = C.gamma_t * (bnd_t(i, j) - tc(i, j, 1)) * g12.msk(i, j, 1) / gi2.dpr[1];
        p1_(i, j, 1) = p1_(i, j, 1) + pb;
        pb = C.gamma_s * (bnd_s(i, j) - sc(i, j, 1)) * g12.msk(i, j, 1) * mch(i, j);
        p2_(i, j, 1) = p2_(i, j, 1) + pb;
      }
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) {
          tc(i, j, k) = tp(i, j, k) + p1_(i, j, k) * bc * g12.msk(i, j, k) / mch(i, j);
          sc(i, j, k) = sp(i, j, k) + p2_(i, j, k) * bc * g12.msk(i, j, k) / mch(i, j);
        }
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i)
          if (g12.msk(i, j, k) > 0 && tc(i, j, k) < C.tice) tc(i, j, k) = C.tice;
    convect();
    tp = tc; sp = sc;
    PAR for (long long q = 0; q < (long long)act.v.size(); ++q) {
      act.v[q] = act.v[q] + tc.v[q];
      acs.v[q] = acs.v[q] + sc.v[q];
    }
    /* den_alpha(wk, tp, sp, chc) then acr = acr + 1.0/wk; land points of the
     * reference's wk are never written: acr is left unchanged there. */
    PAR2 for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i)
          if (g12.msk(i, j, k) == 1) {
            double w = 1.0 / den_rho(tp(i, j, k), sp(i, j, k), chc(i, j) * gi2.pr[k], r8);
            acr(i, j, k) = acr(i, j, k) + 1.0 / w;
          }
    n_ts += 1;
  }

  /* int_bnd, mod_int.f90:649-691 */
  void int_bnd() {
    int y = ct.y, m = ct.m, d = ct.d, m1, m2, days;
    double fct;
    if (d < 15) {
      m2 = m; m1 = m - 1;
      if (m == 1) m1 = 12;
      days = days_month(y, m1);
      fct = r8 ? ((days - 15.0 + d) / (days - 15.0 + 15))
               : (double)(((float)days - 15.0f + (float)d) / ((float)days - 15.0f + 15.0f));
    } else {
      m1 = m; m2 = m + 1;
      if (m == 12) m2 = 1;
      days = days_month(y, m1);
      fct = r8 ? ((d - 15.0) / (days - 15 + 15.0)) : (double)(((float)d - 15.0f) / ((float)(days - 15) + 15.0f));
    }
    auto lerp = [&](A3 &b, const A3 &f_) {
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) b(i, j) = (f_(i, j, m2) - f_(i, j, m1)) * fct + f_(i, j, m1);
    };
    lerp(bnd_taux, frc_taux); lerp(bnd_tauy, frc_tauy);
    lerp(bnd_t, frc_t); lerp(bnd_s, frc_s);
    lerp(bnd_pa, frc_pa); lerp(bnd_fw, frc_fw);
  }

  /* the body of the time loop, main.f90:158-238 (nm%out_per /= '6hour'; no
   * output(), which writes files) */
  void step() {
    iter += 1;
    if (iter == 1 || ct.d != pt.d) {
      int_bnd();
      nday += 1;
      den_prho();
    }
    den_alpha(alpha, tc, sc, chc);
    int_pgra();
    int_readyc();
    int_trop();
    int_clin();
    int_ssh();
    int_ts();
    pt = ct;
    ct = time_plus(ct, bc);
  }

  /* ------------------------------------------------------------ setup */
  void setup(const orc_inputs &in);
  void reg();
};

/* Setup, main.f90:86-150 and 252-704 restated for npx = npy = 1. */
void Model::setup(const orc_inputs &in) {
  r8 = in.r8;
  make_consts(C, r8);
  Lit lit{r8};
  glo_ni = in.glo_ni; glo_nj = in.glo_nj; nk = in.nk;
  bt = in.dtbt; bc = in.dtbc; rst = in.rst;
  /* param_set_my / get_neighbor (mod_param.f90:279-344) with px = py = 1 */
  ni = glo_ni + 2; nj = glo_nj + 2;
  nim = ni - 1; njm = nj - 1; nkp = nk + 1;

  /* arrays_allocate, mod_arrays.f90:142-352 */
  HG *gs[4] = {&g1j, &g2j, &g3j, &g4j};
  const int sis[4] = {0, 1, 1, 0}, sjs[4] = {0, 0, 1, 1};
  for (int q = 0; q < 4; ++q) {
    gs[q]->n = q + 1; gs[q]->si = sis[q]; gs[q]->sj = sjs[q];
    gs[q]->rh.init(ni, nj); gs[q]->tn.init(ni, nj); gs[q]->dx1.init(ni, nj); gs[q]->dx2.init(ni, nj);
  }
  /* link_grid_gi, mod_arrays.f90:554-582 */
  g1j.ns = &g4j; g1j.ew = &g2j; g1j.di = &g3j;
  g2j.ns = &g3j; g2j.ew = &g1j; g2j.di = &g4j;
  g3j.ns = &g2j; g3j.ew = &g4j; g3j.di = &g1j;
  g4j.ns = &g1j; g4j.ew = &g3j; g4j.di = &g2j;
  gi1.n = 1; gi1.init(nkp);
  gi2.n = 2; gi2.init(nk);
  g12.msk.init(ni, nj, nk); g12.lev.init(ni, nj); g12.phih.init(ni, nj); g12.prh.init(ni, nj);
  g32.msk.init(ni, nj, nk); g32.lev.init(ni, nj); g32.phih.init(ni, nj); g32.prh.init(ni, nj);
  act.init(ni, nj, nk); acs.init(ni, nj, nk); acu.init(ni, nj, nk); acv.init(ni, nj, nk);
  acw.init(ni, nj, nk); acr.init(ni, nj, nk); acssh.init(ni, nj); acch.init(ni, nj);
  tc.init(ni, nj, nk); sc.init(ni, nj, nk); tp.init(ni, nj, nk); sp.init(ni, nj, nk);
  auc.init(ni, nj, nk); aup.init(ni, nj, nk); aupp.init(ni, nj, nk);
  avc.init(ni, nj, nk); avp.init(ni, nj, nk); avpp.init(ni, nj, nk);
  uc.init(ni, nj, nk); vc.init(ni, nj, nk); up.init(ni, nj, nk); vp.init(ni, nj, nk);
  fx.init(ni, nj, nk); fy.init(ni, nj, nk);
  frc_taux.init(ni, nj, 12); frc_tauy.init(ni, nj, 12); frc_t.init(ni, nj, 12);
  frc_s.init(ni, nj, 12); frc_pa.init(ni, nj, 12); frc_fw.init(ni, nj, 12);
  bnd_taux.init(ni, nj); bnd_tauy.init(ni, nj); bnd_t.init(ni, nj); bnd_s.init(ni, nj);
  bnd_pa.init(ni, nj); bnd_fw.init(ni, nj);
  alpha.init(ni, nj, nk, C.alpha_land);
  adp.init(ni, nj, nk); wm.init(ni, nj, nkp);
  am.init(ni, nj, nk, C.am_c); km.init(ni, nj, nkp, C.km_c); kh.init(ni, nj, nkp);
  graphihx.init(ni, nj); graphihy.init(ni, nj); pax.init(ni, nj); pay.init(ni, nj);
  chc.init(ni, nj, 1, 1.0); chp.init(ni, nj, 1, 1.0); mch.init(ni, nj, 1, 1.0); mch2.init(ni, nj, 1, 1.0);
  cor.init(ni, nj);
  ubc.init(ni, nj); vbc.init(ni, nj); ubp.init(ni, nj); vbp.init(ni, nj); ut.init(ni, nj); vt.init(ni, nj);
  prho1.init(ni, nj, nk); prho2.init(ni, nj, nk);
  hposx.init(ni, nj, 4); hposy.init(ni, nj, 4);
  cv1.init(ni, nj); cv2.init(ni, nj);
  bphi_xn.init(ni, nj); bphi_xs.init(ni, nj); bphi_ye.init(ni, nj); bphi_yw.init(ni, nj);
  bgra_xn.init(ni, nj); bgra_xs.init(ni, nj); bgra_ye.init(ni, nj); bgra_yw.init(ni, nj);
  lon.assign(ni + 1, 0.0); lat.assign(nj + 1, 0.0); z.assign(nk + 1, 0.0);

  /* init(), main.f90:292-308: mympi_divy / mympi_divx */
  for (int k = 1; k <= nk; ++k) z[k] = in.z[k - 1];
  for (int j = 2; j <= nj - 1; ++j) lat[j] = in.lat[j - 2];
  lat[1] = 2 * lat[2] - lat[3];
  lat[nj] = 2 * lat[njm] - lat[nj - 2];
  for (int i = 2; i <= ni - 1; ++i) lon[i] = in.lon[i - 2];
  lon[1] = lon[ni - 1]; lon[ni] = lon[2];

  /* set_cf, main.f90:312-345 */
  {
    A3 gkh(glo_ni, glo_nj, nkp, 0.0);
    const float miss_thr = 9.0e+30f - 1.0f;
    for (int k = 2; k <= nkp; ++k)
      for (int j = 1; j <= glo_nj; ++j)
        for (int i = 1; i <= glo_ni; ++i)
          gkh(i, j, k) = in.vmix ? in.vmix[(size_t)(i - 1) + (size_t)glo_ni * ((j - 1) + (size_t)glo_nj * (k - 2))]
                                 : 9.96920996838687e+36;
    const double thr = r8 ? 9.0e+30 - 1.0 : (double)miss_thr;
    PAR for (long long q = 0; q < (long long)gkh.v.size(); ++q) { double &x = gkh.v[q]; if (x > thr) x = L(0.1); }
    PAR for (long long q = 0; q < (long long)gkh.v.size(); ++q) { double &x = gkh.v[q]; if (x > L(200.0)) x = L(200.0); }
    PAR for (long long q = 0; q < (long long)gkh.v.size(); ++q) { double &x = gkh.v[q]; x = x * L(1.0e-4); }
    for (int k = 1; k <= nkp; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) km(i, j, k) = C.km_c;
    double pf[12] = {L(0.1), L(50.0), L(50.0), L(50.0), L(40.0), L(20.0),
                     L(10.0), L(5.0), L(2.0), L(1.0), L(0.5), L(0.2)};
    for (int q = 0; q < 12; ++q) pf[q] = pf[q] * L(1.0e-4);
    for (int k = 1; k <= 12 && k <= nkp; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) km(i, j, k) = pf[k - 1];
    /* mympi_div: interior then halo exchange; rows 1, nj keep 0 */
    for (int k = 1; k <= nkp; ++k)
      for (int j = 1; j <= glo_nj; ++j)
        for (int i = 1; i <= glo_ni; ++i) kh(i + 1, j + 1, k) = gkh(i, j, k);
    swp(kh);
  }

  /* calc_hpos, main.f90:347-406 */
  for (int j = 2; j <= njm; ++j)
    for (int i = 2; i <= nim; ++i) {
      double loni = lon[i], latj = (lat[j] + lat[j - 1]) * 0.5;
      hposx(i, j, 1) = loni * C.torad; hposy(i, j, 1) = latj * C.torad;
      loni = (lon[i] + lon[i + 1]) * 0.5;
      if (lon[i + 1] < lon[i]) loni = (lon[i] + lon[i + 1] + 360) * 0.5;
      hposx(i, j, 2) = loni * C.torad; hposy(i, j, 2) = latj * C.torad;
      loni = (lon[i] + lon[i + 1]) * 0.5;
      if (lon[i + 1] < lon[i]) loni = (lon[i] + lon[i + 1] + 360) * 0.5;
      latj = lat[j];
      hposx(i, j, 3) = loni * C.torad; hposy(i, j, 3) = latj * C.torad;
      loni = lon[i]; latj = lat[j];
      hposx(i, j, 4) = loni * C.torad; hposy(i, j, 4) = latj * C.torad;
    }
  swp(hposx); swp(hposy);
  for (int q = 1; q <= 4; ++q)
    for (int i = 1; i <= ni; ++i) {
      hposx(i, 1, q) = 2 * hposx(i, 2, q) - hposx(i, 3, q);
      hposy(i, 1, q) = 2 * hposy(i, 2, q) - hposy(i, 3, q);
      hposx(i, nj, q) = 2 * hposx(i, nj - 1, q) - hposx(i, nj - 2, q);
      hposy(i, nj, q) = 2 * hposy(i, nj - 1, q) - hposy(i, nj - 2, q);
    }

  /* set_hgrid, main.f90:408-497 */
  const double wrap = L(360.0) * C.torad;
  for (int j = 2; j <= njm; ++j)
    for (int i = 2; i <= nim; ++i) {
      double d1 = hposx(i, j, 2) - hposx(i - 1, j, 2);
      if (d1 < 0) d1 = d1 + wrap;
      g1j.dx1(i, j) = d1; g1j.dx2(i, j) = hposy(i, j, 4) - hposy(i, j - 1, 4);
      d1 = hposx(i + 1, j, 1) - hposx(i, j, 1);
      if (d1 < 0) d1 = d1 + wrap;
      g2j.dx1(i, j) = d1; g2j.dx2(i, j) = hposy(i, j, 3) - hposy(i, j - 1, 3);
      d1 = hposx(i + 1, j, 4) - hposx(i, j, 4);
      if (d1 < 0) d1 = d1 + wrap;
      g3j.dx1(i, j) = d1; g3j.dx2(i, j) = hposy(i, j + 1, 2) - hposy(i, j, 2);
      d1 = hposx(i, j, 3) - hposx(i - 1, j, 3);
      if (d1 < 0) d1 = d1 + wrap;
      g4j.dx1(i, j) = d1; g4j.dx2(i, j) = hposy(i, j + 1, 1) - hposy(i, j, 1);
    }
  for (int q = 0; q < 4; ++q) {
    HG &G = *gs[q];
    swp(G.dx1); swp(G.dx2);
    for (int i = 1; i <= ni; ++i) {
      G.dx1(i, 1) = 2 * G.dx1(i, 2) - G.dx1(i, 3);
      G.dx2(i, 1) = 2 * G.dx2(i, 2) - G.dx2(i, 3);
      G.dx1(i, nj) = 2 * G.dx1(i, nj - 1) - G.dx1(i, nj - 2);
      G.dx2(i, nj) = 2 * G.dx2(i, nj - 1) - G.dx2(i, nj - 2);
    }
  }
  for (int q = 0; q < 4; ++q)
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni; ++i) {
        gs[q]->rh(i, j) = std::cos(hposy(i, j, q + 1));
        gs[q]->tn(i, j) = std::tan(hposy(i, j, q + 1));
      }

  /* set_vgrid, main.f90:499-583 */
  {
    std::vector<double> dz(nk + 1), rmn(nk + 1), pmn(nk + 1), tmn(nk + 1), smn(nk + 1);
    for (int k = 1; k <= nk; ++k) { tmn[k] = in.tmn[k - 1]; smn[k] = in.smn[k - 1]; }
    dz[1] = 2 * z[1];
    for (int k = 2; k <= nk; ++k) dz[k] = 2 * (z[k] - z[k - 1]) - dz[k - 1];
    double pmnbot = 1.0;
    for (int k = 1; k <= nk; ++k) { pmn[k] = 0.0; rmn[k] = C.rho0; }
    const double tol = L(1e-6);
    int it = 0;
    while (std::fabs(pmn[nk] - pmnbot) > tol) {
      pmnbot = pmn[nk];
      rmn[1] = den_rho(tmn[1], smn[1], pmn[1] * 0.5, r8);
      for (int k = 2; k <= nk; ++k) rmn[k] = den_rho(tmn[k], smn[k], (pmn[k - 1] + pmn[k]) * 0.5, r8);
      pmn[1] = rmn[1] * C.g * dz[1];
      for (int k = 2; k <= nk; ++k) pmn[k] = rmn[k] * C.g * dz[k] + pmn[k - 1];
      if (++it > 100000) { fprintf(stderr, "set_vgrid: no convergence\n"); break; }
    }
    gi1.z[1] = 0.0;
    for (int k = 2; k <= nkp; ++k) gi1.z[k] = gi1.z[k - 1] + dz[k - 1];
    for (int k = 1; k <= nk; ++k) gi2.z[k] = z[k];
    gi1.pr[1] = 0.0;
    for (int k = 2; k <= nkp; ++k) gi1.pr[k] = pmn[k - 1];
    gi2.pr[1] = pmn[1] * 0.5;
    for (int k = 2; k <= nk; ++k) gi2.pr[k] = (pmn[k] + pmn[k - 1]) * 0.5;
    for (int k = 1; k <= nkp; ++k) gi1.dz[k] = 0.0;
    gi1.dz[1] = 0.5 * dz[1];
    for (int k = 2; k <= nk; ++k) gi1.dz[k] = z[k] - z[k - 1];
    gi1.dz[nkp] = gi1.dz[nk];
    for (int k = 1; k <= nk; ++k) gi2.dz[k] = dz[k];
    gi1.dpr[1] = 0.5 * pmn[1];
    for (int k = 2; k <= nk; ++k) gi1.dpr[k] = gi2.pr[k] - gi2.pr[k - 1];
    gi1.dpr[nkp] = gi1.dpr[nk];
    gi2.dpr[1] = pmn[1];
    for (int k = 2; k <= nk; ++k) gi2.dpr[k] = pmn[k] - pmn[k - 1];
  }

  /* set_grid, main.f90:585-659 */
  for (int j = 1; j <= glo_nj; ++j)
    for (int i = 1; i <= glo_ni; ++i) g12.lev(i + 1, j + 1) = in.itn[(size_t)(i - 1) + (size_t)glo_ni * (j - 1)];
  swpi(g12.lev);
  for (int k = 1; k <= nk; ++k)
    for (int j = 2; j <= njm; ++j)
      for (int i = 2; i <= nim; ++i)
        if (g12.lev(i, j) >= k) g12.msk(i, j, k) = 1;
  swpi(g12.msk);
  for (int k = 1; k <= nk; ++k)
    for (int j = 1; j <= njm; ++j)
      for (int i = 1; i <= nim; ++i)
        g32.msk(i, j, k) = g12.msk(i, j, k) * g12.msk(i + 1, j, k) * g12.msk(i, j + 1, k) * g12.msk(i + 1, j + 1, k);
  swpi(g32.msk);
  for (int j = 1; j <= nj; ++j)
    for (int i = 1; i <= ni; ++i) {
      int s = 0;
      for (int k = 1; k <= nk; ++k) s += g32.msk(i, j, k);
      g32.lev(i, j) = s;
    }
  {
    std::vector<double> phimn(nk + 1);
    phimn[1] = -C.g * gi2.dz[1];
    for (int k = 2; k <= nk; ++k) phimn[k] = phimn[k - 1] - C.g * gi2.dz[k];
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni; ++i) {
        int k = g12.lev(i, j);
        if (k == 0) g12.phih(i, j) = 0.0;
        else { g12.phih(i, j) = phimn[k]; g12.prh(i, j) = gi1.pr[k + 1]; }
        k = g32.lev(i, j);
        if (k == 0) g32.phih(i, j) = 0.0;
        else { g32.phih(i, j) = phimn[k]; g32.prh(i, j) = gi1.pr[k + 1]; }
      }
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni; ++i) {
        if (g12.lev(i, j) == 0) g12.prh(i, j) = L(0.1);
        if (g32.lev(i, j) == 0) g32.prh(i, j) = L(0.1);
      }
  }

  /* calc_cf, main.f90:661-673 */
  for (int j = 1; j <= nj; ++j)
    for (int i = 1; i <= ni; ++i) {
      double c3 = std::cos(hposy(i, j, 3));
      double temp = std::sqrt(1 - c3 * c3) / std::cos(hposy(i, j, 3));
      cv1(i, j) = (1 - temp * temp) / (C.a * C.a);
      cv2(i, j) = 2 * temp / C.a;
    }
  /* main.f90:119 (cor%hg = g3j) */
  for (int j = 1; j <= nj; ++j)
    for (int i = 1; i <= ni; ++i) cor(i, j) = 2.0 * C.omega * std::sin(hposy(i, j, 3));

  /* inistat, main.f90:675-704 */
  {
    const double *src[6] = {in.taux, in.tauy, in.bct, in.bcs, in.pa, in.fw};
    A3 *dst[6] = {&frc_taux, &frc_tauy, &frc_t, &frc_s, &frc_pa, &frc_fw};
    for (int q = 0; q < 6; ++q) {
      for (int m = 1; m <= 12; ++m)
        for (int j = 1; j <= glo_nj; ++j)
          for (int i = 1; i <= glo_ni; ++i)
            (*dst[q])(i + 1, j + 1, m) = src[q][(size_t)(i - 1) + (size_t)glo_ni * ((j - 1) + (size_t)glo_nj * (m - 1))];
      swp(*dst[q]);
    }
    const double miss = (double)(-9.99999e30f);
    PAR for (long long q = 0; q < (long long)frc_taux.v.size(); ++q)
      if (frc_taux.v[q] == miss) {
        frc_taux.v[q] = 0.0; frc_tauy.v[q] = 0.0; frc_t.v[q] = 0.0;
        frc_s.v[q] = 0.0; frc_pa.v[q] = 0.0; frc_fw.v[q] = 0.0;
      }
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= glo_nj; ++j)
        for (int i = 1; i <= glo_ni; ++i) {
          size_t q = (size_t)(i - 1) + (size_t)glo_ni * ((j - 1) + (size_t)glo_nj * (k - 1));
          tc(i + 1, j + 1, k) = in.pt[q];
          sc(i + 1, j + 1, k) = in.sa[q];
        }
    swp(tc); swp(sc);
    tp = tc; sp = sc;
    A3 wkx, wky;
    gra(wkx, wky, g12.phih, g1j, *g1j.ew, *g1j.ns);
    ter(graphihx, wkx, *g1j.ew, g3j);
    ter(graphihy, wky, *g1j.ns, g3j);
  }

  /* time prepare, main.f90:125-129 */
  ct = Time{in.year, in.month, in.day, in.hour, 0, 0, days_month(in.year, in.month)};
  pt = ct;
  iter = 0;
  reg();
}

void Model::reg() {
  f["tc"] = &tc; f["sc"] = &sc; f["tp"] = &tp; f["sp"] = &sp;
  f["uc"] = &uc; f["vc"] = &vc; f["up"] = &up; f["vp"] = &vp;
  f["auc"] = &auc; f["aup"] = &aup; f["aupp"] = &aupp; f["avc"] = &avc; f["avp"] = &avp; f["avpp"] = &avpp;
  f["fx"] = &fx; f["fy"] = &fy; f["pax"] = &pax; f["pay"] = &pay;
  f["ubc"] = &ubc; f["vbc"] = &vbc; f["ubp"] = &ubp; f["vbp"] = &vbp; f["ut"] = &ut; f["vt"] = &vt;
  f["chc"] = &chc; f["chp"] = &chp; f["mch"] = &mch; f["mch2"] = &mch2;
  f["am"] = &am; f["prho1"] = &prho1; f["prho2"] = &prho2; f["alpha"] = &alpha; f["adp"] = &adp; f["wm"] = &wm;
  f["bphi_xn"] = &bphi_xn; f["bphi_xs"] = &bphi_xs; f["bphi_ye"] = &bphi_ye; f["bphi_yw"] = &bphi_yw;
  f["bgraphi_xn"] = &bgra_xn; f["bgraphi_xs"] = &bgra_xs; f["bgraphi_ye"] = &bgra_ye; f["bgraphi_yw"] = &bgra_yw;
  f["act"] = &act; f["acs"] = &acs; f["acr"] = &acr; f["acu"] = &acu; f["acv"] = &acv; f["acw"] = &acw;
  f["acch"] = &acch; f["acssh"] = &acssh;
  f["cv1"] = &cv1; f["cv2"] = &cv2; f["cor"] = &cor; f["km"] = &km; f["kh"] = &kh;
  f["graphihx"] = &graphihx; f["graphihy"] = &graphihy;
  f["bnd_taux"] = &bnd_taux; f["bnd_tauy"] = &bnd_tauy; f["bnd_t"] = &bnd_t; f["bnd_s"] = &bnd_s;
  f["bnd_pa"] = &bnd_pa; f["bnd_fw"] = &bnd_fw;
  f["prh_t"] = &g12.prh; f["phih_t"] = &g12.phih; f["prh_u"] = &g32.prh; f["phih_u"] = &g32.phih;
  f["hposx"] = &hposx; f["hposy"] = &hposy;
  HG *gs[4] = {&g1j, &g2j, &g3j, &g4j};
  for (int q = 0; q < 4; ++q) {
    std::string s = std::to_string(q + 1);
    f["rh" + s] = &gs[q]->rh; f["tn" + s] = &gs[q]->tn; f["dx" + s + "x"] = &gs[q]->dx1; f["dx" + s + "y"] = &gs[q]->dx2;
  }
  fi["msk_t"] = &g12.msk; fi["lev_t"] = &g12.lev; fi["msk_u"] = &g32.msk; fi["lev_u"] = &g32.lev;
}

/* 1-D vertical grid vectors exposed as (1,1,n) arrays */
struct VecView { A3 a; };
std::map<void *, std::map<std::string, VecView>> g_vec;

} // namespace

extern "C" {

void *orc_create(const orc_inputs *in) {
  // the step allocates and frees whole-field temporaries (1-14 MB at 1
  // degree) all the time: keep them on the heap and reuse the pages instead
  // of mapping, faulting in and unmapping them on every call
  mallopt(M_MMAP_THRESHOLD, 32 << 20);
  mallopt(M_TRIM_THRESHOLD, 1 << 30);
  Model *m = new Model();
  m->setup(*in);
  return m;
}
void orc_destroy(void *m) { g_vec.erase(m); delete (Model *)m; }
void orc_step(void *m) { ((Model *)m)->step(); }
void orc_phase(void *mp, int phase) {
  Model *m = (Model *)mp;
  switch (phase) {
  case 0: m->int_bnd(); break;
  case 1: m->den_prho(); break;
  case 2: m->den_alpha(m->alpha, m->tc, m->sc, m->chc); break;
  case 3: m->int_pgra(); break;
  case 4: m->int_readyc(); break;
  case 5: m->int_trop(); break;
  case 6: m->int_clin(); break;
  case 7: m->int_ssh(); break;
  case 8: m->int_ts(); break;
  case 9: m->pt = m->ct; m->ct = time_plus(m->ct, m->bc); break;
  default: break;
  }
}
void orc_set_iter(void *m, int64_t i) { ((Model *)m)->iter = i; }
int64_t orc_get_iter(void *m) { return ((Model *)m)->iter; }

double *orc_field(void *mp, const char *name, int32_t *n1, int32_t *n2, int32_t *n3) {
  Model *m = (Model *)mp;
  std::string s(name);
  auto it = m->f.find(s);
  if (it != m->f.end()) {
    *n1 = it->second->n1; *n2 = it->second->n2; *n3 = it->second->n3;
    return it->second->v.data();
  }
  const std::vector<double> *vec = nullptr;
  if (s == "z1") vec = &m->gi1.z; else if (s == "pr1") vec = &m->gi1.pr;
  else if (s == "dz1") vec = &m->gi1.dz; else if (s == "dpr1") vec = &m->gi1.dpr;
  else if (s == "z2") vec = &m->gi2.z; else if (s == "pr2") vec = &m->gi2.pr;
  else if (s == "dz2") vec = &m->gi2.dz; else if (s == "dpr2") vec = &m->gi2.dpr;
  else if (s == "lon") vec = &m->lon; else if (s == "lat") vec = &m->lat;
  if (!vec) return nullptr;
  VecView &vv = g_vec[mp][s];
  vv.a.init((int)vec->size() - 1, 1, 1);
  for (size_t q = 1; q < vec->size(); ++q) vv.a.v[q - 1] = (*vec)[q];
  *n1 = vv.a.n1; *n2 = 1; *n3 = 1;
  return vv.a.v.data();
}
int32_t *orc_ifield(void *mp, const char *name, int32_t *n1, int32_t *n2, int32_t *n3) {
  Model *m = (Model *)mp;
  auto it = m->fi.find(name);
  if (it == m->fi.end()) return nullptr;
  *n1 = it->second->n1; *n2 = it->second->n2; *n3 = it->second->n3;
  return it->second->v.data();
}
double orc_const(void *mp, const char *name) {
  Model *m = (Model *)mp;
  std::string s(name);
  const Consts &C = m->C;
  if (s == "rho0") return C.rho0; if (s == "a0") return C.a0; if (s == "g") return C.g;
  if (s == "a") return C.a; if (s == "pi") return C.pi; if (s == "omega") return C.omega;
  if (s == "torad") return C.torad; if (s == "gamma_t") return C.gamma_t; if (s == "gamma_s") return C.gamma_s;
  if (s == "gamma_b") return C.gamma_b; if (s == "deltat") return C.deltat; if (s == "deltas") return C.deltas;
  if (s == "cdbot") return C.cdbot; if (s == "tice") return C.tice; if (s == "km_c") return C.km_c;
  if (s == "am_c") return C.am_c; if (s == "smag_c") return C.smag_c; if (s == "ah_c") return C.ah_c;
  if (s == "c_tc") return C.c_tc; if (s == "c_tp") return C.c_tp; if (s == "c_tpp") return C.c_tpp;
  if (s == "alpha_land") return C.alpha_land;
  if (s == "n_ts") return m->n_ts; if (s == "n_uv") return m->n_uv; if (s == "n_w") return m->n_w;
  if (s == "n_ch") return m->n_ch; if (s == "n_ssh") return m->n_ssh;
  if (s == "day") return m->ct.d; if (s == "month") return m->ct.m; if (s == "year") return m->ct.y;
  if (s == "hour") return m->ct.h;
  return NAN;
}
double orc_den_rho(double t, double s, double p0, int32_t r8) { return den_rho(t, s, p0, r8); }
void orc_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n);
#else
  (void)n;
#endif
}

} /* extern "C" */
