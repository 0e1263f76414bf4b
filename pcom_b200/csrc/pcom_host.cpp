// pcom_host.cpp -- the host driver (include/pcom_host.h): PCOM's one-time
// setup (main.f90:252-704) and time loop (main.f90:158-238) for a single
// domain, driving the device step through include/pcom_gpu.h.
//
// The setup is host work the reference does once, with transcendental
// functions (cos/tan/sin) and a fixed-point iteration; it is computed here in
// FP64 with the reference's evaluation order and literal precision, and its
// outputs are uploaded as the static data of the device step.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pcom_host.h"

namespace {

// default-REAL literal: REAL(4) rounding (gfortran) or REAL(8) (ifort -r8)
struct Lit {
  bool r8;
  double operator()(float f, double d) const { return r8 ? d : (double)f; }
};
#define LIT(x) lit((float)(x##f), (double)(x))

// a padded field, Fortran order, 1-based accessors
struct Fld {
  int n1 = 0, n2 = 0, n3 = 0;
  std::vector<double> v;
  void init(int a, int b, int c = 1, double x = 0.0) { n1 = a; n2 = b; n3 = c; v.assign((size_t)a * b * c, x); }
  double &operator()(int i, int j, int k = 1) { return v[(size_t)(i - 1) + (size_t)n1 * ((j - 1) + (size_t)n2 * (k - 1))]; }
  double operator()(int i, int j, int k = 1) const { return v[(size_t)(i - 1) + (size_t)n1 * ((j - 1) + (size_t)n2 * (k - 1))]; }
};
struct IFld {
  int n1 = 0, n2 = 0, n3 = 0;
  std::vector<int32_t> v;
  void init(int a, int b, int c = 1) { n1 = a; n2 = b; n3 = c; v.assign((size_t)a * b * c, 0); }
  int32_t &operator()(int i, int j, int k = 1) { return v[(size_t)(i - 1) + (size_t)n1 * ((j - 1) + (size_t)n2 * (k - 1))]; }
};

// x-halo exchange of a single domain: columns 1 and ni take ni-1 and 2
template <class F>
void halo_x(F &f) {
  for (int k = 1; k <= f.n3; ++k)
    for (int j = 1; j <= f.n2; ++j) {
      f(1, j, k) = f(f.n1 - 1, j, k);
      f(f.n1, j, k) = f(2, j, k);
    }
}

struct Date { int y, m, d, h, mi, s, mm; };
int year_days(int y) { return (y % 100 == 0) ? (y % 400 == 0 ? 366 : 365) : (y % 4 == 0 ? 366 : 365); }
int month_days(int y, int m) {
  static const int n[12] = {31, 28, 31, 30, 31, 30, 31, 31, 30, 31, 30, 31};
  return (m == 2 && year_days(y) == 366) ? 29 : n[m - 1];
}
// type_time + integer seconds (mod_type.f90:593-635)
Date advance(Date t, int dt) {
  t.s += dt;
  if (t.s >= 60) { t.mi += t.s / 60; t.s %= 60; }
  if (t.mi >= 60) { t.h += t.mi / 60; t.mi %= 60; }
  if (t.h >= 24) { t.d += t.h / 24; t.h %= 24; }
  if (t.d > t.mm) { t.m += 1; t.d = 1; }
  if (t.m > 12) { t.y += 1; t.m = 1; }
  t.mm = month_days(t.y, t.m);
  return t;
}

}  // namespace

struct pcom_model {
  bool r8 = false;
  int glo_ni, glo_nj, nk, ni, nj, nkp, bt, bc;
  Fld rh[4], tn[4], dx[4];  // dx AoS (2, ni, nj) stored as n1 = 2*ni
  std::vector<double> z1, pr1, dz1, dpr1, z2, pr2, dz2, dpr2;  // 0-based vectors
  IFld msk_t, lev_t, msk_u, lev_u;
  Fld phih_t, prh_t, phih_u, prh_u, cv1, cv2, cor, km, kh, graphihx, graphihy;
  Fld frc[6];   // taux, tauy, t, s, pa, fw (ni, nj, 12)
  Fld t0, s0;   // initial T, S
  Fld bnd[6];
  Date ct, pt;
  long long iter = 0, nday = 0;
  pcom_handle *h = nullptr;
};

namespace {

double dxv(const Fld &f, int comp, int i, int j) { return f.v[2 * ((size_t)(i - 1) + (size_t)(f.n1 / 2) * (j - 1)) + comp]; }
double &dxr(Fld &f, int comp, int i, int j) { return f.v[2 * ((size_t)(i - 1) + (size_t)(f.n1 / 2) * (j - 1)) + comp]; }

// den_rho (mod_den.f90:57-118) for the reference-profile iteration of set_vgrid
double eos_rho(bool r8, double t, double s, double p0) {
  Lit lit{r8};
  double p = p0 * LIT(1e-5);
  double p2 = p * p, t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
  double s32 = s * std::sqrt(s), s2 = s * s;
  double r0 = LIT(999.842594) + LIT(6.793952e-2) * t - LIT(9.095290e-3) * t2 + LIT(1.001685e-4) * t3 -
              LIT(1.120083e-6) * t4 + LIT(6.536336e-9) * t5;
  double a = LIT(8.24493e-1) - LIT(4.0899e-3) * t + LIT(7.6438e-5) * t2 - LIT(8.2467e-7) * t3 + LIT(5.3875e-9) * t4;
  double b = -LIT(5.72466e-3) + LIT(1.0227e-4) * t - LIT(1.6546e-6) * t2;
  double r = r0 + a * s + b * s32 + LIT(4.8314e-4) * s2;
  double k = LIT(1.965933e4) + LIT(1.444304e2) * t - LIT(1.706103) * t2 + LIT(9.648704e-3) * t3 -
             LIT(4.190253e-5) * t4 + (LIT(5.284855e1) - LIT(3.101089e-1) * t + LIT(6.283263e-3) * t2 - LIT(5.084188e-5) * t3) * s +
             (LIT(3.886640e-1) + LIT(9.085835e-3) * t - LIT(4.619924e-4) * t2) * s32 +
             (LIT(3.186519) + LIT(2.212276e-2) * t - LIT(2.984642e-4) * t2 + LIT(1.956415e-6) * t3) * p +
             (LIT(6.704388e-3) - LIT(1.847318e-4) * t + LIT(2.059331e-7) * t2) * s * p + LIT(1.480266e-4) * s32 * p +
             (LIT(2.102898e-4) - LIT(1.202016e-5) * t + LIT(1.394680e-7) * t2) * p2 +
             (-LIT(2.040237e-6) + LIT(6.128773e-8) * t + LIT(6.207323e-10) * t2) * s * p2;
  return r / (1.0 - p / k);
}

void setup(pcom_model &M, const pcom_case &c) {
  const bool r8 = M.r8;
  Lit lit{r8};
  const int ni = M.ni, nj = M.nj, nk = M.nk, nkp = M.nkp, nim = ni - 1, njm = nj - 1;
  const int gi = M.glo_ni, gj = M.glo_nj;
  const double g = LIT(9.8), a = LIT(6370e3), pi = LIT(3.141592653589793);
  const double torad = pi / LIT(180.0), omega = pi / LIT(43082.0), rho0 = LIT(1029.0);

  // local lon/lat with halos (init, main.f90:301-308)
  std::vector<double> lon(ni + 1, 0.0), lat(nj + 1, 0.0), z(nk + 1, 0.0);
  for (int k = 1; k <= nk; ++k) z[k] = c.z[k - 1];
  for (int j = 2; j <= nj - 1; ++j) lat[j] = c.lat[j - 2];
  lat[1] = 2 * lat[2] - lat[3];
  lat[nj] = 2 * lat[njm] - lat[nj - 2];
  for (int i = 2; i <= ni - 1; ++i) lon[i] = c.lon[i - 2];
  lon[1] = lon[ni - 1];
  lon[ni] = lon[2];

  // km, kh (set_cf, main.f90:312-345)
  M.km.init(ni, nj, nkp, LIT(1.0e-5));
  {
    const double pf0[12] = {LIT(0.1), LIT(50.0), LIT(50.0), LIT(50.0), LIT(40.0), LIT(20.0),
                            LIT(10.0), LIT(5.0), LIT(2.0), LIT(1.0), LIT(0.5), LIT(0.2)};
    for (int k = 1; k <= 12 && k <= nkp; ++k) {
      const double pf = pf0[k - 1] * LIT(1.0e-4);
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) M.km(i, j, k) = pf;
    }
    M.kh.init(ni, nj, nkp, 0.0);
    const double thr = r8 ? 9.0e+30 - 1.0 : (double)(9.0e+30f - 1.0f);
    for (int k = 2; k <= nkp; ++k)
      for (int j = 1; j <= gj; ++j)
        for (int i = 1; i <= gi; ++i) {
          double v = c.vmix ? c.vmix[(size_t)(i - 1) + (size_t)gi * ((j - 1) + (size_t)gj * (k - 2))] : 9.96920996838687e+36;
          if (v > thr) v = LIT(0.1);
          if (v > LIT(200.0)) v = LIT(200.0);
          M.kh(i + 1, j + 1, k) = v * LIT(1.0e-4);
        }
    halo_x(M.kh);
  }

  // positions of the four staggered grids (calc_hpos, main.f90:347-406)
  Fld hx, hy;
  hx.init(ni, nj, 4);
  hy.init(ni, nj, 4);
  for (int j = 2; j <= njm; ++j)
    for (int i = 2; i <= nim; ++i) {
      const double latc = (lat[j] + lat[j - 1]) * 0.5;
      double lone = (lon[i] + lon[i + 1]) * 0.5;
      if (lon[i + 1] < lon[i]) lone = (lon[i] + lon[i + 1] + 360) * 0.5;
      hx(i, j, 1) = lon[i] * torad; hy(i, j, 1) = latc * torad;
      hx(i, j, 2) = lone * torad;   hy(i, j, 2) = latc * torad;
      hx(i, j, 3) = lone * torad;   hy(i, j, 3) = lat[j] * torad;
      hx(i, j, 4) = lon[i] * torad; hy(i, j, 4) = lat[j] * torad;
    }
  halo_x(hx);
  halo_x(hy);
  for (int q = 1; q <= 4; ++q)
    for (int i = 1; i <= ni; ++i) {
      hx(i, 1, q) = 2 * hx(i, 2, q) - hx(i, 3, q);
      hy(i, 1, q) = 2 * hy(i, 2, q) - hy(i, 3, q);
      hx(i, nj, q) = 2 * hx(i, nj - 1, q) - hx(i, nj - 2, q);
      hy(i, nj, q) = 2 * hy(i, nj - 1, q) - hy(i, nj - 2, q);
    }

  // metric increments, Lame coefficients (set_hgrid, main.f90:408-497)
  for (int q = 0; q < 4; ++q) {
    M.rh[q].init(ni, nj);
    M.tn[q].init(ni, nj);
    M.dx[q].init(2 * ni, nj);
  }
  const double wrap = LIT(360.0) * torad;
  auto pos = [](double d, double w) { return d < 0 ? d + w : d; };
  for (int j = 2; j <= njm; ++j)
    for (int i = 2; i <= nim; ++i) {
      dxr(M.dx[0], 0, i, j) = pos(hx(i, j, 2) - hx(i - 1, j, 2), wrap);
      dxr(M.dx[0], 1, i, j) = hy(i, j, 4) - hy(i, j - 1, 4);
      dxr(M.dx[1], 0, i, j) = pos(hx(i + 1, j, 1) - hx(i, j, 1), wrap);
      dxr(M.dx[1], 1, i, j) = hy(i, j, 3) - hy(i, j - 1, 3);
      dxr(M.dx[2], 0, i, j) = pos(hx(i + 1, j, 4) - hx(i, j, 4), wrap);
      dxr(M.dx[2], 1, i, j) = hy(i, j + 1, 2) - hy(i, j, 2);
      dxr(M.dx[3], 0, i, j) = pos(hx(i, j, 3) - hx(i - 1, j, 3), wrap);
      dxr(M.dx[3], 1, i, j) = hy(i, j + 1, 1) - hy(i, j, 1);
    }
  for (int q = 0; q < 4; ++q) {
    Fld &D = M.dx[q];
    for (int j = 1; j <= nj; ++j)
      for (int cpt = 0; cpt < 2; ++cpt) {
        dxr(D, cpt, 1, j) = dxv(D, cpt, ni - 1, j);
        dxr(D, cpt, ni, j) = dxv(D, cpt, 2, j);
      }
    for (int i = 1; i <= ni; ++i)
      for (int cpt = 0; cpt < 2; ++cpt) {
        dxr(D, cpt, i, 1) = 2 * dxv(D, cpt, i, 2) - dxv(D, cpt, i, 3);
        dxr(D, cpt, i, nj) = 2 * dxv(D, cpt, i, nj - 1) - dxv(D, cpt, i, nj - 2);
      }
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni; ++i) {
        M.rh[q](i, j) = std::cos(hy(i, j, q + 1));
        M.tn[q](i, j) = std::tan(hy(i, j, q + 1));
      }
  }

  // vertical grids from the hydrostatic mean profile (set_vgrid, main.f90:499-583)
  {
    std::vector<double> dz(nk + 1), rmn(nk + 1, rho0), pmn(nk + 1, 0.0);
    dz[1] = 2 * z[1];
    for (int k = 2; k <= nk; ++k) dz[k] = 2 * (z[k] - z[k - 1]) - dz[k - 1];
    double pbot = 1.0;
    const double tol = LIT(1e-6);
    for (int it = 0; std::fabs(pmn[nk] - pbot) > tol && it < 100000; ++it) {
      pbot = pmn[nk];
      rmn[1] = eos_rho(r8, c.tmn[0], c.smn[0], pmn[1] * 0.5);
      for (int k = 2; k <= nk; ++k) rmn[k] = eos_rho(r8, c.tmn[k - 1], c.smn[k - 1], (pmn[k - 1] + pmn[k]) * 0.5);
      pmn[1] = rmn[1] * g * dz[1];
      for (int k = 2; k <= nk; ++k) pmn[k] = rmn[k] * g * dz[k] + pmn[k - 1];
    }
    M.z1.assign(nkp, 0.0); M.pr1.assign(nkp, 0.0); M.dz1.assign(nkp, 0.0); M.dpr1.assign(nkp, 0.0);
    M.z2.assign(nk, 0.0); M.pr2.assign(nk, 0.0); M.dz2.assign(nk, 0.0); M.dpr2.assign(nk, 0.0);
    for (int k = 2; k <= nkp; ++k) M.z1[k - 1] = M.z1[k - 2] + dz[k - 1];
    for (int k = 1; k <= nk; ++k) M.z2[k - 1] = z[k];
    for (int k = 2; k <= nkp; ++k) M.pr1[k - 1] = pmn[k - 1];
    M.pr2[0] = pmn[1] * 0.5;
    for (int k = 2; k <= nk; ++k) M.pr2[k - 1] = (pmn[k] + pmn[k - 1]) * 0.5;
    M.dz1[0] = 0.5 * dz[1];
    for (int k = 2; k <= nk; ++k) M.dz1[k - 1] = z[k] - z[k - 1];
    M.dz1[nkp - 1] = M.dz1[nk - 1];
    for (int k = 1; k <= nk; ++k) M.dz2[k - 1] = dz[k];
    M.dpr1[0] = 0.5 * pmn[1];
    for (int k = 2; k <= nk; ++k) M.dpr1[k - 1] = M.pr2[k - 1] - M.pr2[k - 2];
    M.dpr1[nkp - 1] = M.dpr1[nk - 1];
    M.dpr2[0] = pmn[1];
    for (int k = 2; k <= nk; ++k) M.dpr2[k - 1] = pmn[k] - pmn[k - 1];
  }

  // masks, levels, bottom pressure and geopotential (set_grid, main.f90:585-659)
  M.lev_t.init(ni, nj); M.msk_t.init(ni, nj, nk); M.lev_u.init(ni, nj); M.msk_u.init(ni, nj, nk);
  for (int j = 1; j <= gj; ++j)
    for (int i = 1; i <= gi; ++i) M.lev_t(i + 1, j + 1) = c.itn[(size_t)(i - 1) + (size_t)gi * (j - 1)];
  halo_x(M.lev_t);
  for (int k = 1; k <= nk; ++k)
    for (int j = 2; j <= njm; ++j)
      for (int i = 2; i <= nim; ++i) M.msk_t(i, j, k) = M.lev_t(i, j) >= k ? 1 : 0;
  halo_x(M.msk_t);
  for (int k = 1; k <= nk; ++k)
    for (int j = 1; j <= njm; ++j)
      for (int i = 1; i <= nim; ++i)
        M.msk_u(i, j, k) = M.msk_t(i, j, k) * M.msk_t(i + 1, j, k) * M.msk_t(i, j + 1, k) * M.msk_t(i + 1, j + 1, k);
  halo_x(M.msk_u);
  for (int j = 1; j <= nj; ++j)
    for (int i = 1; i <= ni; ++i) {
      int s = 0;
      for (int k = 1; k <= nk; ++k) s += M.msk_u(i, j, k);
      M.lev_u(i, j) = s;
    }
  {
    std::vector<double> phimn(nk + 1);
    phimn[1] = -g * M.dz2[0];
    for (int k = 2; k <= nk; ++k) phimn[k] = phimn[k - 1] - g * M.dz2[k - 1];
    M.phih_t.init(ni, nj); M.prh_t.init(ni, nj); M.phih_u.init(ni, nj); M.prh_u.init(ni, nj);
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni; ++i) {
        const int kt = M.lev_t(i, j), ku = M.lev_u(i, j);
        if (kt == 0) M.prh_t(i, j) = LIT(0.1);
        else { M.phih_t(i, j) = phimn[kt]; M.prh_t(i, j) = M.pr1[kt]; }
        if (ku == 0) M.prh_u(i, j) = LIT(0.1);
        else { M.phih_u(i, j) = phimn[ku]; M.prh_u(i, j) = M.pr1[ku]; }
      }
  }

  // friction coefficients and Coriolis (calc_cf, main.f90:661-673; main.f90:119)
  M.cv1.init(ni, nj); M.cv2.init(ni, nj); M.cor.init(ni, nj);
  for (int j = 1; j <= nj; ++j)
    for (int i = 1; i <= ni; ++i) {
      const double cs = std::cos(hy(i, j, 3));
      const double tt = std::sqrt(1 - cs * cs) / std::cos(hy(i, j, 3));
      M.cv1(i, j) = (1 - tt * tt) / (a * a);
      M.cv2(i, j) = 2 * tt / a;
      M.cor(i, j) = 2.0 * omega * std::sin(hy(i, j, 3));
    }

  // forcing and initial state (inistat, main.f90:675-704)
  const double *src[6] = {c.taux, c.tauy, c.bct, c.bcs, c.pa, c.fw};
  for (int q = 0; q < 6; ++q) {
    M.frc[q].init(ni, nj, 12);
    for (int m = 1; m <= 12; ++m)
      for (int j = 1; j <= gj; ++j)
        for (int i = 1; i <= gi; ++i)
          M.frc[q](i + 1, j + 1, m) = src[q][(size_t)(i - 1) + (size_t)gi * ((j - 1) + (size_t)gj * (m - 1))];
    halo_x(M.frc[q]);
  }
  const double miss = (double)(-9.99999e30f);
  for (size_t p = 0; p < M.frc[0].v.size(); ++p)
    if (M.frc[0].v[p] == miss)
      for (int q = 0; q < 6; ++q) M.frc[q].v[p] = 0.0;
  M.t0.init(ni, nj, nk); M.s0.init(ni, nj, nk);
  for (int k = 1; k <= nk; ++k)
    for (int j = 1; j <= gj; ++j)
      for (int i = 1; i <= gi; ++i) {
        const size_t p = (size_t)(i - 1) + (size_t)gi * ((j - 1) + (size_t)gj * (k - 1));
        M.t0(i + 1, j + 1, k) = c.pt[p];
        M.s0(i + 1, j + 1, k) = c.sa[p];
      }
  halo_x(M.t0);
  halo_x(M.s0);
  // graphihx/y = ter(gra(phih)) on the U grid
  {
    Fld gx, gy;
    gx.init(ni, nj); gy.init(ni, nj);
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= nim; ++i) gx(i, j) = M.phih_t(i + 1, j) - M.phih_t(i, j);
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni; ++i) gx(i, j) = gx(i, j) / dxv(M.dx[1], 0, i, j);
    halo_x(gx);
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni; ++i) gx(i, j) = gx(i, j) / (a * M.rh[1](i, j));
    for (int j = 1; j <= njm; ++j)
      for (int i = 1; i <= ni; ++i) gy(i, j) = M.phih_t(i, j + 1) - M.phih_t(i, j);
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni; ++i) gy(i, j) = gy(i, j) / dxv(M.dx[3], 1, i, j);
    halo_x(gy);
    for (auto &v : gy.v) v = v / a;
    M.graphihx.init(ni, nj); M.graphihy.init(ni, nj);
    for (int j = 1; j <= njm; ++j)
      for (int i = 1; i <= ni; ++i) M.graphihx(i, j) = 0.5 * (gx(i, j) + gx(i, j + 1));
    halo_x(M.graphihx);
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= nim; ++i) M.graphihy(i, j) = 0.5 * (gy(i, j) + gy(i + 1, j));
    halo_x(M.graphihy);
  }
  for (int q = 0; q < 6; ++q) M.bnd[q].init(ni, nj);
  M.ct = Date{c.year, c.month, c.day, c.hour, 0, 0, month_days(c.year, c.month)};
  M.pt = M.ct;
}

// int_bnd (mod_int.f90:649-691): monthly forcing interpolated to the day
// the months and weight of int_bnd (mod_int.f90:649-691) at the model date
void bnd_weights(const pcom_model &M, int &m1, int &m2, double &f) {
  const int y = M.ct.y, m = M.ct.m, d = M.ct.d;
  if (d < 15) {
    m2 = m;
    m1 = (m == 1) ? 12 : m - 1;
    const int days = month_days(y, m1);
    f = M.r8 ? (days - 15.0 + d) / (days - 15.0 + 15)
             : (double)(((float)days - 15.0f + (float)d) / ((float)days - 15.0f + 15.0f));
  } else {
    m1 = m;
    m2 = (m == 12) ? 1 : m + 1;
    const int days = month_days(y, m1);
    f = M.r8 ? (d - 15.0) / (days - 15 + 15.0) : (double)(((float)d - 15.0f) / ((float)(days - 15) + 15.0f));
  }
}

void int_bnd(pcom_model &M) {
  int m1, m2;
  double f;
  bnd_weights(M, m1, m2, f);
  for (int q = 0; q < 6; ++q)
    for (int j = 1; j <= M.nj; ++j)
      for (int i = 1; i <= M.ni; ++i)
        M.bnd[q](i, j) = (M.frc[q](i, j, m2) - M.frc[q](i, j, m1)) * f + M.frc[q](i, j, m1);
}

std::string g_err;

}  // namespace

extern "C" {

int pcom_model_create(const pcom_case *c, int32_t flags, pcom_model **out) {
  if (!c || !out) return PCOM_ERR_ARG;
  // rst = 1: the setup is the same; the caller then loads the restart state
  // (pcom_gpu_set_state) and the AB3 start-up is skipped (mod_int.f90:122-132)
  if (c->rst != 0 && c->rst != 1) return PCOM_ERR_ARG;
  pcom_model *M = new pcom_model();
  M->r8 = c->r8 != 0;
  M->glo_ni = c->glo_ni; M->glo_nj = c->glo_nj; M->nk = c->nk;
  M->ni = c->glo_ni + 2; M->nj = c->glo_nj + 2; M->nkp = c->nk + 1;
  M->bt = c->dtbt; M->bc = c->dtbc;
  if (M->glo_ni < 2 || M->glo_nj < 2 || M->nk < 2) { delete M; return PCOM_ERR_ARG; }
  setup(*M, *c);
  if (flags & PCOM_MODEL_HOST_ONLY) {
    *out = M;
    return PCOM_OK;
  }
  pcom_dims d{};
  d.glo_ni = M->glo_ni; d.glo_nj = M->glo_nj; d.nk = M->nk; d.ni = M->ni; d.nj = M->nj;
  d.dtbt = M->bt; d.dtbc = M->bc; d.flags = flags | (M->r8 ? PCOM_LIT_R8 : 0); d.rst = c->rst;
  int rc = pcom_gpu_create(&d, &M->h);
  if (rc) { delete M; return rc; }
  pcom_static s{};
  pcom_model_static(M, &s);
  rc = pcom_gpu_upload_static(M->h, &s);
  if (!rc) {
    pcom_state st{};
    st.tc = M->t0.v.data(); st.sc = M->s0.v.data();
    rc = pcom_gpu_set_state(M->h, &st);
  }
  if (!rc) {
    // the 12 monthly forcing fields, for int_bnd on the device
    pcom_forcing mo{M->frc[0].v.data(), M->frc[1].v.data(), M->frc[2].v.data(),
                    M->frc[3].v.data(), M->frc[4].v.data(), M->frc[5].v.data()};
    rc = pcom_gpu_set_forcing_months(M->h, &mo);
  }
  if (rc) { pcom_gpu_destroy(M->h); delete M; return rc; }
  *out = M;
  return PCOM_OK;
}

int pcom_model_destroy(pcom_model *m) {
  if (!m) return PCOM_OK;
  pcom_gpu_destroy(m->h);
  delete m;
  return PCOM_OK;
}

pcom_handle *pcom_model_handle(pcom_model *m) { return m ? m->h : nullptr; }

int pcom_model_begin_step(pcom_model *M, int64_t *it, int32_t *new_day) {
  if (!M || !it || !new_day) return PCOM_ERR_ARG;
  if (!M->h) return PCOM_ERR_STATE;
  M->iter += 1;
  *it = M->iter;
  *new_day = 0;
  if (M->iter == 1 || M->ct.d != M->pt.d) {
    // int_bnd on the device from the monthly fields uploaded at create
    int m1, m2;
    double f;
    bnd_weights(*M, m1, m2, f);
    M->nday += 1;
    *new_day = 1;
    int rc = pcom_gpu_int_bnd(M->h, m1, m2, f);
    if (!rc) rc = pcom_gpu_den_prho(M->h);
    if (rc) return rc;
  }
  return PCOM_OK;
}

int pcom_model_end_step(pcom_model *M) {
  if (!M) return PCOM_ERR_ARG;
  M->pt = M->ct;
  M->ct = advance(M->ct, M->bc);
  return PCOM_OK;
}

int pcom_model_run(pcom_model *M, int64_t nsteps) {
  if (!M) return PCOM_ERR_ARG;
  if (!M->h) return PCOM_ERR_STATE;
  for (int64_t n = 0; n < nsteps; ++n) {
    int64_t it = 0;
    int32_t day = 0;
    int rc = pcom_model_begin_step(M, &it, &day);
    if (!rc) rc = pcom_gpu_step(M->h, it);
    if (rc) return rc;
    pcom_model_end_step(M);
  }
  return PCOM_OK;
}

int pcom_model_run_batch(pcom_model *const *ms, int32_t n, pcom_batch *b, int64_t nsteps) {
  if (!ms || n <= 0 || !b) return PCOM_ERR_ARG;
  for (int m = 0; m < n; ++m) {
    if (!ms[m] || !ms[m]->h) return PCOM_ERR_STATE;
    const pcom_model &A = *ms[m], &B = *ms[0];
    if (A.iter != B.iter || A.bc != B.bc || A.ct.y != B.ct.y || A.ct.m != B.ct.m || A.ct.d != B.ct.d || A.ct.h != B.ct.h)
      return PCOM_ERR_STATE;
  }
  for (int64_t s = 0; s < nsteps; ++s) {
    pcom_model &M0 = *ms[0];
    const bool day = M0.iter + 1 == 1 || M0.ct.d != M0.pt.d;
    if (day) {
      // the members' forcing buffers are rewritten: wait for the batch first
      int rc = pcom_gpu_batch_sync(b);
      if (rc) return rc;
    }
    for (int m = 0; m < n; ++m) {
      pcom_model &M = *ms[m];
      M.iter += 1;
      if (day) {
        int m1, m2;
        double f;
        bnd_weights(M, m1, m2, f);
        M.nday += 1;
        int rc = pcom_gpu_int_bnd(M.h, m1, m2, f);
        if (rc) return rc;
      }
    }
    if (day) {
      int rc = pcom_gpu_batch_den_prho(b);
      if (rc) return rc;
    }
    int rc = pcom_gpu_batch_step_async(b, M0.iter);
    if (rc) return rc;
    for (int m = 0; m < n; ++m) {
      pcom_model &M = *ms[m];
      M.pt = M.ct;
      M.ct = advance(M.ct, M.bc);
    }
  }
  return pcom_gpu_batch_sync(b);
}

int64_t pcom_model_iter(pcom_model *m) { return m ? m->iter : -1; }

int pcom_model_date(pcom_model *m, int32_t *ymdh4) {
  if (!m || !ymdh4) return PCOM_ERR_ARG;
  ymdh4[0] = m->ct.y; ymdh4[1] = m->ct.m; ymdh4[2] = m->ct.d; ymdh4[3] = m->ct.h;
  return PCOM_OK;
}

int pcom_model_static(pcom_model *m, pcom_static *s) {
  if (!m || !s) return PCOM_ERR_ARG;
  for (int q = 0; q < 4; ++q) { s->rh[q] = m->rh[q].v.data(); s->tn[q] = m->tn[q].v.data(); s->dx[q] = m->dx[q].v.data(); }
  s->z1 = m->z1.data(); s->pr1 = m->pr1.data(); s->dz1 = m->dz1.data(); s->dpr1 = m->dpr1.data();
  s->z2 = m->z2.data(); s->pr2 = m->pr2.data(); s->dz2 = m->dz2.data(); s->dpr2 = m->dpr2.data();
  s->msk_t = m->msk_t.v.data(); s->lev_t = m->lev_t.v.data(); s->msk_u = m->msk_u.v.data(); s->lev_u = m->lev_u.v.data();
  s->phih_t = m->phih_t.v.data(); s->prh_t = m->prh_t.v.data(); s->phih_u = m->phih_u.v.data(); s->prh_u = m->prh_u.v.data();
  s->cv1 = m->cv1.v.data(); s->cv2 = m->cv2.v.data(); s->cor = m->cor.v.data();
  s->km = m->km.v.data(); s->kh = m->kh.v.data();
  s->graphihx = m->graphihx.v.data(); s->graphihy = m->graphihy.v.data();
  return PCOM_OK;
}

int pcom_model_int_bnd(pcom_model *m, double *taux, double *tauy, double *t, double *s, double *pa, double *fw) {
  if (!m) return PCOM_ERR_ARG;
  int_bnd(*m);
  double *dst[6] = {taux, tauy, t, s, pa, fw};
  for (int q = 0; q < 6; ++q)
    if (dst[q]) memcpy(dst[q], m->bnd[q].v.data(), m->bnd[q].v.size() * sizeof(double));
  return PCOM_OK;
}

int pcom_model_initial_state(pcom_model *m, pcom_state *out) {
  if (!m || !out) return PCOM_ERR_ARG;
  const size_t n3 = m->t0.v.size() * sizeof(double);
  if (out->tc) memcpy(out->tc, m->t0.v.data(), n3);
  if (out->sc) memcpy(out->sc, m->s0.v.data(), n3);
  if (out->tp) memcpy(out->tp, m->t0.v.data(), n3);
  if (out->sp) memcpy(out->sp, m->s0.v.data(), n3);
  return PCOM_OK;
}

}  // extern "C"
