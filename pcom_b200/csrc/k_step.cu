// k_step.cu -- FP64 column kernels of the PCOM baroclinic step:
// den_alpha + int_tobot, the int_pgra column integrals, the 2-D helper fields,
// upwelling, int_readyc's advection/friction, int_clin, smag, int_ssh, int_ts
// (with convective adjustment) and den_prho.
//
// One thread owns one (i, j) water column and walks it top to bottom, so the
// reference's sequential SUM(..., 3) and cumulative vertical sums are kept in
// the same order.  Horizontal operators are evaluated point-wise from their
// definitions in mod_op.f90 (see pcom_dev.cuh for the halo conventions).
#include "pcom_dev.cuh"
#include "pcom_kernels.h"

namespace {

__device__ __forceinline__ bool col_ij(const Dev &P, int &i, int &j, bool interior) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  if (interior) {
    i = x + 2;
    return x < P.glo_ni && j <= P.nj;
  }
  i = x + 1;
  return i <= P.ni && j <= P.nj;
}

// ----------------------------------------------------------------------------
// den_alpha (mod_den.f90:33-55) with T, S = tc, sc and ch = chc, fused with
// int_tobot (mod_op.f90:927-944) -> adp.
__global__ void k_alpha_tobot(const __grid_constant__ Dev P) {
  int i, j;
  if (!col_ij(P, i, j, false)) return;
  const long long q2 = I2(P, i, j);
  const int lev = P.lev_t[q2];
  const double ch = P.chc[q2];
  double temp[PCOM_MAXK];
  for (int k = 1; k <= P.nk; ++k) {
    const long long q = q2 + P.n2 * (k - 1);
    double al;
    if (k <= lev) {
      al = 1.0 / den_rho(P.c, P.tc[q], P.sc[q], ch * P.pr2[k]);
      P.alpha[q] = al;
    } else {
      al = P.alpha[q];
    }
    temp[k - 1] = al * P.dpr2[k] * (double)(k <= lev);
  }
  for (int k = 1; k <= P.nk - 1; ++k) {
    double s = 0.0;
    for (int kk = k + 1; kk <= P.nk; ++kk) s = s + temp[kk - 1];
    P.adp[q2 + P.n2 * (k - 1)] = temp[k - 1] * 0.5 + s;
  }
  P.adp[q2 + P.n2 * (P.nk - 1)] = temp[P.nk - 1] * 0.5;
}

// ----------------------------------------------------------------------------
// int_pgra (mod_int.f90:64-88): bphi and bgraphi, the column integrals of the
// E/N-averaged geopotential and of the adp gradient (op_vint_ns/op_vint_ew,
// mod_op.f90:946-981, incl. their cshift(-1) masks).
__global__ void k_pgra2d(const __grid_constant__ Dev P) {
  int i, j;
  if (!col_ij(P, i, j, true)) return;
  const long long q2 = I2(P, i, j);
  const int js = (j == 1) ? P.nj : j - 1;
  const long long qs = I2(P, i, js), qw = q2 - 1;  // cshift(-1) in j and in i
  const int lu = P.lev_u[q2], lus = P.lev_u[qs], luw = P.lev_u[qw];
  const bool nrow = j <= P.njm;
  const double dx2 = ld(P.dxx[2], q2), rh2 = ld(P.rh[2], q2), dy4 = ld(P.dxy[4], q2);
  const double a = P.c.a;
  double xn = 0.0, xs = 0.0, ye = 0.0, yw = 0.0, gxn = 0.0, gxs = 0.0, gye = 0.0, gyw = 0.0;
  for (int k = 1; k <= P.nk; ++k) {
    const long long q = q2 + P.n2 * (k - 1);
    const double dp = P.dpr2[k], pr = P.pr2[k];
    const double mij = (double)(lu >= k), mjs = (double)(lus >= k), miw = (double)(luw >= k);
    const double adc = ld(P.adp, q), ade = ld(P.adp, q + 1);
    const double alc = ld(P.alpha, q), ale = ld(P.alpha, q + 1);
    const double wkE = 0.5 * (adc + ade) + pr * (0.5 * (alc + ale));
    xn = xn + wkE * dp * mij;
    xs = xs + wkE * dp * mjs;
    double wkN = 0.0, wky = 0.0;
    if (nrow) {
      const double adn = ld(P.adp, q + P.ni), aln = ld(P.alpha, q + P.ni);
      wkN = 0.5 * (adc + adn) + pr * (0.5 * (alc + aln));
      wky = ((adn - adc) / dy4) / a;
    }
    ye = ye + wkN * dp * mij;
    yw = yw + wkN * dp * miw;
    const double wkx = ((ade - adc) / dx2) / (a * rh2);
    gxn = gxn + wkx * dp * mij;
    gxs = gxs + wkx * dp * mjs;
    gye = gye + wky * dp * mij;
    gyw = gyw + wky * dp * miw;
  }
  const double pu = ld(P.prh_u, q2), pus = ld(P.prh_u, qs), puw = ld(P.prh_u, qw);
  st2(P.bphi[0], P, i, q2, xn / pu);
  st2(P.bphi[1], P, i, q2, xs / pus);
  st2(P.bphi[2], P, i, q2, ye / pu);
  st2(P.bphi[3], P, i, q2, yw / puw);
  st2(P.bgra[0], P, i, q2, gxn / pu);
  st2(P.bgra[1], P, i, q2, gxs / pus);
  st2(P.bgra[2], P, i, q2, gye / pu);
  st2(P.bgra[3], P, i, q2, gyw / puw);
}

// ----------------------------------------------------------------------------
// 2-D helper fields on the U grid.
//  mode 0 (int_readyc, mod_int.f90:100-109; upwelling :636-637):
//     pax, pay = ter(gra(pa)); sch_r = sqrt(ter(chc, dft 1)), 1 on land;
//     sch_w = sqrt(ter(chp))
//  mode 1 (int_ts: upwelling :636-637 and op_adv_ts :294-295):
//     sch_w = sqrt(ter(chp)); sch_r = sqrt(ter(chc, dft 1)) (no land fix)
__global__ void k_uv2d(const __grid_constant__ Dev P, int mode) {
  int i, j;
  if (!col_ij(P, i, j, true)) return;
  const long long q2 = I2(P, i, j);
  const double a = P.c.a;
  if (mode == 0) {
    // gra_r2d_b(pa, g1j) -> (E, N); ter E->U (ns, sj=0) and N->U (ew, si=0)
    auto wkx = [&](long long q) { return ((ld(P.bnd_pa, q + 1) - ld(P.bnd_pa, q)) / ld(P.dxx[2], q)) / (a * ld(P.rh[2], q)); };
    auto wky = [&](int ii, int jj) {
      if (jj > P.njm) return 0.0;
      long long q = I2(P, ii, jj);
      return ((ld(P.bnd_pa, q + P.ni) - ld(P.bnd_pa, q)) / ld(P.dxy[4], q)) / a;
    };
    double pax = (j <= P.njm) ? 0.5 * (wkx(q2) + wkx(q2 + P.ni)) : 0.0;
    double pay = 0.5 * (wky(i, j) + wky(IP(P, i), j));
    st2(P.pax, P, i, q2, pax);
    st2(P.pay, P, i, q2, pay);
    double s = sqrt(terTU(P, P.chc, i, j, 1.0));
    if (P.lev_u[q2] == 0) s = 1.0;
    st2(P.sch_r, P, i, q2, s);
  } else {
    st2(P.sch_r, P, i, q2, sqrt(terTU(P, P.chc, i, j, 1.0)));
  }
  st2(P.sch_w, P, i, q2, sqrt(terTU(P, P.chp, i, j, 0.0)));
}

// ----------------------------------------------------------------------------
// upwelling (mod_int.f90:626-647): wk3d = div(sqrt(ter(chp)) * (uc, vc)),
// wm(k) = (wm(k-1) + dpr(k-1) (wk3d(k-1) - vint(wk3d))) msk(k).
// with_acw: also int_ts's acw accumulation (mod_int.f90:458-461).
__global__ void k_upwelling(const __grid_constant__ Dev P, int with_acw) {
  int i, j;
  if (!col_ij(P, i, j, true)) return;
  const long long q2 = I2(P, i, j);
  const int lev = P.lev_t[q2];
  const double a = P.c.a;
  const double dx1 = ld(P.dxx[1], q2), dy1 = ld(P.dxy[1], q2), rh1 = ld(P.rh[1], q2);
  const long long qw = q2 - 1, qs = q2 - P.ni, qsw = qs - 1;
  const bool srow = j >= 2;
  double s_c = ld(P.sch_w, q2), s_w = ld(P.sch_w, qw), r_c = ld(P.rh[3], q2), r_w = ld(P.rh[3], qw);
  double s_s = 0, s_sw = 0, r_s = 0, r_sw = 0;
  if (srow) { s_s = ld(P.sch_w, qs); s_sw = ld(P.sch_w, qsw); r_s = ld(P.rh[3], qs); r_sw = ld(P.rh[3], qsw); }
  double wk3d[PCOM_MAXK];
  double s = 0.0;
  for (int k = 1; k <= P.nk; ++k) {
    const long long o = P.n2 * (k - 1);
    // p1(ter_{U->E}(sch uc)) : tE(i') = 0.5 (va(i', j-1) + va(i', j)) for j >= 2
    double tEc = 0.0, tEw = 0.0, tNc, tNs = 0.0;
    if (srow) {
      tEc = 0.5 * (s_s * ld(P.uc, qs + o) + s_c * ld(P.uc, q2 + o));
      tEw = 0.5 * (s_sw * ld(P.uc, qsw + o) + s_w * ld(P.uc, qw + o));
    }
    const double A = (tEc - tEw) / dx1;
    // p2(ter_{U->N}(sch vc rh3)) : tN(j') = 0.5 (x(i-1, j') + x(i, j'))
    tNc = 0.5 * (s_w * ld(P.vc, qw + o) * r_w + s_c * ld(P.vc, q2 + o) * r_c);
    double B = 0.0;
    if (srow) {
      tNs = 0.5 * (s_sw * ld(P.vc, qsw + o) * r_sw + s_s * ld(P.vc, qs + o) * r_s);
      B = (tNc - tNs) / dy1;
    }
    const double w = (A + B) / (a * rh1);
    wk3d[k - 1] = w;
    s = s + w * P.dpr2[k] * (double)(k <= lev);
  }
  const double wk2d = -(s / ld(P.prh_t, q2));
  double wprev = P.wm[q2];
  for (int k = 2; k <= P.nk; ++k) {
    double w = wprev + P.dpr2[k - 1] * (wk2d + wk3d[k - 2]);
    w = w * (double)(k <= lev);
    st2(P.wm, P, i, q2 + P.n2 * (k - 1), w);
    wprev = w;
  }
  if (with_acw) {
    const double gm = P.c.g * ld(P.mch2, q2);
    for (int k = 1; k <= P.nk; ++k) {
      const long long q = q2 + P.n2 * (k - 1);
      const double v = P.acw[q] + P.wm[q] * ld(P.alpha, q) / gm;
      st2(P.acw, P, i, q, v);
    }
  }
}

// ----------------------------------------------------------------------------
// int_readyc 3-D part (mod_int.f90:114-149): op_adv for uc and vc
// (mod_op.f90:224-278), op_fri -> fri_r3d for both components
// (mod_op.f90:103-184) and the depth integral of the baroclinic tendency.
__global__ void k_readyc3d(const __grid_constant__ Dev P) {
  int i, j;
  if (!col_ij(P, i, j, true)) return;
  const long long q2 = I2(P, i, j);
  const int ni = P.ni;
  const double a = P.c.a, g = P.c.g;
  const double grho = g * P.c.rho0;
  const bool nrow = j <= P.njm, srow = j >= 2;
  const long long qe = q2 + 1, qw = q2 - 1, qn = q2 + ni, qs = q2 - ni;
  const int lu = P.lev_u[q2];
  // 2-D coefficients
  const double sch = ld(P.sch_r, q2), sch_e = ld(P.sch_r, qe), sch_w = ld(P.sch_r, qw);
  const double sch_n = nrow ? ld(P.sch_r, qn) : 1.0, sch_s = srow ? ld(P.sch_r, qs) : 1.0;
  const double rh3 = ld(P.rh[3], q2), rh3n = nrow ? ld(P.rh[3], qn) : 0.0, rh3s = srow ? ld(P.rh[3], qs) : 0.0;
  const double dx3 = ld(P.dxx[3], q2), dy3 = ld(P.dxy[3], q2);
  const double dx4 = ld(P.dxx[4], q2), dx4e = ld(P.dxx[4], qe), rh4 = ld(P.rh[4], q2), rh4e = ld(P.rh[4], qe);
  const double dy2 = ld(P.dxy[2], q2), dy2n = nrow ? ld(P.dxy[2], qn) : 1.0;
  const double rh2 = ld(P.rh[2], q2), rh2n = nrow ? ld(P.rh[2], qn) : 0.0;
  const double cv1 = ld(P.cv1, q2), cv2 = ld(P.cv2, q2);
  const double pax = ld(P.pax, q2), pay = ld(P.pay, q2);
  // ter(chc) to N (ns, sj=0) at (i,j), (i+1,j) and to E (ew, si=0) at (i,j), (i,j+1)
  const double c00 = ld(P.chc, q2), c10 = ld(P.chc, qe);
  const double c01 = nrow ? ld(P.chc, qn) : 0.0, c11 = nrow ? ld(P.chc, qn + 1) : 0.0;
  const double chN0 = nrow ? 0.5 * (c00 + c01) : 0.0;
  const double chN1 = nrow ? 0.5 * (c10 + c11) : 0.0;
  const double chE0 = 0.5 * (c00 + c10);
  const double chE1 = nrow ? 0.5 * (c01 + c11) : 0.0;
  // w on U: ter_{T->U}(wm / chc) (di, valid for j <= njm)
  double wc00 = c00, wc10 = c10, wc01 = c01, wc11 = c11;
  auto wU = [&](int kk) -> double {
    if (!nrow) return 0.0;
    const long long o = P.n2 * (kk - 1);
    return (ld(P.wm, q2 + o) / wc00 + ld(P.wm, qn + o) / wc01 + ld(P.wm, qe + o) / wc10 +
            ld(P.wm, qn + 1 + o) / wc11) * 0.25;
  };
  const double tx = ld(P.taux, q2), ty = ld(P.tauy, q2);
  double utS = 0.0, vtS = 0.0;
  // vertical neighbours carried down the column
  double wU_k = wU(1);
  double wkbp_u = 0.0, wkbp_v = 0.0;                 // wkbp(k) for var = uc, vc
  double wkpx = g * tx / sch, wkpy = g * ty / sch;   // wkp(1): surface stress
  double uc_k = P.uc[q2], vc_k = P.vc[q2];
  const int nk = P.nk;
  for (int k = 1; k <= nk; ++k) {
    const long long o = P.n2 * (k - 1);
    const double mu_k = (double)(lu >= k);
    double uc_k1 = 0.0, vc_k1 = 0.0;
    if (k < nk) { uc_k1 = ld(P.uc, q2 + o + P.n2); vc_k1 = ld(P.vc, q2 + o + P.n2); }
    // ---- horizontal neighbours at level k
    const double u_c = uc_k, u_e = ld(P.uc, qe + o), u_w = ld(P.uc, qw + o);
    const double u_n = nrow ? ld(P.uc, qn + o) : 0.0, u_s = srow ? ld(P.uc, qs + o) : 0.0;
    const double v_c = vc_k, v_e = ld(P.vc, qe + o), v_w = ld(P.vc, qw + o);
    const double v_n = nrow ? ld(P.vc, qn + o) : 0.0, v_s = srow ? ld(P.vc, qs + o) : 0.0;
    // unweighted velocity wu = uc/sch, wv = vc/sch
    const double wu_c = u_c / sch, wu_e = u_e / sch_e, wu_w = u_w / sch_w;
    const double wu_n = nrow ? u_n / sch_n : 0.0, wu_s = srow ? u_s / sch_s : 0.0;
    const double wv_c = v_c / sch, wv_e = v_e / sch_e, wv_w = v_w / sch_w;
    const double wv_n = nrow ? v_n / sch_n : 0.0, wv_s = srow ? v_s / sch_s : 0.0;
    // u on N (i, j) and (i+1, j) ; v*cos on E (i, j) and (i, j+1)
    const double uN0 = 0.5 * (wu_w + wu_c), uN1 = 0.5 * (wu_c + wu_e);
    const double vE0 = srow ? 0.5 * (wv_s * rh3s + wv_c * rh3) : 0.0;
    const double vE1 = nrow ? 0.5 * (wv_c * rh3 + wv_n * rh3n) : 0.0;
    // div(v) pieces shared by both advected components
    const double dm1 = (uN1 - uN0) / dx3;
    const double dm2 = nrow ? (vE1 - vE0) / dy3 : 0.0;
    const double wU_k1 = wU(k + 1);
    const double dw = (wU_k - wU_k1) / P.dpr2[k];
    const double rdiv = (dm1 + dm2) / (a * rh3) + dw;
    // ---- op_adv(var): horizontal flux divergence + vertical flux - 0.5 var div(v)
    auto adv = [&](double x_c, double x_e, double x_w, double x_n, double x_s, double x_k1,
                   double &wkbp_k) -> double {
      const double wk1_0 = (0.5 * (x_w + x_c)) * uN0, wk1_1 = (0.5 * (x_c + x_e)) * uN1;
      const double wk2_0 = srow ? (0.5 * (x_s + x_c)) * vE0 : 0.0;
      const double wk2_1 = nrow ? (0.5 * (x_c + x_n)) * vE1 : 0.0;
      const double wa = (wk1_1 - wk1_0) / dx3;
      const double wb = nrow ? (wk2_1 - wk2_0) / dy3 : 0.0;
      double ans = (wa + wb) / (a * rh3);
      // wkbp(k+1) = vter(var)(k+1) * w(k+1) * msk(k) * msk(k+1) for k+1 <= nk
      double wkbp_k1 = 0.0;
      if (k < nk) wkbp_k1 = ((x_c + x_k1) * 0.5 * wU_k1) * mu_k * (double)(lu >= k + 1);
      ans = ans + (wkbp_k - wkbp_k1) / P.dpr2[k];
      wkbp_k = wkbp_k1;
      ans = ans - 0.5 * x_c * rdiv;
      return ans * mu_k;
    };
    const double auc = adv(u_c, u_e, u_w, u_n, u_s, uc_k1, wkbp_u);
    const double avc = adv(v_c, v_e, v_w, v_n, v_s, vc_k1, wkbp_v);
    // ---- fri_r3d(ans, sch, v, vp, vc, tau)
    const double am = ld(P.am, q2 + o);
    auto fri = [&](double v_c_, double v_e_, double v_w_, double v_n_, double v_s_, double vp_c, double vp_k1,
                   double vc_e_, double vc_w_, double v_bot, double vc_bot, double &wkp_k) -> double {
      // gra(v) to N (i', j) and E (i, j')
      const double wx0 = ((v_c_ - v_w_) / dx4) / (a * rh4);
      const double wx1 = ((v_e_ - v_c_) / dx4e) / (a * rh4e);
      const double wy0 = srow ? ((v_c_ - v_s_) / dy2) / a : 0.0;
      const double wy1 = nrow ? ((v_n_ - v_c_) / dy2n) / a : 0.0;
      const double va0 = chN0 * wx0, va1 = chN1 * wx1;
      const double vb0 = (chE0 * wy0) * rh2, vb1 = (chE1 * wy1) * rh2n;
      const double A = (va1 - va0) / dx3;
      const double B = nrow ? (vb1 - vb0) / dy3 : 0.0;
      const double wka = (A + B) / (a * rh3);
      double ans = am / sch * wka;
      ans = ans + am * cv1 * vp_c;
      const double dxc = a * rh4 * (dx4 + dx4e);
      const double pxc = (vc_e_ - vc_w_) / dxc;
      ans = ans + am * cv2 * sch * pxc;
      // wkp(k+1): pz(vp) scaled by km, or the bottom drag at lev+1
      double wkp_k1;
      if (lu > 0 && k == lu) {
        const double mag = sqrt(v_bot * v_bot + vc_bot * vc_bot);
        wkp_k1 = v_bot * g * P.c.cdbot * mag / sch;
      } else if (k + 1 <= nk) {
        const double pzv = (vp_c - vp_k1) * mu_k * (double)(lu >= k + 1) / P.dz1[k + 1];
        wkp_k1 = grho * ld(P.km, q2 + P.n2 * k) * pzv / (sch * sch);
      } else {
        wkp_k1 = 0.0;
      }
      const double wka3 = (wkp_k - wkp_k1) / P.dpr2[k];
      wkp_k = wkp_k1;
      return ans * mu_k + wka3;
    };
    // fx = fri(u = uc/sch, vp = uc, vc = -(vc/sch), taux)
    const double fx = fri(wu_c, wu_e, wu_w, wu_n, wu_s, u_c, uc_k1, -wv_e, -wv_w, wu_c, -wv_c, wkpx);
    // fy = fri(v = vc/sch, vp = vc, vc = uc/sch, tauy)
    const double fy = fri(wv_c, wv_e, wv_w, wv_n, wv_s, v_c, vc_k1, wu_e, wu_w, wv_c, wu_c, wkpy);
    const long long q = q2 + o;
    st2(P.auc, P, i, q, auc);
    st2(P.avc, P, i, q, avc);
    if (P.ab3_mode == 1) {
      st2(P.aup, P, i, q, auc); st2(P.aupp, P, i, q, auc);
      st2(P.avp, P, i, q, avc); st2(P.avpp, P, i, q, avc);
    }
    st2(P.fx, P, i, q, fx);
    st2(P.fy, P, i, q, fy);
    const double wx = -auc - sch * P.c.a0 * pax + fx;
    const double wy = -avc - sch * P.c.a0 * pay + fy;
    utS = utS + wx * P.dpr2[k] * mu_k;
    vtS = vtS + wy * P.dpr2[k] * mu_k;
    // shift the column window
    wU_k = wU_k1;
    uc_k = uc_k1; vc_k = vc_k1;
  }
  const double pu = ld(P.prh_u, q2);
  st2(P.ut, P, i, q2, utS / pu);
  st2(P.vt, P, i, q2, vtS / pu);
}

// ----------------------------------------------------------------------------
// int_clin (mod_int.f90:298-396): baroclinic momentum, barotropic
// replacement, unweighted velocity and its accumulation.  smag runs after.
__global__ void k_clin(const __grid_constant__ Dev P) {
  int i, j;
  if (!col_ij(P, i, j, true)) return;
  const long long q2 = I2(P, i, j);
  const int ni = P.ni;
  const double a = P.c.a;
  const bool nrow = j <= P.njm;
  const int lu = P.lev_u[q2];
  const long long qe = q2 + 1, qn = q2 + ni;
  double sch = 1.0;
  if (lu > 0) sch = sqrt(terTU(P, P.mch, i, j, 1.0));
  // gra(mch) to E at (i,j), (i,j+1) and to N at (i,j), (i+1,j)
  auto gE = [&](const double *f, long long q) { return ((ld(f, q + 1) - ld(f, q)) / ld(P.dxx[2], q)) / (a * ld(P.rh[2], q)); };
  auto gN = [&](const double *f, long long q, int jj) {
    if (jj > P.njm) return 0.0;
    return ((ld(f, q + ni) - ld(f, q)) / ld(P.dxy[4], q)) / a;
  };
  const double mx0 = gE(P.mch, q2), mx1 = nrow ? gE(P.mch, qn) : 0.0;
  const double my0 = gN(P.mch, q2, j), my1 = gN(P.mch, qe, j);
  const double pax = ld(P.pax, q2), pay = ld(P.pay, q2), cor = ld(P.cor, q2);
  const double a0 = P.c.a0, bc = (double)P.bc;
  // T points (i..i+1, j..j+1)
  const double ph00 = ld(P.phih_t, q2), ph10 = ld(P.phih_t, qe);
  const double ph01 = nrow ? ld(P.phih_t, qn) : 0.0, ph11 = nrow ? ld(P.phih_t, qn + 1) : 0.0;
  const double m00 = ld(P.mch, q2), m10 = ld(P.mch, qe);
  const double m01 = nrow ? ld(P.mch, qn) : 0.0, m11 = nrow ? ld(P.mch, qn + 1) : 0.0;
  // column i+2 is needed for px at (i+1, j)? no: px lives on E (i, j), (i, j+1);
  // py lives on N (i, j), (i+1, j) and needs T (i+1, j), (i+1, j+1).
  const double dx2_0 = ld(P.dxx[2], q2), rh2_0 = ld(P.rh[2], q2);
  const double dx2_1 = nrow ? ld(P.dxx[2], qn) : 1.0, rh2_1 = nrow ? ld(P.rh[2], qn) : 1.0;
  const double dy4_0 = ld(P.dxy[4], q2), dy4_1 = ld(P.dxy[4], qe);
  double w1s = 0.0, w2s = 0.0;
  for (int k = 1; k <= P.nk; ++k) {
    const long long o = P.n2 * (k - 1);
    const double pr = P.pr2[k];
    const double ad00 = ld(P.adp, q2 + o), ad10 = ld(P.adp, qe + o);
    const double ad01 = nrow ? ld(P.adp, qn + o) : 0.0, ad11 = nrow ? ld(P.adp, qn + 1 + o) : 0.0;
    const double al00 = ld(P.alpha, q2 + o), al10 = ld(P.alpha, qe + o);
    const double al01 = nrow ? ld(P.alpha, qn + o) : 0.0, al11 = nrow ? ld(P.alpha, qn + 1 + o) : 0.0;
    const double wk00 = ph00 + m00 * ad00, wk10 = ph10 + m10 * ad10;
    const double wk01 = nrow ? ph01 + m01 * ad01 : 0.0, wk11 = nrow ? ph11 + m11 * ad11 : 0.0;
    // px on E (i, j) and (i, j+1)
    const double px0 = ((wk10 - wk00) / dx2_0) / (a * rh2_0) + 0.5 * (al00 + al10) * pr * mx0;
    double t1 = 0.0;
    if (nrow) {
      const double px1 = ((wk11 - wk01) / dx2_1) / (a * rh2_1) + 0.5 * (al01 + al11) * pr * mx1;
      t1 = 0.5 * (px0 + px1);
    }
    // py on N (i, j) and (i+1, j)
    double py0 = 0.0, py1 = 0.0;
    if (nrow) {
      py0 = ((wk01 - wk00) / dy4_0) / a + 0.5 * (al00 + al01) * pr * my0;
      py1 = ((wk11 - wk10) / dy4_1) / a + 0.5 * (al10 + al11) * pr * my1;
    } else {
      py0 = 0.0 + 0.0 * pr * my0;
      py1 = 0.0 + 0.0 * pr * my1;
    }
    const double t2 = 0.5 * (py0 + py1);
    const long long q = q2 + o;
    double p1 = -((t1 + a0 * pax) * sch);
    double p2 = -((t2 + a0 * pay) * sch);
    p1 = p1 - (P.c.c_tc * ld(P.auc, q) + P.c.c_tp * ld(P.aup, q) + P.c.c_tpp * ld(P.aupp, q));
    p2 = p2 - (P.c.c_tc * ld(P.avc, q) + P.c.c_tp * ld(P.avp, q) + P.c.c_tpp * ld(P.avpp, q));
    p1 = p1 + ld(P.fx, q);
    p2 = p2 + ld(P.fy, q);
    const double uck = P.uc[q], vck = P.vc[q];
    p1 = p1 + cor * vck;
    p2 = p2 - cor * uck;
    const double w1 = p1, w2 = p2;
    double w = 0.5 * cor * bc;
    p1 = w1 + w * w2;
    p2 = w2 - w * w1;
    w = 1 + w * w;
    const double mu = (double)(lu >= k);
    p1 = p1 * mu / w;
    p2 = p2 * mu / w;
    const double un = P.up[q] + p1 * bc;
    const double vn = P.vp[q] + p2 * bc;
    P.uc[q] = un;  // in place; fixed up below
    P.vc[q] = vn;
    w1s = w1s + un * P.dpr2[k] * mu;
    w2s = w2s + vn * P.dpr2[k] * mu;
  }
  const double pu = ld(P.prh_u, q2);
  const double w1 = w1s / pu, w2 = w2s / pu;
  const double ubc = ld(P.ubc, q2), vbc = ld(P.vbc, q2);
  const double schu = sqrt(terTU(P, P.mch2, i, j, 1.0));
  const double mch2 = ld(P.mch2, q2);
  for (int k = 1; k <= P.nk; ++k) {
    const long long q = q2 + P.n2 * (k - 1);
    double un = P.uc[q], vn = P.vc[q];
    if (lu >= k) {
      un = un - w1 + ubc;
      vn = vn - w2 + vbc;
    }
    st2(P.uc, P, i, q, un);
    st2(P.vc, P, i, q, vn);
    st2(P.up, P, i, q, un);
    st2(P.vp, P, i, q, vn);
    const double uu = un * schu / mch2, vv = vn * schu / mch2;
    st2(P.uu, P, i, q, uu);
    st2(P.vv, P, i, q, vv);
    st2(P.acu, P, i, q, P.acu[q] + uu);
    st2(P.acv, P, i, q, P.acv[q] + vv);
  }
}

// ----------------------------------------------------------------------------
// smag (mod_int.f90:403-440): Smagorinsky viscosity, rows 2..nj-1.
__global__ void k_smag(const __grid_constant__ Dev P) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  int k = blockIdx.z + 1;
  if (x >= P.glo_ni || j > P.nj - 1) return;
  const int i = x + 2;
  const long long q2 = I2(P, i, j), q = q2 + P.n2 * (k - 1);
  const int ni = P.ni;
  const double a = P.c.a;
  const double dx = a * (ld(P.rh[4], q2) * ld(P.dxx[4], q2) + ld(P.rh[4], q2 + 1) * ld(P.dxx[4], q2 + 1));
  const double dy = a * (ld(P.dxy[2], q2) + ld(P.dxy[2], q2 + ni));
  const double tn = ld(P.tn3, q2);
  const double *u = P.uu, *v = P.vv;
  const double dt = 4 * (ld(u, q + 1) - ld(u, q - 1)) / dx - 4 * (ld(v, q + ni) - ld(v, q - ni)) / dy +
                    ld(v, q) * tn / a;
  const double ds = 4 * (ld(v, q + 1) - ld(v, q - 1)) / dx + 4 * (ld(u, q + ni) - ld(u, q - ni)) / dy -
                    ld(u, q) * tn / a;
  double c = 0.5 * P.c.smag_c / P.c.pi * (0.5 * dx + 0.5 * dy);
  c = c * c;
  const double wk = c * sqrt(dt * dt + ds * ds);
  const double am_max = (dx * dx + dy * dy) / (double)(4 * 8 * P.bc);
  st2(P.am, P, i, q, wk < am_max ? wk : am_max);
}

// ----------------------------------------------------------------------------
// int_ssh (mod_int.f90:602-624): alpha from (tp, sp, mch), SSH accumulation.
__global__ void k_ssh(const __grid_constant__ Dev P) {
  int i, j;
  if (!col_ij(P, i, j, false)) return;
  const long long q2 = I2(P, i, j);
  const int lev = P.lev_t[q2];
  const double mch = P.mch[q2];
  double s = 0.0;
  for (int k = 1; k <= P.nk; ++k) {
    const long long q = q2 + P.n2 * (k - 1);
    double al;
    if (k <= lev) {
      al = 1.0 / den_rho(P.c, P.tp[q], P.sp[q], mch * P.pr2[k]);
      P.alpha[q] = al;
    } else {
      al = P.alpha[q];
    }
    s = s + al * P.dpr2[k] * mch * (double)(k <= lev);
  }
  double ssh = s / P.c.g;
  ssh = P.phih_t[q2] / P.c.g + ssh;
  P.acssh[q2] = P.acssh[q2] + ssh;
}

// ----------------------------------------------------------------------------
// int_ts (mod_int.f90:442-507) after upwelling: tracer advection op_adv_ts
// (mod_op.f90:280-325), diffusion op_dif (mod_op.f90:186-222), surface
// restoring, time step, ice floor, convective adjustment (convect/adjust/mix,
// mod_int.f90:509-600), tp = tc, and the act/acs/acr accumulations.
__device__ void ts_mix(const Dev &P, long long q2, double *t, double *s, double *rhoa, double *rhob, int na, int nb) {
  double st = 0.0, sd = 0.0;
  for (int k = na; k <= nb; ++k) st = st + t[k] * P.dpr2[k];
  for (int k = na; k <= nb; ++k) sd = sd + P.dpr2[k];
  const double tn = st / sd;
  for (int k = na; k <= nb; ++k) t[k] = tn;
  double ss = 0.0;
  for (int k = na; k <= nb; ++k) ss = ss + s[k] * P.dpr2[k];
  const double sn = ss / sd;
  for (int k = na; k <= nb; ++k) s[k] = sn;
  for (int k = na; k <= nb; ++k) {
    const double2 pr = P.prho[q2 + P.n2 * (k - 1)];
    rhoa[k] = pr.x * t[k] + pr.y * s[k];
  }
  for (int k = na; k <= nb - 1; ++k) {
    const double2 pr = P.prho[q2 + P.n2 * k];
    rhob[k] = pr.x * t[k] + pr.y * s[k];
  }
  if (nb < P.nk) {
    const double2 pr = P.prho[q2 + P.n2 * nb];
    rhob[nb] = pr.x * t[nb] + pr.y * s[nb];
  }
}

__device__ void ts_convect(const Dev &P, long long q2, int nlev, double *t, double *s) {
  double rhoa[PCOM_MAXK + 2], rhob[PCOM_MAXK + 2];
  for (int k = 0; k <= P.nk + 1; ++k) { rhoa[k] = 0.0; rhob[k] = 0.0; }
  for (int k = 2; k <= nlev; ++k) {
    const double2 pr = P.prho[q2 + P.n2 * (k - 1)];
    rhoa[k] = pr.x * t[k] + pr.y * s[k];
  }
  for (int k = 1; k <= nlev - 1; ++k) {
    const double2 pr = P.prho[q2 + P.n2 * k];
    rhob[k] = pr.x * t[k] + pr.y * s[k];
  }
  int kcnt = 1;
  int guard = 0;
  while (kcnt < nlev && guard < 4 * PCOM_MAXK * PCOM_MAXK) {
    ++guard;
    if (rhob[kcnt] > rhoa[kcnt + 1]) {
      // adjust (mod_int.f90:544-581)
      int na = kcnt, nb = kcnt + 1;
      ts_mix(P, q2, t, s, rhoa, rhob, na, nb);
      while (nb < nlev) {
        if (rhob[nb] > rhoa[nb + 1]) {
          nb = nb + 1;
          ts_mix(P, q2, t, s, rhoa, rhob, na, nb);
        } else {
          if ((na <= 1) || (rhob[na - 1] <= rhoa[na])) break;
          na = na - 1;
          ts_mix(P, q2, t, s, rhoa, rhob, na, nb);
        }
      }
      while (na > 1) {
        if (rhob[na - 1] <= rhoa[na]) break;
        na = na - 1;
        ts_mix(P, q2, t, s, rhoa, rhob, na, nb);
      }
      kcnt = nb;
    } else {
      kcnt = kcnt + 1;
    }
  }
}

__global__ void k_ts(const __grid_constant__ Dev P) {
  int i, j;
  if (!col_ij(P, i, j, true)) return;
  const long long q2 = I2(P, i, j);
  const int ni = P.ni;
  const double a = P.c.a, g = P.c.g;
  const double grho = g * P.c.rho0;
  const bool nrow = j <= P.njm, srow = j >= 2;
  const long long qw = q2 - 1, qs = q2 - ni, qsw = qs - 1, qe = q2 + 1, qn = q2 + ni;
  const int lev = P.lev_t[q2];
  const int lw = P.lev_t[qw], le = P.lev_t[qe], ln = nrow ? P.lev_t[qn] : 0, ls = srow ? P.lev_t[qs] : 0;
  const double rh1 = ld(P.rh[1], q2), dx1 = ld(P.dxx[1], q2), dy1 = ld(P.dxy[1], q2);
  const double dx2c = ld(P.dxx[2], q2), dx2w = ld(P.dxx[2], qw), rh2c = ld(P.rh[2], q2), rh2w = ld(P.rh[2], qw);
  const double dy4c = ld(P.dxy[4], q2), dy4s = srow ? ld(P.dxy[4], qs) : 1.0;
  const double rh4c = ld(P.rh[4], q2), rh4s = srow ? ld(P.rh[4], qs) : 0.0;
  // sch_t (= sch_r in mode 1) at U (i, j), (i-1, j), (i, j-1), (i-1, j-1)
  const double sc_c = ld(P.sch_r, q2), sc_w = ld(P.sch_r, qw);
  const double sc_s = srow ? ld(P.sch_r, qs) : 0.0, sc_sw = srow ? ld(P.sch_r, qsw) : 0.0;
  const double r3c = ld(P.rh[3], q2), r3w = ld(P.rh[3], qw);
  const double r3s = srow ? ld(P.rh[3], qs) : 0.0, r3sw = srow ? ld(P.rh[3], qsw) : 0.0;
  // ter(mch) to E (i-1, j), (i, j) and to N (i, j-1), (i, j)
  const double mc = ld(P.mch, q2), me = ld(P.mch, qe), mw = ld(P.mch, qw);
  const double mn = nrow ? ld(P.mch, qn) : 0.0, ms = srow ? ld(P.mch, qs) : 0.0;
  const double c1c = 0.5 * (mc + me), c1w = 0.5 * (mw + mc);
  const double c2c = nrow ? 0.5 * (mc + mn) : 0.0, c2s = srow ? 0.5 * (ms + mc) : 0.0;
  const double bc = (double)P.bc;
  double tcol[PCOM_MAXK + 1], scol[PCOM_MAXK + 1];
  const int nk = P.nk;
  // vertical carries
  double wmp_t_k = 0.0, wmp_s_k = 0.0;   // wm(k) * dx3(var)(k), k = 1 -> 0
  double wkp_t_k = 0.0, wkp_s_k = 0.0;   // kh-scaled pz at k, k = 1 -> 0
  double tck = P.tc[q2], sck = P.sc[q2], tpk = P.tp[q2], spk = P.sp[q2];
  for (int k = 1; k <= nk; ++k) {
    const long long o = P.n2 * (k - 1), q = q2 + o;
    const double m_c = (double)(lev >= k), m_w = (double)(lw >= k), m_e = (double)(le >= k);
    const double m_n = (double)(ln >= k), m_s = (double)(ls >= k);
    double tck1 = 0, sck1 = 0, tpk1 = 0, spk1 = 0;
    if (k < nk) {
      tck1 = P.tc[q + P.n2]; sck1 = P.sc[q + P.n2]; tpk1 = P.tp[q + P.n2]; spk1 = P.sp[q + P.n2];
    }
    // mass-weighted velocity: um1 = uc*sch on U, um2 = vc*sch*rh3
    const double um1c = ld(P.uc, q) * sc_c, um1w = ld(P.uc, qw + o) * sc_w;
    const double um1s = srow ? ld(P.uc, qs + o) * sc_s : 0.0, um1sw = srow ? ld(P.uc, qsw + o) * sc_sw : 0.0;
    const double um2c = ld(P.vc, q) * sc_c * r3c, um2w = ld(P.vc, qw + o) * sc_w * r3w;
    const double um2s = srow ? ld(P.vc, qs + o) * sc_s * r3s : 0.0;
    const double um2sw = srow ? ld(P.vc, qsw + o) * sc_sw * r3sw : 0.0;
    // ter U->E (ns, sj=1) at (i, j), (i-1, j); ter U->N (ew, si=1) at (i, j), (i, j-1)
    const double wa1c = srow ? 0.5 * (um1s + um1c) : 0.0, wa1w = srow ? 0.5 * (um1sw + um1w) : 0.0;
    const double wa2c = 0.5 * (um2w + um2c), wa2s = srow ? 0.5 * (um2sw + um2s) : 0.0;
    const double wmk = ld(P.wm, q), wmk1 = ld(P.wm, q + P.n2);  // wm has nkp levels
    const double dpr = P.dpr2[k];
    auto adv = [&](const double *var, double xc, double xk1, double &wmp_k) -> double {
      const double xe = ld(var, qe + o), xw = ld(var, qw + o);
      const double xn = nrow ? ld(var, qn + o) : 0.0, xs = srow ? ld(var, qs + o) : 0.0;
      const double w1c = (xe - xc) / dx2c, w1w = (xc - xw) / dx2w;
      const double wb1 = 0.5 * (wa1w * w1w + wa1c * w1c);
      double ans = wb1 / (a * rh1);
      const double w2c = nrow ? (xn - xc) / dy4c : 0.0;
      double wb2 = 0.0;
      if (srow) {
        const double w2s = (xc - xs) / dy4s;
        wb2 = 0.5 * (wa2s * w2s + wa2c * w2c);
      }
      ans = ans + wb2 / (a * rh1);
      const double wmp_k1 = (k < nk) ? wmk1 * (xc - xk1) : wmk1 * 0.0;
      ans = ans + (wmp_k + wmp_k1) * 0.5 / dpr;
      wmp_k = wmp_k1;
      return ans;
    };
    auto dif = [&](const double *var, double xc, double xk1, double &wkp_k) -> double {
      const double xe = ld(var, qe + o), xw = ld(var, qw + o);
      const double xn = nrow ? ld(var, qn + o) : 0.0, xs = srow ? ld(var, qs + o) : 0.0;
      const double w1c = (xe - xc) * m_e * m_c / dx2c / (a * rh2c);
      const double w1w = (xc - xw) * m_c * m_w / dx2w / (a * rh2w);
      const double A = (c1c * w1c - c1w * w1w) / dx1;
      const double w2c = nrow ? (xn - xc) * m_n * m_c / dy4c / a : 0.0;
      double B = 0.0;
      if (srow) {
        const double w2s = (xc - xs) * m_c * m_s / dy4s / a;
        B = ((c2c * w2c) * rh4c - (c2s * w2s) * rh4s) / dy1;
      }
      double ans = P.c.ah_c * ((A + B) / (a * rh1));
      double wkp_k1 = 0.0;
      if (k < nk) {
        const double pz = (xc - xk1) * m_c * (double)(lev >= k + 1) / P.dz1[k + 1];
        wkp_k1 = grho * ld(P.kh, q2 + P.n2 * k) * pz;
      }
      ans = ans + (wkp_k - wkp_k1) / dpr;
      wkp_k = wkp_k1;
      return ans;
    };
    const double at = adv(P.tc, tck, tck1, wmp_t_k);
    const double as = adv(P.sc, sck, sck1, wmp_s_k);
    const double dt_ = dif(P.tp, tpk, tpk1, wkp_t_k);
    const double ds_ = dif(P.sp, spk, spk1, wkp_s_k);
    double p1 = -at, p2 = -as;
    p1 = p1 + dt_;
    p2 = p2 + ds_;
    if (k == 1) {
      p1 = p1 + P.c.gamma_t * (ld(P.bnd_t, q2) - tck) * m_c / P.dpr2[1];
      p2 = p2 + P.c.gamma_s * (ld(P.bnd_s, q2) - sck) * m_c * mc;
    }
    double tn = tpk + p1 * bc * m_c / mc;
    const double sn = spk + p2 * bc * m_c / mc;
    if (m_c > 0 && tn < P.c.tice) tn = P.c.tice;
    tcol[k] = tn;
    scol[k] = sn;
    tck = tck1; sck = sck1; tpk = tpk1; spk = spk1;
  }
  if (lev > 1) ts_convect(P, q2, lev, tcol, scol);
  const double chc = ld(P.chc, q2);
  for (int k = 1; k <= nk; ++k) {
    const long long q = q2 + P.n2 * (k - 1);
    st2(P.tn_, P, i, q, tcol[k]);
    st2(P.sn_, P, i, q, scol[k]);
    st2(P.act, P, i, q, P.act[q] + tcol[k]);
    st2(P.acs, P, i, q, P.acs[q] + scol[k]);
    if (k <= lev) {
      const double w = 1.0 / den_rho(P.c, tcol[k], scol[k], chc * P.pr2[k]);
      st2(P.acr, P, i, q, P.acr[q] + 1.0 / w);
    }
  }
}

// ----------------------------------------------------------------------------
// den_prho (mod_den.f90:120-153)
__global__ void k_den_prho(const __grid_constant__ Dev P) {
  int i, j;
  if (!col_ij(P, i, j, false)) return;
  const long long q2 = I2(P, i, j);
  const int lev = P.lev_t[q2];
  const double ch = P.chc[q2];
  const double dt = P.c.deltat, ds = P.c.deltas;
  for (int k = 1; k <= lev && k <= P.nk; ++k) {
    const long long q = q2 + P.n2 * (k - 1);
    const double t = P.tc[q], s = P.sc[q], p = ch * P.pr2[k];
    double ra = den_rho(P.c, t + dt, s, p), rb = den_rho(P.c, t - dt, s, p);
    double2 r;
    r.x = (ra - rb) / (2 * dt);
    ra = den_rho(P.c, t, s + ds, p);
    rb = den_rho(P.c, t, s - ds, p);
    r.y = (ra - rb) / (2 * ds);
    P.prho[q] = r;
  }
}

}  // namespace

// ---------------------------------------------------------------- launchers
static inline dim3 cols_grid(const Dev &P, bool interior) {
  int nx = interior ? P.glo_ni : P.ni;
  return dim3((nx + COLS_X - 1) / COLS_X, (P.nj + COLS_Y - 1) / COLS_Y, 1);
}
static const dim3 kColsBlock(COLS_X, COLS_Y, 1);

void launch_alpha_tobot(const Dev &P, cudaStream_t s) { k_alpha_tobot<<<cols_grid(P, false), kColsBlock, 0, s>>>(P); }
void launch_pgra2d(const Dev &P, cudaStream_t s) { k_pgra2d<<<cols_grid(P, true), kColsBlock, 0, s>>>(P); }
void launch_uv2d(const Dev &P, int mode, cudaStream_t s) { k_uv2d<<<cols_grid(P, true), kColsBlock, 0, s>>>(P, mode); }
void launch_upwelling(const Dev &P, int with_acw, cudaStream_t s) {
  k_upwelling<<<cols_grid(P, true), kColsBlock, 0, s>>>(P, with_acw);
}
void launch_readyc3d(const Dev &P, cudaStream_t s) { k_readyc3d<<<cols_grid(P, true), kColsBlock, 0, s>>>(P); }
void launch_clin(const Dev &P, cudaStream_t s) { k_clin<<<cols_grid(P, true), kColsBlock, 0, s>>>(P); }
void launch_smag(const Dev &P, cudaStream_t s) {
  dim3 g((P.glo_ni + COLS_X - 1) / COLS_X, (P.nj - 2 + COLS_Y - 1) / COLS_Y, P.nk);
  if (P.nj > 2) k_smag<<<g, kColsBlock, 0, s>>>(P);
}
void launch_ssh(const Dev &P, cudaStream_t s) { k_ssh<<<cols_grid(P, false), kColsBlock, 0, s>>>(P); }
void launch_ts(const Dev &P, cudaStream_t s) { k_ts<<<cols_grid(P, true), kColsBlock, 0, s>>>(P); }
void launch_den_prho(const Dev &P, cudaStream_t s) { k_den_prho<<<cols_grid(P, false), kColsBlock, 0, s>>>(P); }
