// k_step.cu -- FP64 kernels of the PCOM baroclinic step outside the
// barotropic subcycle: den_alpha + int_tobot, the int_pgra column integrals,
// the 2-D prep fields, upwelling, int_readyc's advection/friction, int_clin,
// smag, int_ssh, int_ts (with convective adjustment) and den_prho.
//
// Work decomposition: a CTA covers 32 consecutive columns of one row and all
// levels; each thread computes whole (i, j, k) points, so there are nk
// threads' worth of parallelism per column.  Vertical reductions (the
// reference's SUM(..., 3), the cumulative upwelling sum, the column integral
// of the baroclinic velocity) and the data-dependent convective adjustment
// are done from shared memory by one thread per column, in the reference's
// sequential order.  int_ts and int_readyc's 3-D part on the FP64 path are
// the exceptions: one thread per column marches down the levels (k_ts_col,
// k_readyc_col), and a point-parallel kernel forms int_ts's accumulations
// (k_ts_acc).  Horizontal operators are evaluated point-wise from their
// definitions in mod_op.f90 (halo conventions in pcom_dev.cuh).  Every
// division by a static metric, a bottom pressure or a per-step 2-D field uses
// its precomputed correctly rounded reciprocal with dvr (bitwise equal to the
// IEEE quotient); the equation of state keeps its IEEE divisions.
#include <type_traits>

#include "pcom_dev.cuh"
#include "pcom_kernels.h"

// block of the level-parallel 3-D kernels: 32 columns of one row x TB_K
// threads down the levels.  8 (256 threads) rather than 16: the kernels
// end in a serial column pass by one or two warps, and smaller blocks let
// more of them per SM overlap that pass with other blocks' loads (1-degree
// FP64 step 1.240 -> 1.188 ms).  k_pgra2d needs TB_K >= 8 (one column sum per
// thread row).
#define TB_X 32
#define TB_K 8
static_assert(TB_K >= 8, "k_pgra2d computes one of its 8 column sums per thread row");

namespace {

// metric accessors of a separable (lat-lon) grid
#define MX(g, i) __ldg(P.dxx1d[g] + (i) - 1)
#define RMX(g, i) __ldg(P.rdxx1d[g] + (i) - 1)
#define MY(g, j) __ldg(P.dxy1d[g] + (j) - 1)
#define RMY(g, j) __ldg(P.rdxy1d[g] + (j) - 1)
#define RH(g, j) __ldg(P.rh1d[g] + (j) - 1)
#define RRH(g, j) __ldg(P.rrh1d[g] + (j) - 1)
#define ARH(g, j) __ldg(P.arh1d[g] + (j) - 1)
#define RARH(g, j) __ldg(P.rarh1d[g] + (j) - 1)
// x / dx?x(i), x / dx?y(j), x / (a rh?(j)), x / a, x / dpr(k)
#define DIVX(x, g, i) dvr((x), MX(g, i), RMX(g, i))
#define DIVY(x, g, j) dvr((x), MY(g, j), RMY(g, j))
#define DIVARH(x, g, j) dvr((x), ARH(g, j), RARH(g, j))
#define DIVA(x) dvr((x), P.c.a, P.ra)
#define DIVDP(x, k) dvr((x), P.dpr2[k], P.rdpr2[k])

// column/row of this thread; interior: i in 2..ni-1, else i in 1..ni
template <int BX = TB_X, typename R>
__device__ __forceinline__ bool cell(const DevT<R> &P, int &i, int &j, bool interior) {
  const int x = blockIdx.x * BX + threadIdx.x;
  j = blockIdx.y + P.j_lo;
  if (interior) {
    i = x + 2;
    return x < P.glo_ni && j <= P.j_hi;
  }
  i = x + 1;
  return i <= P.ni && j <= P.j_hi;
}

// smag covers rows 2..nj-1 of the row window
template <typename R>
__host__ __device__ __forceinline__ int smag_j0(const DevT<R> &P) { return P.j_lo > 2 ? P.j_lo : 2; }
template <typename R>
__host__ __device__ __forceinline__ int smag_j1(const DevT<R> &P) { return P.j_hi < P.nj - 1 ? P.j_hi : P.nj - 1; }

// ----------------------------------------------------------------------------
// den_alpha (mod_den.f90:33-55) with T, S = tc, sc and ch = chc, fused with
// int_tobot (mod_op.f90:927-944) -> adp.
template <typename R, bool BATCH>
__global__ void __launch_bounds__(512) k_alpha_tobot(const __grid_constant__ DevT<R> P0, const DevT<R> *__restrict__ Ps) {
  const DevT<R> &P = BATCH ? Ps[blockIdx.z] : P0;
  constexpr bool MIXED = std::is_same<R, float>::value;
  (void)MIXED;
  extern __shared__ double sh[];
  double *tmp = sh;  // [nk][TB_X]
  int i, j;
  const bool ok = cell(P, i, j, false);
  const int tx = threadIdx.x;
  const long long q2 = ok ? I2(P, i, j) : 0;
  const int lev = ok ? P.lev_t[q2] : 0;
  const double ch = ok ? P.chc[q2] : 0.0;
  const int nk = P.nk;
  for (int k = threadIdx.y + 1; k <= nk; k += TB_K) {
    if (!ok) continue;
    const long long q = q2 + P.n2 * (k - 1);
    double al;
    if (k <= lev) {
      al = 1.0 / den_rho(P.c, P.tc[q], P.sc[q], ch * P.pr2[k]);
      P.alpha[q] = alpha_store(P, al, k);
    } else {
      al = alpha_full(P, P.alpha[q], k);
    }
    tmp[(k - 1) * TB_X + tx] = al * P.dpr2[k] * (double)(k <= lev);
  }
  __syncthreads();
  for (int k = threadIdx.y + 1; k <= nk; k += TB_K) {
    if (!ok) continue;
    double v;
    if (k < nk) {
      double s = 0.0;
      for (int kk = k + 1; kk <= nk; ++kk) s = s + tmp[(kk - 1) * TB_X + tx];
      v = tmp[(k - 1) * TB_X + tx] * 0.5 + s;
    } else {
      v = tmp[(nk - 1) * TB_X + tx] * 0.5;
    }
    P.adp[q2 + P.n2 * (k - 1)] = adp_store(P, v, k, q2);
  }
}

// ----------------------------------------------------------------------------
// int_pgra (mod_int.f90:64-88): bphi and bgraphi, the column integrals of the
// E/N-averaged geopotential and of the adp gradient (op_vint_ns/op_vint_ew,
// mod_op.f90:946-981, incl. their cshift(-1) masks).
template <typename R, bool BATCH>
__global__ void __launch_bounds__(512) k_pgra2d(const __grid_constant__ DevT<R> P0, const DevT<R> *__restrict__ Ps) {
  const DevT<R> &P = BATCH ? Ps[blockIdx.z] : P0;
  constexpr bool MIXED = std::is_same<R, float>::value;
  (void)MIXED;
  extern __shared__ double sh[];
  const int nk = P.nk;
  double *bE = sh, *bN = sh + nk * TB_X, *bX = sh + 2 * nk * TB_X, *bY = sh + 3 * nk * TB_X;
  int i, j;
  const bool ok = cell(P, i, j, true);
  const int tx = threadIdx.x;
  const long long q2 = ok ? I2(P, i, j) : 0;
  const bool nrow = j <= P.njm;
  for (int k = threadIdx.y + 1; k <= nk; k += TB_K) {
    if (!ok) continue;
    const long long q = q2 + P.n2 * (k - 1);
    const double dp = P.dpr2[k], pr = P.pr2[k];
    const double adc = adp_full(P, ld(P.adp, q), k, q2), ade = adp_full(P, ld(P.adp, q + 1), k, q2 + 1);
    const double alc = alpha_full(P, ld(P.alpha, q), k), ale = alpha_full(P, ld(P.alpha, q + 1), k);
    const double wkE = 0.5 * (adc + ade) + pr * (0.5 * (alc + ale));
    double wkN = 0.0, wky = 0.0;
    if (nrow) {
      const double adn = adp_full(P, ld(P.adp, q + P.ni), k, q2 + P.ni), aln = alpha_full(P, ld(P.alpha, q + P.ni), k);
      wkN = 0.5 * (adc + adn) + pr * (0.5 * (alc + aln));
      wky = DIVA(DIVY(adn - adc, 4, j));
    }
    const double wkx = DIVARH(DIVX(ade - adc, 2, i), 2, j);
    const int o = (k - 1) * TB_X + tx;
    bE[o] = wkE * dp;
    bN[o] = wkN * dp;
    bX[o] = wkx * dp;
    bY[o] = wky * dp;
  }
  __syncthreads();
  const int which = threadIdx.y;  // 8 column sums, one per thread row
  if (!ok || which >= 8) return;
  const int js = (j == 1) ? P.nj : j - 1;
  const long long qs = I2(P, i, js), qw = q2 - 1;  // cshift(-1) in j and in i
  const double *base = (which < 2) ? bE : (which < 4) ? bN : (which < 6) ? bX : bY;
  // masks: own point, the point cshift(-1) in j (xs) or in i (yw)
  const long long qm = (which & 1) ? ((which == 1 || which == 5) ? qs : qw) : q2;
  const int lm = P.lev_u[qm];
  double s = 0.0;
  for (int k = 1; k <= nk; ++k) s = s + base[(k - 1) * TB_X + tx] * (double)(lm >= k);
  const double v = dvr(s, ld(P.prh_u, qm), ld(P.rprh_u, qm));
  double *dst = (which < 4) ? P.bphi[which] : P.bgra[which - 4];
  st2(dst, P, i, q2, v);
}

// ----------------------------------------------------------------------------
// 2-D prep fields on the U grid (plus reciprocals of T-grid fields).
//  mode 0 (int_readyc, mod_int.f90:100-109; upwelling :636-637):
//     pax, pay = ter(gra(pa)); sch_r = sqrt(ter(chc, dft 1)), 1 on land;
//     sch_w = sqrt(ter(chp)); 1/sch_r, 1/sch_r^2, 1/chc
//  mode 1 (int_ts: upwelling :636-637 and op_adv_ts :294-295):
//     sch_w = sqrt(ter(chp)); sch_r = sqrt(ter(chc, dft 1)) (no land fix);
//     1/mch, 1/(g mch2)
//  mode 2 (int_clin, mod_int.f90:318-320, 385-386): sqrt(ter(mch, dft 1))
//     with 1 on land, sqrt(ter(mch2, dft 1)), 1/mch2
template <typename R, bool BATCH>
__global__ void k_uv2d(const __grid_constant__ DevT<R> P0, const DevT<R> *__restrict__ Ps, int mode) {
  const DevT<R> &P = BATCH ? Ps[blockIdx.z] : P0;
  constexpr bool MIXED = std::is_same<R, float>::value;
  (void)MIXED;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  if (x >= P.glo_ni || j > P.nj) return;
  const int i = x + 2;
  const long long q2 = I2(P, i, j);
  if (mode == 0) {
    // gra_r2d_b(pa, g1j) -> (E, N); ter E->U (ns, sj=0) and N->U (ew, si=0)
    auto wkx = [&](long long q, int jj) { return DIVARH(DIVX(ld(P.bnd_pa, q + 1) - ld(P.bnd_pa, q), 2, i), 2, jj); };
    auto wky = [&](int ii) {
      if (j > P.njm) return 0.0;
      const long long q = I2(P, ii, j);
      return DIVA(DIVY(ld(P.bnd_pa, q + P.ni) - ld(P.bnd_pa, q), 4, j));
    };
    const double pax = (j <= P.njm) ? 0.5 * (wkx(q2, j) + wkx(q2 + P.ni, j + 1)) : 0.0;
    const double pay = 0.5 * (wky(i) + wky(IP(P, i)));
    st2(P.pax, P, i, q2, pax);
    st2(P.pay, P, i, q2, pay);
    double s = sqrt(terTU(P, P.chc, i, j, 1.0));
    if (P.lev_u[q2] == 0) s = 1.0;
    st2(P.sch_r, P, i, q2, s);
    st2(P.rsch, P, i, q2, 1.0 / s);
    st2(P.rsch2, P, i, q2, 1.0 / (s * s));
    st2(P.rchc, P, i, q2, 1.0 / P.chc[q2]);
    st2(P.sch_w, P, i, q2, sqrt(terTU(P, P.chp, i, j, 0.0)));
  } else {
    // mode 2: int_clin's fields; mode 1: int_ts's; mode 3: both (all read
    // only the barotropic subcycle's chc, chp, mch, mch2, which nothing
    // between int_clin and int_ts changes)
    if (mode != 1) {
      double s = 1.0;
      if (P.lev_u[q2] > 0) s = sqrt(terTU(P, P.mch, i, j, 1.0));
      st2(P.schc, P, i, q2, s);
      st2(P.schu, P, i, q2, sqrt(terTU(P, P.mch2, i, j, 1.0)));
      st2(P.rmch2, P, i, q2, 1.0 / P.mch2[q2]);
    }
    if (mode != 2) {
      st2(P.sch_r, P, i, q2, sqrt(terTU(P, P.chc, i, j, 1.0)));
      st2(P.sch_w, P, i, q2, sqrt(terTU(P, P.chp, i, j, 0.0)));
      st2(P.rmch, P, i, q2, 1.0 / P.mch[q2]);
      st2(P.rgm2, P, i, q2, 1.0 / (P.c.g * P.mch2[q2]));
    }
  }
}

// ----------------------------------------------------------------------------
// columns per block of k_upwelling: 16 on the FP64 path (its serial column
// pass then overlaps better with other blocks' loads: 50 -> 44 us and 57 ->
// 49 us at 1 degree), 32 on the mixed path (no gain there)
template <typename R>
__host__ __device__ constexpr int upw_cols() { return std::is_same<R, double>::value ? 16 : TB_X; }
// upwelling (mod_int.f90:626-647): wk3d = div(sqrt(ter(chp)) * (uc, vc)),
// wm(k) = (wm(k-1) + dpr(k-1) (wk3d(k-1) - vint(wk3d))) msk(k).
// with_acw: also int_ts's acw accumulation (mod_int.f90:458-461).
template <typename R, bool BATCH>
__global__ void __launch_bounds__(512) k_upwelling(const __grid_constant__ DevT<R> P0, const DevT<R> *__restrict__ Ps, int with_acw) {
  const DevT<R> &P = BATCH ? Ps[blockIdx.z] : P0;
  constexpr bool MIXED = std::is_same<R, float>::value;
  (void)MIXED;
  extern __shared__ double sh[];
  const int nk = P.nk;
  constexpr int UX = upw_cols<R>();
  double *wk = sh, *tm = sh + nk * UX, *wmv = sh + 2 * nk * UX;
  int i, j;
  const bool ok = cell<UX>(P, i, j, true);
  const int tx = threadIdx.x;
  const long long q2 = ok ? I2(P, i, j) : 0;
  const int lev = ok ? P.lev_t[q2] : 0;
  const bool srow = j >= 2;
  const long long qw = q2 - 1, qs = q2 - P.ni, qsw = qs - 1;
  for (int k = threadIdx.y + 1; k <= nk; k += TB_K) {
    if (!ok) continue;
    const long long o = P.n2 * (k - 1);
    const R s_c = ld(P.sch_w, q2), s_w = ld(P.sch_w, qw);
    const R r_c = RH(3, j);
    // p1(ter_{U->E}(sch uc)): tE(i') = 0.5 (va(i', j-1) + va(i', j)) for j >= 2
    R tEc = 0.0, tEw = 0.0, B = 0.0;
    if (srow) {
      const R s_s = ld(P.sch_w, qs), s_sw = ld(P.sch_w, qsw), r_s = RH(3, j - 1);
      tEc = 0.5 * (s_s * ld(P.uc, qs + o) + s_c * ld(P.uc, q2 + o));
      tEw = 0.5 * (s_sw * ld(P.uc, qsw + o) + s_w * ld(P.uc, qw + o));
      // p2(ter_{U->N}(sch vc rh3)): tN(j') = 0.5 (x(i-1, j') + x(i, j'))
      const R tNc = 0.5 * (s_w * ld(P.vc, qw + o) * r_c + s_c * ld(P.vc, q2 + o) * r_c);
      const R tNs = 0.5 * (s_sw * ld(P.vc, qsw + o) * r_s + s_s * ld(P.vc, qs + o) * r_s);
      B = DIVY(tNc - tNs, 1, j);
    }
    const R A = DIVX(tEc - tEw, 1, i);
    const R w = DIVARH(A + B, 1, j);
    wk[(k - 1) * UX + tx] = w;
    tm[(k - 1) * UX + tx] = w * P.dpr2[k] * (R)(k <= lev);
  }
  __syncthreads();
  if (ok && threadIdx.y == 0) {
    double s = 0.0;
    for (int k = 1; k <= nk; ++k) s = s + tm[(k - 1) * UX + tx];
    const double wk2d = -dvr(s, ld(P.prh_t, q2), ld(P.rprh_t, q2));
    double wprev = P.wm[q2];
    wmv[tx] = wprev;
    for (int k = 2; k <= nk; ++k) {
      double w = wprev + P.dpr2[k - 1] * (wk2d + wk[(k - 2) * UX + tx]);
      w = w * (double)(k <= lev);
      wmv[(k - 1) * UX + tx] = w;
      wprev = w;
    }
  }
  __syncthreads();
  if (!ok) return;
  for (int k = threadIdx.y + 1; k <= nk; k += TB_K) {
    const long long q = q2 + P.n2 * (k - 1);
    const double w = wmv[(k - 1) * UX + tx];
    if (k >= 2) st2(P.wm, P, i, q, w);
    if (with_acw) {
      const double gm = P.c.g * ld(P.mch2, q2);
      st2(P.acw, P, i, q, P.acw[q] + dvr(w * alpha_full(P, ld(P.alpha, q), k), gm, ld(P.rgm2, q2)));
    }
  }
}

// ----------------------------------------------------------------------------
// int_readyc 3-D part (mod_int.f90:114-149): op_adv for uc and vc
// (mod_op.f90:224-278), op_fri -> fri_r3d for both components
// (mod_op.f90:103-184) and the depth integral of the baroclinic tendency.
template <typename R, bool BATCH>
__global__ void __launch_bounds__(512) k_readyc3d(const __grid_constant__ DevT<R> P0, const DevT<R> *__restrict__ Ps) {
  const DevT<R> &P = BATCH ? Ps[blockIdx.z] : P0;
  constexpr bool MIXED = std::is_same<R, float>::value;
  (void)MIXED;
  extern __shared__ double sh[];
  const int nk = P.nk;
  double *tu = sh, *tv = sh + nk * TB_X;
  int i, j;
  const bool ok = cell(P, i, j, true);
  const int tx = threadIdx.x;
  const long long q2 = ok ? I2(P, i, j) : 0;
  const int ni = P.ni;
  const R g = P.c.g, a = P.c.a;
  const R grho = g * P.c.rho0;
  const bool nrow = j <= P.njm, srow = j >= 2;
  const long long qe = q2 + 1, qw = q2 - 1, qn = q2 + ni, qs = q2 - ni;
  const int lu = ok ? P.lev_u[q2] : 0;
  for (int k = threadIdx.y + 1; k <= nk && ok; k += TB_K) {
    const long long o = P.n2 * (k - 1);
    // per-column coefficients
    const R sch = ld(P.sch_r, q2), rsch = ld(P.rsch, q2);
    const R rsc_e = ld(P.rsch, qe), rsc_w = ld(P.rsch, qw);
    const R sch_e = ld(P.sch_r, qe), sch_w = ld(P.sch_r, qw);
    const R rh3 = RH(3, j), dx3 = MX(3, i), rdx3 = RMX(3, i), dy3 = MY(3, j), rdy3 = RMY(3, j);
    const R arh3 = ARH(3, j), rarh3 = RARH(3, j);
    const R mu_k = (R)(lu >= k), mu_k1 = (R)(lu >= k + 1), mu_km = (R)(lu >= k - 1);
    auto U = [&](long long q, int kk) { return ld(P.uc, q + P.n2 * (kk - 1)); };
    auto V = [&](long long q, int kk) { return ld(P.vc, q + P.n2 * (kk - 1)); };
    // velocities at level k (unweighted wu = uc/sch, wv = vc/sch)
    const R u_c = U(q2, k), u_e = U(qe, k), u_w = U(qw, k);
    const R v_c = V(q2, k), v_e = V(qe, k), v_w = V(qw, k);
    const R wu_c = dvr(u_c, sch, rsch), wu_e = dvr(u_e, sch_e, rsc_e), wu_w = dvr(u_w, sch_w, rsc_w);
    const R wv_c = dvr(v_c, sch, rsch), wv_e = dvr(v_e, sch_e, rsc_e), wv_w = dvr(v_w, sch_w, rsc_w);
    R u_n = 0, u_s = 0, v_n = 0, v_s = 0, wu_n = 0, wu_s = 0, wv_n = 0, wv_s = 0, rh3n = 0, rh3s = 0;
    if (nrow) {
      const R sn = ld(P.sch_r, qn), rsn = ld(P.rsch, qn);
      u_n = U(qn, k); v_n = V(qn, k);
      wu_n = dvr(u_n, sn, rsn); wv_n = dvr(v_n, sn, rsn);
      rh3n = RH(3, j + 1);
    }
    if (srow) {
      const R ss = ld(P.sch_r, qs), rss = ld(P.rsch, qs);
      u_s = U(qs, k); v_s = V(qs, k);
      wu_s = dvr(u_s, ss, rss); wv_s = dvr(v_s, ss, rss);
      rh3s = RH(3, j - 1);
    }
    // vertical neighbours at (i, j)
    const R u_km = (k > 1) ? U(q2, k - 1) : 0.0, v_km = (k > 1) ? V(q2, k - 1) : 0.0;
    const R u_k1 = (k < nk) ? U(q2, k + 1) : 0.0, v_k1 = (k < nk) ? V(q2, k + 1) : 0.0;
    // u on N (i, j), (i+1, j); v*cos on E (i, j), (i, j+1)
    const R uN0 = 0.5 * (wu_w + wu_c), uN1 = 0.5 * (wu_c + wu_e);
    const R vE0 = srow ? 0.5 * (wv_s * rh3s + wv_c * rh3) : 0.0;
    const R vE1 = nrow ? 0.5 * (wv_c * rh3 + wv_n * rh3n) : 0.0;
    // w on U: ter_{T->U}(wm / chc) (di, rows j <= njm)
    auto wU = [&](int kk) -> R {
      if (!nrow) return 0.0;
      const long long ok_ = P.n2 * (kk - 1);
      const long long t00 = q2, t01 = qn, t10 = qe, t11 = qn + 1;
      return (dvr(ld(P.wm, t00 + ok_), ld(P.chc, t00), ld(P.rchc, t00)) +
              dvr(ld(P.wm, t01 + ok_), ld(P.chc, t01), ld(P.rchc, t01)) +
              dvr(ld(P.wm, t10 + ok_), ld(P.chc, t10), ld(P.rchc, t10)) +
              dvr(ld(P.wm, t11 + ok_), ld(P.chc, t11), ld(P.rchc, t11))) * 0.25;
    };
    const R wUk = wU(k), wUk1 = wU(k + 1);
    const R dm1 = dvr(uN1 - uN0, dx3, rdx3);
    const R dm2 = nrow ? dvr(vE1 - vE0, dy3, rdy3) : 0.0;
    const R dw = DIVDP(wUk - wUk1, k);
    const R rdiv = dvr(dm1 + dm2, arh3, rarh3) + dw;
    // op_adv(var)
    auto adv = [&](R x_c, R x_e, R x_w, R x_n, R x_s, R x_km, R x_k1) {
      const R wk1_0 = (0.5 * (x_w + x_c)) * uN0, wk1_1 = (0.5 * (x_c + x_e)) * uN1;
      const R wk2_0 = srow ? (0.5 * (x_s + x_c)) * vE0 : 0.0;
      const R wk2_1 = nrow ? (0.5 * (x_c + x_n)) * vE1 : 0.0;
      const R wa = dvr(wk1_1 - wk1_0, dx3, rdx3);
      const R wb = nrow ? dvr(wk2_1 - wk2_0, dy3, rdy3) : 0.0;
      R ans = dvr(wa + wb, arh3, rarh3);
      // wkbp(kk) = vter(var)(kk) w(kk) msk(kk-1) msk(kk) for 2 <= kk <= nk
      const R wkbp_k = (k >= 2) ? ((x_km + x_c) * 0.5 * wUk) * mu_km * mu_k : 0.0;
      const R wkbp_k1 = (k < nk) ? ((x_c + x_k1) * 0.5 * wUk1) * mu_k * mu_k1 : 0.0;
      ans = ans + DIVDP(wkbp_k - wkbp_k1, k);
      ans = ans - 0.5 * x_c * rdiv;
      return ans * mu_k;
    };
    const R auc = adv(u_c, u_e, u_w, u_n, u_s, u_km, u_k1);
    const R avc = adv(v_c, v_e, v_w, v_n, v_s, v_km, v_k1);
    // fri_r3d(ans, sch, v, vp, vc, tau)
    const R am = ld(P.am, q2 + o);
    const R cv1 = ld(P.cv1, q2), cv2 = ld(P.cv2, q2);
    const R dx4 = MX(4, i), dx4e = MX(4, i + 1);
    const R c00 = ld(P.chc, q2), c10 = ld(P.chc, qe);
    const R c01 = nrow ? ld(P.chc, qn) : 0.0, c11 = nrow ? ld(P.chc, qn + 1) : 0.0;
    const R chN0 = nrow ? 0.5 * (c00 + c01) : 0.0, chN1 = nrow ? 0.5 * (c10 + c11) : 0.0;
    const R chE0 = 0.5 * (c00 + c10), chE1 = nrow ? 0.5 * (c01 + c11) : 0.0;
    const R rh2 = RH(2, j), rh2n = nrow ? RH(2, j + 1) : 0.0;
    const R dxc = a * RH(4, j) * (dx4 + dx4e);
    const R rdxc = 1.0 / dxc;
    const int lev1 = lu;
    auto fri = [&](R vc_, R ve_, R vw_, R vn_, R vs_, R vp_km, R vp_c,
                   R vp_k1, R vce, R vcw, R v_bot_k, R vc_bot_k, R v_bot_km,
                   R vc_bot_km, R tau) -> R {
      const R wx0 = DIVARH(dvr(vc_ - vw_, dx4, RMX(4, i)), 4, j);
      const R wx1 = DIVARH(dvr(ve_ - vc_, dx4e, RMX(4, i + 1)), 4, j);
      const R wy0 = srow ? DIVA(DIVY(vc_ - vs_, 2, j)) : 0.0;
      const R wy1 = nrow ? DIVA(DIVY(vn_ - vc_, 2, j + 1)) : 0.0;
      const R va0 = chN0 * wx0, va1 = chN1 * wx1;
      const R vb0 = (chE0 * wy0) * rh2, vb1 = (chE1 * wy1) * rh2n;
      const R A = dvr(va1 - va0, dx3, rdx3);
      const R B = nrow ? dvr(vb1 - vb0, dy3, rdy3) : 0.0;
      const R wka = dvr(A + B, arh3, rarh3);
      R ans = dvr(am, sch, rsch) * wka;
      ans = ans + am * cv1 * vp_c;
      const R pxc = dvr(vce - vcw, dxc, rdxc);
      ans = ans + am * cv2 * sch * pxc;
      // wkp at kk = k and k+1: surface stress, bottom drag at lev+1, else
      // the km-scaled pz (mod_op.f90:147-161)
      auto wkp = [&](int kk, R vp_a, R vp_b, R v_bot, R vc_bot) -> R {
        if (kk == 1) return dvr(g * tau, sch, rsch);
        if (lev1 > 0 && kk == lev1 + 1) {
          const R mag = sqrt(v_bot * v_bot + vc_bot * vc_bot);
          return dvr(v_bot * g * P.c.cdbot * mag, sch, rsch);
        }
        if (kk > nk) return 0.0;
        const R pzv = dvr((vp_a - vp_b) * (R)(lev1 >= kk - 1) * (R)(lev1 >= kk), P.dz1[kk], P.rdz1[kk]);
        return dvr(grho * ld(P.km, q2 + P.n2 * (kk - 1)) * pzv, sch * sch, ld(P.rsch2, q2));
      };
      const R wkp_k = wkp(k, vp_km, vp_c, v_bot_km, vc_bot_km);
      const R wkp_k1 = wkp(k + 1, vp_c, vp_k1, v_bot_k, vc_bot_k);
      return ans * mu_k + DIVDP(wkp_k - wkp_k1, k);
    };
    // level k-1 values for a bottom drag at kk = k (lev = k-1)
    R wu_km = 0.0, wv_km = 0.0;
    if (k > 1 && lev1 == k - 1) { wu_km = dvr(u_km, sch, rsch); wv_km = dvr(v_km, sch, rsch); }
    const R tx_ = ld(P.taux, q2), ty_ = ld(P.tauy, q2);
    // fx = fri(v = uc/sch, vp = uc, vc = -(vc/sch), taux)
    const R fx = fri(wu_c, wu_e, wu_w, wu_n, wu_s, u_km, u_c, u_k1, -wv_e, -wv_w, wu_c, -wv_c, wu_km, -wv_km, tx_);
    // fy = fri(v = vc/sch, vp = vc, vc = uc/sch, tauy)
    const R fy = fri(wv_c, wv_e, wv_w, wv_n, wv_s, v_km, v_c, v_k1, wu_e, wu_w, wv_c, wu_c, wv_km, wu_km, ty_);
    const long long q = q2 + o;
    st2(P.auc, P, i, q, auc);
    st2(P.avc, P, i, q, avc);
    if (P.ab3_mode == 1) {
      st2(P.aup, P, i, q, auc); st2(P.aupp, P, i, q, auc);
      st2(P.avp, P, i, q, avc); st2(P.avpp, P, i, q, avc);
    }
    st2(P.fx, P, i, q, fx);
    st2(P.fy, P, i, q, fy);
    const R pax = ld(P.pax, q2), pay = ld(P.pay, q2);
    const R wx = -auc - sch * P.c.a0 * pax + fx;
    const R wy = -avc - sch * P.c.a0 * pay + fy;
    tu[(k - 1) * TB_X + tx] = (double)wx * P.dpr2[k] * (double)mu_k;
    tv[(k - 1) * TB_X + tx] = (double)wy * P.dpr2[k] * (double)mu_k;
  }
  __syncthreads();
  if (!ok || threadIdx.y >= 2) return;
  const double *t = threadIdx.y == 0 ? tu : tv;
  double s = 0.0;
  for (int k = 1; k <= nk; ++k) s = s + t[(k - 1) * TB_X + tx];
  st2(threadIdx.y == 0 ? P.ut : P.vt, P, i, q2, dvr(s, ld(P.prh_u, q2), ld(P.rprh_u, q2)));
}

// ----------------------------------------------------------------------------
// int_readyc's 3-D part on the FP64 path, one thread per column marching
// down the levels (the per-point arithmetic of k_readyc3d above, in the same
// order).  The column's 2-D fields and metric factors are read once; u, v
// at k-1 and k+1, w on U at k+1 (the next level's w at k) and km roll
// through registers, so a level reads only the horizontal neighbours of u
// and v, the four wm of the next level, am and km.  The depth integral of
// the baroclinic tendency accumulates in registers in level order.
constexpr int kRcX = 32, kRcY = 2;

template <bool BATCH>
__global__ void __launch_bounds__(kRcX * kRcY, 7) k_readyc_col(const __grid_constant__ DevT<double> P0,
                                                              const DevT<double> *__restrict__ Ps) {
  using R = double;
  const DevT<R> &P = BATCH ? Ps[blockIdx.z] : P0;
  const int x = blockIdx.x * kRcX + threadIdx.x;
  const int j = blockIdx.y * kRcY + threadIdx.y + P.j_lo;
  if (x >= P.glo_ni || j > P.j_hi) return;
  const int i = x + 2;
  const int nk = P.nk;
  const long long n2 = P.n2;
  const long long q2 = I2(P, i, j);
  const int ni = P.ni;
  const R g = P.c.g, a = P.c.a;
  const R grho = g * P.c.rho0;
  const bool nrow = j <= P.njm, srow = j >= 2;
  const long long qe = q2 + 1, qw = q2 - 1, qn = q2 + ni, qs = q2 - ni;
  const int lu = P.lev_u[q2];
  // column constants (k_readyc3d: the per-point prologue)
  const R sch = ld(P.sch_r, q2), rsch = ld(P.rsch, q2);
  const R rsc_e = ld(P.rsch, qe), rsc_w = ld(P.rsch, qw);
  const R sch_e = ld(P.sch_r, qe), sch_w = ld(P.sch_r, qw);
  const R rh3 = RH(3, j), dx3 = MX(3, i), rdx3 = RMX(3, i), dy3 = MY(3, j), rdy3 = RMY(3, j);
  const R arh3 = ARH(3, j), rarh3 = RARH(3, j);
  const R sn = nrow ? ld(P.sch_r, qn) : 1.0, rsn = nrow ? ld(P.rsch, qn) : 1.0;
  const R ss = srow ? ld(P.sch_r, qs) : 1.0, rss = srow ? ld(P.rsch, qs) : 1.0;
  const R rh3n = nrow ? RH(3, j + 1) : 0.0, rh3s = srow ? RH(3, j - 1) : 0.0;
  const R cv1 = ld(P.cv1, q2), cv2 = ld(P.cv2, q2);
  const R dx4 = MX(4, i), dx4e = MX(4, i + 1), rdx4 = RMX(4, i), rdx4e = RMX(4, i + 1);
  const R arh4 = ARH(4, j), rarh4 = RARH(4, j);
  const R my2 = MY(2, j), rmy2 = RMY(2, j);
  const R my2n = nrow ? MY(2, j + 1) : 1.0, rmy2n = nrow ? RMY(2, j + 1) : 1.0;
  const R c00 = ld(P.chc, q2), c10 = ld(P.chc, qe);
  const R c01 = nrow ? ld(P.chc, qn) : 0.0, c11 = nrow ? ld(P.chc, qn + 1) : 0.0;
  const R chN0 = nrow ? 0.5 * (c00 + c01) : 0.0, chN1 = nrow ? 0.5 * (c10 + c11) : 0.0;
  const R chE0 = 0.5 * (c00 + c10), chE1 = nrow ? 0.5 * (c01 + c11) : 0.0;
  const R rh2 = RH(2, j), rh2n = nrow ? RH(2, j + 1) : 0.0;
  const R dxc = a * RH(4, j) * (dx4 + dx4e);
  const R rdxc = 1.0 / dxc;
  const R rsch2 = ld(P.rsch2, q2);
  const R tx_ = ld(P.taux, q2), ty_ = ld(P.tauy, q2);
  const R pax = ld(P.pax, q2), pay = ld(P.pay, q2);
  // w on U: ter_{T->U}(wm / chc) at level kk (rows j <= njm)
  const R rc00 = ld(P.rchc, q2), rc01 = nrow ? ld(P.rchc, qn) : 1.0;
  const R rc10 = ld(P.rchc, qe), rc11 = nrow ? ld(P.rchc, qn + 1) : 1.0;
  auto wU = [&](int kk) -> R {
    if (!nrow) return 0.0;
    const long long ok_ = n2 * (kk - 1);
    return (dvr(ld(P.wm, q2 + ok_), c00, rc00) + dvr(ld(P.wm, qn + ok_), c01, rc01) +
            dvr(ld(P.wm, qe + ok_), c10, rc10) + dvr(ld(P.wm, qn + 1 + ok_), c11, rc11)) *
           0.25;
  };
  const int lev1 = lu;
  // rolling: u, v at k-1, k; w on U at k; km at k
  R u_km = 0.0, v_km = 0.0;
  R u_c = ld(P.uc, q2), v_c = ld(P.vc, q2);
  R wUk = wU(1);
  R km_k = ld(P.km, q2);
  double su = 0.0, sv = 0.0;
  for (int k = 1; k <= nk; ++k) {
    const long long o = n2 * (k - 1);
    const R mu_k = (R)(lu >= k), mu_k1 = (R)(lu >= k + 1), mu_km = (R)(lu >= k - 1);
    auto U = [&](long long q) { return ld(P.uc, q + o); };
    auto V = [&](long long q) { return ld(P.vc, q + o); };
    // velocities at level k (unweighted wu = uc/sch, wv = vc/sch)
    const R u_e = U(qe), u_w = U(qw);
    const R v_e = V(qe), v_w = V(qw);
    const R wu_c = dvr(u_c, sch, rsch), wu_e = dvr(u_e, sch_e, rsc_e), wu_w = dvr(u_w, sch_w, rsc_w);
    const R wv_c = dvr(v_c, sch, rsch), wv_e = dvr(v_e, sch_e, rsc_e), wv_w = dvr(v_w, sch_w, rsc_w);
    R u_n = 0, u_s = 0, v_n = 0, v_s = 0, wu_n = 0, wu_s = 0, wv_n = 0, wv_s = 0;
    if (nrow) {
      u_n = U(qn); v_n = V(qn);
      wu_n = dvr(u_n, sn, rsn); wv_n = dvr(v_n, sn, rsn);
    }
    if (srow) {
      u_s = U(qs); v_s = V(qs);
      wu_s = dvr(u_s, ss, rss); wv_s = dvr(v_s, ss, rss);
    }
    // vertical neighbours at (i, j)
    const R u_k1 = (k < nk) ? ld(P.uc, q2 + o + n2) : 0.0, v_k1 = (k < nk) ? ld(P.vc, q2 + o + n2) : 0.0;
    // u on N (i, j), (i+1, j); v*cos on E (i, j), (i, j+1)
    const R uN0 = 0.5 * (wu_w + wu_c), uN1 = 0.5 * (wu_c + wu_e);
    const R vE0 = srow ? 0.5 * (wv_s * rh3s + wv_c * rh3) : 0.0;
    const R vE1 = nrow ? 0.5 * (wv_c * rh3 + wv_n * rh3n) : 0.0;
    const R wUk1 = wU(k + 1);  // wm has nkp levels
    const R dm1 = dvr(uN1 - uN0, dx3, rdx3);
    const R dm2 = nrow ? dvr(vE1 - vE0, dy3, rdy3) : 0.0;
    const R dw = DIVDP(wUk - wUk1, k);
    const R rdiv = dvr(dm1 + dm2, arh3, rarh3) + dw;
    // op_adv(var)
    auto adv = [&](R x_c, R x_e, R x_w, R x_n, R x_s, R x_km, R x_k1) {
      const R wk1_0 = (0.5 * (x_w + x_c)) * uN0, wk1_1 = (0.5 * (x_c + x_e)) * uN1;
      const R wk2_0 = srow ? (0.5 * (x_s + x_c)) * vE0 : 0.0;
      const R wk2_1 = nrow ? (0.5 * (x_c + x_n)) * vE1 : 0.0;
      const R wa = dvr(wk1_1 - wk1_0, dx3, rdx3);
      const R wb = nrow ? dvr(wk2_1 - wk2_0, dy3, rdy3) : 0.0;
      R ans = dvr(wa + wb, arh3, rarh3);
      const R wkbp_k = (k >= 2) ? ((x_km + x_c) * 0.5 * wUk) * mu_km * mu_k : 0.0;
      const R wkbp_k1 = (k < nk) ? ((x_c + x_k1) * 0.5 * wUk1) * mu_k * mu_k1 : 0.0;
      ans = ans + DIVDP(wkbp_k - wkbp_k1, k);
      ans = ans - 0.5 * x_c * rdiv;
      return ans * mu_k;
    };
    const R auc = adv(u_c, u_e, u_w, u_n, u_s, u_km, u_k1);
    const R avc = adv(v_c, v_e, v_w, v_n, v_s, v_km, v_k1);
    // fri_r3d(ans, sch, v, vp, vc, tau)
    const R am = ld(P.am, q2 + o);
    const R km_k1 = ld(P.km, q2 + o + n2);  // km has nkp levels
    auto fri = [&](R vc_, R ve_, R vw_, R vn_, R vs_, R vp_km, R vp_c, R vp_k1, R vce, R vcw, R v_bot_k,
                   R vc_bot_k, R v_bot_km, R vc_bot_km, R tau) -> R {
      const R wx0 = dvr(dvr(vc_ - vw_, dx4, rdx4), arh4, rarh4);
      const R wx1 = dvr(dvr(ve_ - vc_, dx4e, rdx4e), arh4, rarh4);
      const R wy0 = srow ? DIVA(dvr(vc_ - vs_, my2, rmy2)) : 0.0;
      const R wy1 = nrow ? DIVA(dvr(vn_ - vc_, my2n, rmy2n)) : 0.0;
      const R va0 = chN0 * wx0, va1 = chN1 * wx1;
      const R vb0 = (chE0 * wy0) * rh2, vb1 = (chE1 * wy1) * rh2n;
      const R A = dvr(va1 - va0, dx3, rdx3);
      const R B = nrow ? dvr(vb1 - vb0, dy3, rdy3) : 0.0;
      const R wka = dvr(A + B, arh3, rarh3);
      R ans = dvr(am, sch, rsch) * wka;
      ans = ans + am * cv1 * vp_c;
      const R pxc = dvr(vce - vcw, dxc, rdxc);
      ans = ans + am * cv2 * sch * pxc;
      // wkp at kk = k and k+1: surface stress, bottom drag at lev+1, else
      // the km-scaled pz (mod_op.f90:147-161)
      auto wkp = [&](int kk, R vp_a, R vp_b, R v_bot, R vc_bot, R kmv) -> R {
        if (kk == 1) return dvr(g * tau, sch, rsch);
        if (lev1 > 0 && kk == lev1 + 1) {
          const R mag = sqrt(v_bot * v_bot + vc_bot * vc_bot);
          return dvr(v_bot * g * P.c.cdbot * mag, sch, rsch);
        }
        if (kk > nk) return 0.0;
        const R pzv = dvr((vp_a - vp_b) * (R)(lev1 >= kk - 1) * (R)(lev1 >= kk), P.dz1[kk], P.rdz1[kk]);
        return dvr(grho * kmv * pzv, sch * sch, rsch2);
      };
      const R wkp_k = wkp(k, vp_km, vp_c, v_bot_km, vc_bot_km, km_k);
      const R wkp_k1 = wkp(k + 1, vp_c, vp_k1, v_bot_k, vc_bot_k, km_k1);
      return ans * mu_k + DIVDP(wkp_k - wkp_k1, k);
    };
    // level k-1 values for a bottom drag at kk = k (lev = k-1)
    R wu_km = 0.0, wv_km = 0.0;
    if (k > 1 && lev1 == k - 1) { wu_km = dvr(u_km, sch, rsch); wv_km = dvr(v_km, sch, rsch); }
    // fx = fri(v = uc/sch, vp = uc, vc = -(vc/sch), taux)
    const R fx = fri(wu_c, wu_e, wu_w, wu_n, wu_s, u_km, u_c, u_k1, -wv_e, -wv_w, wu_c, -wv_c, wu_km, -wv_km, tx_);
    // fy = fri(v = vc/sch, vp = vc, vc = uc/sch, tauy)
    const R fy = fri(wv_c, wv_e, wv_w, wv_n, wv_s, v_km, v_c, v_k1, wu_e, wu_w, wv_c, wu_c, wv_km, wu_km, ty_);
    const long long q = q2 + o;
    st2(P.auc, P, i, q, auc);
    st2(P.avc, P, i, q, avc);
    if (P.ab3_mode == 1) {
      st2(P.aup, P, i, q, auc); st2(P.aupp, P, i, q, auc);
      st2(P.avp, P, i, q, avc); st2(P.avpp, P, i, q, avc);
    }
    st2(P.fx, P, i, q, fx);
    st2(P.fy, P, i, q, fy);
    const R wx = -auc - sch * P.c.a0 * pax + fx;
    const R wy = -avc - sch * P.c.a0 * pay + fy;
    su = su + (double)wx * P.dpr2[k] * (double)mu_k;
    sv = sv + (double)wy * P.dpr2[k] * (double)mu_k;
    u_km = u_c; u_c = u_k1; v_km = v_c; v_c = v_k1;
    wUk = wUk1;
    km_k = km_k1;
  }
  st2(P.ut, P, i, q2, dvr(su, ld(P.prh_u, q2), ld(P.rprh_u, q2)));
  st2(P.vt, P, i, q2, dvr(sv, ld(P.prh_u, q2), ld(P.rprh_u, q2)));
}

// ----------------------------------------------------------------------------
// int_clin (mod_int.f90:298-396): baroclinic momentum, barotropic
// replacement, unweighted velocity and its accumulation.  smag runs after.
template <typename R, bool BATCH>
__global__ void __launch_bounds__(512, 2) k_clin(const __grid_constant__ DevT<R> P0, const DevT<R> *__restrict__ Ps) {
  const DevT<R> &P = BATCH ? Ps[blockIdx.z] : P0;
  constexpr bool MIXED = std::is_same<R, float>::value;
  (void)MIXED;
  extern __shared__ double sh[];
  const int nk = P.nk;
  // column-sum terms, the two column sums, and the new u, v of the first
  // pass (as stored: rounded to R), which the second pass finishes without
  // a round trip through global memory
  double *t1s = sh, *t2s = sh + nk * TB_X, *wsum = sh + 2 * nk * TB_X;
  double *uns = wsum + 2 * TB_X, *vns = uns + nk * TB_X;
  int i, j;
  const bool ok = cell(P, i, j, true);
  const int tx = threadIdx.x;
  const long long q2 = ok ? I2(P, i, j) : 0;
  const int ni = P.ni;
  const bool nrow = j <= P.njm;
  const int lu = ok ? P.lev_u[q2] : 0;
  const long long qe = q2 + 1, qn = q2 + ni;
  const double bc = (double)P.bc;
  for (int k = threadIdx.y + 1; k <= nk && ok; k += TB_K) {
    const double sch = ld(P.schc, q2);
    // gra(mch) on E (i, j), (i, j+1) and on N (i, j), (i+1, j)
    auto gE = [&](const double *f, long long q, int jj) { return DIVARH(DIVX(ld(f, q + 1) - ld(f, q), 2, i), 2, jj); };
    auto gN = [&](const double *f, long long q) { return nrow ? DIVA(DIVY(ld(f, q + ni) - ld(f, q), 4, j)) : 0.0; };
    const double mx0 = gE(P.mch, q2, j), mx1 = nrow ? gE(P.mch, qn, j + 1) : 0.0;
    const double my0 = gN(P.mch, q2), my1 = gN(P.mch, qe);
    const double pr = P.pr2[k];
    const long long o = P.n2 * (k - 1);
    const double ph00 = ld(P.phih_t, q2), ph10 = ld(P.phih_t, qe);
    const double m00 = ld(P.mch, q2), m10 = ld(P.mch, qe);
    const double ad00 = adp_full(P, ld(P.adp, q2 + o), k, q2), ad10 = adp_full(P, ld(P.adp, qe + o), k, qe);
    const double al00 = alpha_full(P, ld(P.alpha, q2 + o), k), al10 = alpha_full(P, ld(P.alpha, qe + o), k);
    const double wk00 = ph00 + m00 * ad00, wk10 = ph10 + m10 * ad10;
    // px on E (i, j) and (i, j+1): gra(phih + mch adp) + ter(alpha) pr gra(mch)
    const double px0 = DIVARH(DIVX(wk10 - wk00, 2, i), 2, j) + 0.5 * (al00 + al10) * pr * mx0;
    double t1 = 0.0, py0 = 0.0, py1 = 0.0;
    if (nrow) {
      const double ph01 = ld(P.phih_t, qn), ph11 = ld(P.phih_t, qn + 1);
      const double m01 = ld(P.mch, qn), m11 = ld(P.mch, qn + 1);
      const double ad01 = adp_full(P, ld(P.adp, qn + o), k, qn), ad11 = adp_full(P, ld(P.adp, qn + 1 + o), k, qn + 1);
      const double al01 = alpha_full(P, ld(P.alpha, qn + o), k), al11 = alpha_full(P, ld(P.alpha, qn + 1 + o), k);
      const double wk01 = ph01 + m01 * ad01, wk11 = ph11 + m11 * ad11;
      const double px1 = DIVARH(DIVX(wk11 - wk01, 2, i), 2, j + 1) + 0.5 * (al01 + al11) * pr * mx1;
      t1 = 0.5 * (px0 + px1);
      // py on N (i, j) and (i+1, j)
      py0 = DIVA(DIVY(wk01 - wk00, 4, j)) + 0.5 * (al00 + al01) * pr * my0;
      py1 = DIVA(DIVY(wk11 - wk10, 4, j)) + 0.5 * (al10 + al11) * pr * my1;
    } else {
      py0 = 0.0 + 0.0 * pr * my0;
      py1 = 0.0 + 0.0 * pr * my1;
    }
    const double t2 = 0.5 * (py0 + py1);
    const long long q = q2 + o;
    const double pax = ld(P.pax, q2), pay = ld(P.pay, q2), cor = ld(P.cor, q2), a0 = P.c.a0;
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
    const double rw = ld(P.rwc, q2);
    const double mu = (double)(lu >= k);
    p1 = dvr(p1 * mu, w, rw);
    p2 = dvr(p2 * mu, w, rw);
    const double un = P.up[q] + p1 * bc;
    const double vn = P.vp[q] + p2 * bc;
    uns[(k - 1) * TB_X + tx] = (double)(R)un;
    vns[(k - 1) * TB_X + tx] = (double)(R)vn;
    t1s[(k - 1) * TB_X + tx] = un * P.dpr2[k] * mu;
    t2s[(k - 1) * TB_X + tx] = vn * P.dpr2[k] * mu;
  }
  __syncthreads();
  if (ok && threadIdx.y < 2) {
    const double *t = threadIdx.y == 0 ? t1s : t2s;
    double s = 0.0;
    for (int k = 1; k <= nk; ++k) s = s + t[(k - 1) * TB_X + tx];
    wsum[threadIdx.y * TB_X + tx] = dvr(s, ld(P.prh_u, q2), ld(P.rprh_u, q2));
  }
  __syncthreads();
  if (!ok) return;
  const double w1 = wsum[tx], w2 = wsum[TB_X + tx];
  const double ubc = ld(P.ubc, q2), vbc = ld(P.vbc, q2);
  const double schu = ld(P.schu, q2), mch2 = ld(P.mch2, q2), rmch2 = ld(P.rmch2, q2);
  for (int k = threadIdx.y + 1; k <= nk; k += TB_K) {
    const long long q = q2 + P.n2 * (k - 1);
    double un = uns[(k - 1) * TB_X + tx], vn = vns[(k - 1) * TB_X + tx];
    if (lu >= k) {
      un = un - w1 + ubc;
      vn = vn - w2 + vbc;
    }
    st2(P.uc, P, i, q, un);
    st2(P.vc, P, i, q, vn);
    st2(P.up, P, i, q, un);
    st2(P.vp, P, i, q, vn);
    const double uu = dvr(un * schu, mch2, rmch2), vv = dvr(vn * schu, mch2, rmch2);
    st2(P.uu, P, i, q, uu);
    st2(P.vv, P, i, q, vv);
    st2(P.acu, P, i, q, P.acu[q] + uu);
    st2(P.acv, P, i, q, P.acv[q] + vv);
  }
}

// ----------------------------------------------------------------------------
// smag (mod_int.f90:403-440): Smagorinsky viscosity, rows 2..nj-1.
constexpr int kSmagK = 4;  // levels per thread of a single-domain launch
template <typename R, bool BATCH>
__global__ void k_smag(const __grid_constant__ DevT<R> P0, const DevT<R> *__restrict__ Ps) {
  const DevT<R> &P = BATCH ? Ps[blockIdx.z] : P0;
  constexpr bool MIXED = std::is_same<R, float>::value;
  (void)MIXED;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + smag_j0(P);
  if (x >= P.glo_ni || j > smag_j1(P)) return;
  const int i = x + 2;
  const long long q2 = I2(P, i, j);
  const int ni = P.ni;
  const R dx = ld(P.dxs, q2), rdx = ld(P.rdxs, q2);
  const R dy = __ldg(P.dys1d + j - 1), rdy = __ldg(P.rdys1d + j - 1);
  const R tn = ld(P.tn3, q2);
  const R *u = P.uu, *v = P.vv;
  // one domain: grid z splits the levels into groups of kSmagK; a batch
  // (grid z = member) walks all levels
  const int k0 = BATCH ? 1 : (int)blockIdx.z * kSmagK + 1;
  const int k1 = BATCH ? P.nk : min(P.nk, k0 + kSmagK - 1);
  for (int k = k0; k <= k1; ++k) {
  const long long q = q2 + P.n2 * (k - 1);
  const R dt = dvr(4 * (ld(u, q + 1) - ld(u, q - 1)), dx, rdx) - dvr(4 * (ld(v, q + ni) - ld(v, q - ni)), dy, rdy) +
                    DIVA(ld(v, q) * tn);
  const R ds = dvr(4 * (ld(v, q + 1) - ld(v, q - 1)), dx, rdx) + dvr(4 * (ld(u, q + ni) - ld(u, q - ni)), dy, rdy) -
                    DIVA(ld(u, q) * tn);
  R c = 0.5 * P.c.smag_c / P.c.pi * (0.5 * dx + 0.5 * dy);
  c = c * c;
  const R wk = c * sqrt(dt * dt + ds * ds);
  const R am_max = dvr(dx * dx + dy * dy, (R)(4 * 8 * P.bc), P.rbc32);
  st2(P.am, P, i, q, wk < am_max ? wk : am_max);
  if (MIXED && k == 1) st2(P.am1, P, i, q, wk < am_max ? wk : am_max);
  }
}

// ----------------------------------------------------------------------------
// int_ssh (mod_int.f90:602-624): alpha from (tp, sp, mch), SSH accumulation.
template <typename R, bool BATCH>
__global__ void __launch_bounds__(512) k_ssh(const __grid_constant__ DevT<R> P0, const DevT<R> *__restrict__ Ps) {
  const DevT<R> &P = BATCH ? Ps[blockIdx.z] : P0;
  constexpr bool MIXED = std::is_same<R, float>::value;
  (void)MIXED;
  extern __shared__ double sh[];
  const int nk = P.nk;
  int i, j;
  const bool ok = cell(P, i, j, false);
  const int tx = threadIdx.x;
  const long long q2 = ok ? I2(P, i, j) : 0;
  const int lev = ok ? P.lev_t[q2] : 0;
  const double mch = ok ? P.mch[q2] : 0.0;
  for (int k = threadIdx.y + 1; k <= nk && ok; k += TB_K) {
    const long long q = q2 + P.n2 * (k - 1);
    double al;
    if (k <= lev) {
      al = 1.0 / den_rho(P.c, P.tp[q], P.sp[q], mch * P.pr2[k]);
      P.alpha[q] = alpha_store(P, al, k);
    } else {
      al = alpha_full(P, P.alpha[q], k);
    }
    sh[(k - 1) * TB_X + tx] = al * P.dpr2[k] * mch * (double)(k <= lev);
  }
  __syncthreads();
  if (!ok || threadIdx.y != 0) return;
  double s = 0.0;
  for (int k = 1; k <= nk; ++k) s = s + sh[(k - 1) * TB_X + tx];
  double ssh = dvr(s, P.c.g, P.rg);
  ssh = dvr(P.phih_t[q2], P.c.g, P.rg) + ssh;
  P.acssh[q2] = P.acssh[q2] + ssh;
}

// ----------------------------------------------------------------------------
// int_ts (mod_int.f90:442-507) after upwelling: tracer advection op_adv_ts
// (mod_op.f90:280-325), diffusion op_dif (mod_op.f90:186-222), surface
// restoring, time step, ice floor, convective adjustment (convect/adjust/mix,
// mod_int.f90:509-600), tp = tc, and the act/acs/acr accumulations.
struct Col {  // one column of T, S and prho in shared memory, stride TB_X
  double *t, *s, *p1, *p2;
  __device__ double &T(int k) { return t[(k - 1) * TB_X]; }
  __device__ double &S(int k) { return s[(k - 1) * TB_X]; }
  __device__ double P1(int k) const { return p1[(k - 1) * TB_X]; }
  __device__ double P2(int k) const { return p2[(k - 1) * TB_X]; }
};

template <typename R, typename C>
__device__ void ts_mix(const DevT<R> &P, long long q2, C &c, double *rhoa, double *rhob, int na, int nb) {
  double st = 0.0, sd = 0.0;
  for (int k = na; k <= nb; ++k) st = st + c.T(k) * P.dpr2[k];
  for (int k = na; k <= nb; ++k) sd = sd + P.dpr2[k];
  const double tn = st / sd;
  for (int k = na; k <= nb; ++k) c.T(k) = tn;
  double ss = 0.0;
  for (int k = na; k <= nb; ++k) ss = ss + c.S(k) * P.dpr2[k];
  const double sn = ss / sd;
  for (int k = na; k <= nb; ++k) c.S(k) = sn;
  for (int k = na; k <= nb; ++k) rhoa[k] = c.P1(k) * c.T(k) + c.P2(k) * c.S(k);
  for (int k = na; k <= nb - 1; ++k) rhob[k] = c.P1(k + 1) * c.T(k) + c.P2(k + 1) * c.S(k);
  if (nb < P.nk) rhob[nb] = c.P1(nb + 1) * c.T(nb) + c.P2(nb + 1) * c.S(nb);
}

template <typename R, typename C>
__device__ void ts_convect(const DevT<R> &P, long long q2, int nlev, C c) {
  double rhoa[PCOM_MAXK + 2], rhob[PCOM_MAXK + 2];
  for (int k = 0; k <= P.nk + 1; ++k) { rhoa[k] = 0.0; rhob[k] = 0.0; }
  for (int k = 2; k <= nlev; ++k) rhoa[k] = c.P1(k) * c.T(k) + c.P2(k) * c.S(k);
  for (int k = 1; k <= nlev - 1; ++k) rhob[k] = c.P1(k + 1) * c.T(k) + c.P2(k + 1) * c.S(k);
  int kcnt = 1, guard = 0;
  while (kcnt < nlev && guard < 4 * PCOM_MAXK * PCOM_MAXK) {
    ++guard;
    if (rhob[kcnt] > rhoa[kcnt + 1]) {
      // adjust (mod_int.f90:544-581)
      int na = kcnt, nb = kcnt + 1;
      ts_mix(P, q2, c, rhoa, rhob, na, nb);
      while (nb < nlev) {
        if (rhob[nb] > rhoa[nb + 1]) {
          nb = nb + 1;
          ts_mix(P, q2, c, rhoa, rhob, na, nb);
        } else {
          if ((na <= 1) || (rhob[na - 1] <= rhoa[na])) break;
          na = na - 1;
          ts_mix(P, q2, c, rhoa, rhob, na, nb);
        }
      }
      while (na > 1) {
        if (rhob[na - 1] <= rhoa[na]) break;
        na = na - 1;
        ts_mix(P, q2, c, rhoa, rhob, na, nb);
      }
      kcnt = nb;
    } else {
      kcnt = kcnt + 1;
    }
  }
}

template <typename R, bool BATCH>
// (FP32 storage: registers for two CTAs per SM)
__global__ void __launch_bounds__(512, sizeof(R) == 4 ? 2 : 1) k_ts(const __grid_constant__ DevT<R> P0,
                                                                    const DevT<R> *__restrict__ Ps) {
  const DevT<R> &P = BATCH ? Ps[blockIdx.z] : P0;
  constexpr bool MIXED = std::is_same<R, float>::value;
  (void)MIXED;
  extern __shared__ double sh[];
  const int nk = P.nk;
  double *tcs = sh, *scs = sh + nk * TB_X, *p1s = sh + 2 * nk * TB_X, *p2s = sh + 3 * nk * TB_X;
  __shared__ int unstable[TB_X];
  int i, j;
  const bool ok = cell(P, i, j, true);
  const int tx = threadIdx.x;
  const long long q2 = ok ? I2(P, i, j) : 0;
  const int ni = P.ni;
  const R g = P.c.g;
  if (threadIdx.y == 0) unstable[tx] = 0;
  const R grho = g * P.c.rho0;
  const bool nrow = j <= P.njm, srow = j >= 2;
  const long long qw = q2 - 1, qs = q2 - ni, qsw = qs - 1, qe = q2 + 1, qn = q2 + ni;
  const int lev = ok ? P.lev_t[q2] : 0;
  for (int k = threadIdx.y + 1; k <= nk && ok; k += TB_K) {
    const int lw = P.lev_t[qw], le = P.lev_t[qe], ln = nrow ? P.lev_t[qn] : 0, ls = srow ? P.lev_t[qs] : 0;
    const R rh4c = RH(4, j), rh4s = srow ? RH(4, j - 1) : 0.0;
    // sch (op_adv_ts) at U (i, j), (i-1, j), (i, j-1), (i-1, j-1)
    const R sc_c = ld(P.sch_r, q2), sc_w = ld(P.sch_r, qw);
    const R sc_s = srow ? ld(P.sch_r, qs) : 0.0, sc_sw = srow ? ld(P.sch_r, qsw) : 0.0;
    const R r3c = RH(3, j), r3s = srow ? RH(3, j - 1) : 0.0;
    // ter(mch) to E (i-1, j), (i, j) and to N (i, j-1), (i, j)
    const R mc = ld(P.mch, q2), me = ld(P.mch, qe), mw = ld(P.mch, qw);
    const R mn = nrow ? ld(P.mch, qn) : 0.0, ms = srow ? ld(P.mch, qs) : 0.0;
    const R c1c = 0.5 * (mc + me), c1w = 0.5 * (mw + mc);
    const R c2c = nrow ? 0.5 * (mc + mn) : 0.0, c2s = srow ? 0.5 * (ms + mc) : 0.0;
    const R bc = (R)P.bc;
    const long long o = P.n2 * (k - 1), q = q2 + o;
    const R m_c = (R)(lev >= k), m_w = (R)(lw >= k), m_e = (R)(le >= k);
    const R m_n = (R)(ln >= k), m_s = (R)(ls >= k);
    const R m_k1 = (R)(lev >= k + 1), m_km = (R)(lev >= k - 1);
    // mass-weighted velocity: um1 = uc*sch on U, um2 = vc*sch*rh3
    const R um1c = ld(P.uc, q) * sc_c, um1w = ld(P.uc, qw + o) * sc_w;
    const R um1s = srow ? ld(P.uc, qs + o) * sc_s : 0.0, um1sw = srow ? ld(P.uc, qsw + o) * sc_sw : 0.0;
    const R um2c = ld(P.vc, q) * sc_c * r3c, um2w = ld(P.vc, qw + o) * sc_w * r3c;
    const R um2s = srow ? ld(P.vc, qs + o) * sc_s * r3s : 0.0;
    const R um2sw = srow ? ld(P.vc, qsw + o) * sc_sw * r3s : 0.0;
    // ter U->E (ns, sj=1) at (i, j), (i-1, j); ter U->N (ew, si=1) at (i, j), (i, j-1)
    const R wa1c = srow ? 0.5 * (um1s + um1c) : 0.0, wa1w = srow ? 0.5 * (um1sw + um1w) : 0.0;
    const R wa2c = 0.5 * (um2w + um2c), wa2s = srow ? 0.5 * (um2sw + um2s) : 0.0;
    const R wmk = ld(P.wm, q), wmk1 = ld(P.wm, q + P.n2);  // wm has nkp levels
    auto adv = [&](const R *var) -> R {
      const R xc = ld(var, q), xe = ld(var, qe + o), xw = ld(var, qw + o);
      const R xn = nrow ? ld(var, qn + o) : 0.0, xs = srow ? ld(var, qs + o) : 0.0;
      const R xkm = (k > 1) ? ld(var, q - P.n2) : 0.0, xk1 = (k < nk) ? ld(var, q + P.n2) : 0.0;
      const R w1c = DIVX(xe - xc, 2, i), w1w = DIVX(xc - xw, 2, i - 1);
      const R wb1 = 0.5 * (wa1w * w1w + wa1c * w1c);
      R ans = DIVARH(wb1, 1, j);
      const R w2c = nrow ? DIVY(xn - xc, 4, j) : 0.0;
      R wb2 = 0.0;
      if (srow) {
        const R w2s = DIVY(xc - xs, 4, j - 1);
        wb2 = 0.5 * (wa2s * w2s + wa2c * w2c);
      }
      ans = ans + DIVARH(wb2, 1, j);
      // vter(wm * dx3(var)) / dpr
      const R wmp_k = (k >= 2) ? wmk * (xkm - xc) : wmk * 0.0;
      const R wmp_k1 = (k < nk) ? wmk1 * (xc - xk1) : wmk1 * 0.0;
      ans = ans + DIVDP((wmp_k + wmp_k1) * 0.5, k);
      return ans;
    };
    auto dif = [&](const R *var) -> R {
      const R xc = ld(var, q), xe = ld(var, qe + o), xw = ld(var, qw + o);
      const R xn = nrow ? ld(var, qn + o) : 0.0, xs = srow ? ld(var, qs + o) : 0.0;
      const R xkm = (k > 1) ? ld(var, q - P.n2) : 0.0, xk1 = (k < nk) ? ld(var, q + P.n2) : 0.0;
      const R w1c = DIVARH(DIVX((xe - xc) * m_e * m_c, 2, i), 2, j);
      const R w1w = DIVARH(DIVX((xc - xw) * m_c * m_w, 2, i - 1), 2, j);
      const R A = DIVX(c1c * w1c - c1w * w1w, 1, i);
      const R w2c = nrow ? DIVA(DIVY((xn - xc) * m_n * m_c, 4, j)) : 0.0;
      R B = 0.0;
      if (srow) {
        const R w2s = DIVA(DIVY((xc - xs) * m_c * m_s, 4, j - 1));
        B = DIVY((c2c * w2c) * rh4c - (c2s * w2s) * rh4s, 1, j);
      }
      R ans = P.c.ah_c * DIVARH(A + B, 1, j);
      R wkp_k = 0.0, wkp_k1 = 0.0;
      if (k >= 2) {
        const R pz = dvr((xkm - xc) * m_km * m_c, P.dz1[k], P.rdz1[k]);
        wkp_k = grho * ld(P.kh, q2 + P.n2 * (k - 1)) * pz;
      }
      if (k < nk) {
        const R pz = dvr((xc - xk1) * m_c * m_k1, P.dz1[k + 1], P.rdz1[k + 1]);
        wkp_k1 = grho * ld(P.kh, q2 + P.n2 * k) * pz;
      }
      ans = ans + DIVDP(wkp_k - wkp_k1, k);
      return ans;
    };
    const R at = adv(P.tc), as = adv(P.sc);
    const R dt_ = dif(P.tp), ds_ = dif(P.sp);
    R p1 = -at, p2 = -as;
    p1 = p1 + dt_;
    p2 = p2 + ds_;
    if (k == 1) {
      p1 = p1 + DIVDP(P.c.gamma_t * (ld(P.bnd_t, q2) - ld(P.tc, q)) * m_c, 1);
      p2 = p2 + P.c.gamma_s * (ld(P.bnd_s, q2) - ld(P.sc, q)) * m_c * mc;
    }
    // the tracer update in FP64 (mixed path: FP32 tendency, FP64 sum)
    const double rmc = ld(P.rmch, q2);
    double tn = (double)ld(P.tp, q) + dvr((double)(p1 * bc * m_c), (double)mc, rmc);
    const double sn = (double)ld(P.sp, q) + dvr((double)(p2 * bc * m_c), (double)mc, rmc);
    if (m_c > 0 && tn < P.c.tice) tn = P.c.tice;
    tcs[(k - 1) * TB_X + tx] = tn;
    scs[(k - 1) * TB_X + tx] = sn;
    const auto pr = P.prho[q];
    p1s[(k - 1) * TB_X + tx] = pr.x;
    p2s[(k - 1) * TB_X + tx] = pr.y;
  }
  __syncthreads();
  // the adjustment scan of convect starts only where rhob(k) > rhoa(k+1)
  // for some 1 <= k < nlev (mod_int.f90:530-537); test every level at once
  for (int k = threadIdx.y + 1; k < lev && ok; k += TB_K) {
    const int o = (k - 1) * TB_X + tx, o1 = k * TB_X + tx;
    const double rb = p1s[o1] * tcs[o] + p2s[o1] * scs[o];
    const double ra = p1s[o1] * tcs[o1] + p2s[o1] * scs[o1];
    if (rb > ra) unstable[tx] = 1;
  }
  __syncthreads();
  if (ok && threadIdx.y == 0 && lev > 1 && unstable[tx]) {
    Col c{tcs + tx, scs + tx, p1s + tx, p2s + tx};
    ts_convect(P, q2, lev, c);
  }
  __syncthreads();
  if (!ok) return;
  const double chc = ld(P.chc, q2);
  for (int k = threadIdx.y + 1; k <= nk; k += TB_K) {
    const long long q = q2 + P.n2 * (k - 1);
    const double tn = tcs[(k - 1) * TB_X + tx], sn = scs[(k - 1) * TB_X + tx];
    st2(P.tn_, P, i, q, tn);
    st2(P.sn_, P, i, q, sn);
    st2(P.act, P, i, q, P.act[q] + tn);
    st2(P.acs, P, i, q, P.acs[q] + sn);
    if (k <= lev) {
      const double w = 1.0 / den_rho(P.c, tn, sn, chc * P.pr2[k]);
      st2(P.acr, P, i, q, P.acr[q] + 1.0 / w);
    }
  }
}

// ----------------------------------------------------------------------------
// int_ts on the FP64 path in two kernels (the per-point arithmetic of k_ts
// above, in the same order).
//
// k_ts_col: one thread per column marching down the levels.  The column's
// masks, 2-D fields and metric factors are read once; the vertical
// neighbours of T, S, tp, sp, wm and kh roll through registers, so a level
// reads only the horizontal neighbours.  The new T, S of the column go to
// the output buffers as they are formed; a column whose density test finds
// an instability (rhob(k) > rhoa(k+1) for some k < lev) is copied to local
// arrays, adjusted there (convect) and written back.  The output buffers are
// never a tracer buffer this kernel reads (three-buffer pool).
//
// k_ts_acc: point-parallel, the halo twins of the new T, S and the
// act/acs/acr accumulations (acr through the equation of state).
constexpr int kColX = 32, kColY = 2;

// one column of T, S and prho copied to local arrays, levels 1..nlev (+1 for prho)
struct ColL {
  double *t, *s, *p1, *p2;
  __device__ double &T(int k) { return t[k - 1]; }
  __device__ double &S(int k) { return s[k - 1]; }
  __device__ double P1(int k) const { return p1[k - 1]; }
  __device__ double P2(int k) const { return p2[k - 1]; }
};

template <bool BATCH>
__global__ void __launch_bounds__(kColX * kColY, 7) k_ts_col(const __grid_constant__ DevT<double> P0,
                                                            const DevT<double> *__restrict__ Ps) {
  using R = double;
  const DevT<R> &P = BATCH ? Ps[blockIdx.z] : P0;
  const int x = blockIdx.x * kColX + threadIdx.x;
  const int j = blockIdx.y * kColY + threadIdx.y + P.j_lo;
  if (x >= P.glo_ni || j > P.j_hi) return;
  const int i = x + 2;
  const int nk = P.nk;
  const long long n2 = P.n2;
  const long long q2 = I2(P, i, j);
  const int ni = P.ni;
  const R g = P.c.g;
  const R grho = g * P.c.rho0;
  const bool nrow = j <= P.njm, srow = j >= 2;
  const long long qw = q2 - 1, qs = q2 - ni, qsw = qs - 1, qe = q2 + 1, qn = q2 + ni;
  const int lev = P.lev_t[q2];
  // column constants (k_ts: the per-point prologue)
  const int lw = P.lev_t[qw], le = P.lev_t[qe], ln = nrow ? P.lev_t[qn] : 0, ls = srow ? P.lev_t[qs] : 0;
  const R rh4c = RH(4, j), rh4s = srow ? RH(4, j - 1) : 0.0;
  const R sc_c = ld(P.sch_r, q2), sc_w = ld(P.sch_r, qw);
  const R sc_s = srow ? ld(P.sch_r, qs) : 0.0, sc_sw = srow ? ld(P.sch_r, qsw) : 0.0;
  const R r3c = RH(3, j), r3s = srow ? RH(3, j - 1) : 0.0;
  const R mc = ld(P.mch, q2), me = ld(P.mch, qe), mw = ld(P.mch, qw);
  const R mn = nrow ? ld(P.mch, qn) : 0.0, ms = srow ? ld(P.mch, qs) : 0.0;
  const R c1c = 0.5 * (mc + me), c1w = 0.5 * (mw + mc);
  const R c2c = nrow ? 0.5 * (mc + mn) : 0.0, c2s = srow ? 0.5 * (ms + mc) : 0.0;
  const R bc = (R)P.bc;
  const double rmc = ld(P.rmch, q2);
  // metric factors of the divisions (the DIVX/DIVY/DIVARH operands)
  const R mx2c = MX(2, i), rmx2c = RMX(2, i), mx2w = MX(2, i - 1), rmx2w = RMX(2, i - 1);
  const R mx1c = MX(1, i), rmx1c = RMX(1, i);
  const R my4c = MY(4, j), rmy4c = RMY(4, j), my1c = MY(1, j), rmy1c = RMY(1, j);
  const R my4s = srow ? MY(4, j - 1) : 1.0, rmy4s = srow ? RMY(4, j - 1) : 1.0;
  const R arh1 = ARH(1, j), rarh1 = RARH(1, j), arh2 = ARH(2, j), rarh2 = RARH(2, j);
  // rolling vertical neighbours: x(k-1), x(k)
  R tc_m = 0, tc_c = ld(P.tc, q2), sc_m = 0, sc_cc = ld(P.sc, q2);
  R tp_m = 0, tp_c = ld(P.tp, q2), sp_m = 0, sp_c = ld(P.sp, q2);
  R wm_c = ld(P.wm, q2), kh_c = ld(P.kh, q2);
  double t_prev = 0.0, s_prev = 0.0;
  bool unstable = false;
  for (int k = 1; k <= nk; ++k) {
    const long long o = n2 * (k - 1), q = q2 + o;
    const R m_c = (R)(lev >= k), m_w = (R)(lw >= k), m_e = (R)(le >= k);
    const R m_n = (R)(ln >= k), m_s = (R)(ls >= k);
    const R m_k1 = (R)(lev >= k + 1), m_km = (R)(lev >= k - 1);
    // mass-weighted velocity: um1 = uc*sch on U, um2 = vc*sch*rh3
    const R um1c = ld(P.uc, q) * sc_c, um1w = ld(P.uc, qw + o) * sc_w;
    const R um1s = srow ? ld(P.uc, qs + o) * sc_s : 0.0, um1sw = srow ? ld(P.uc, qsw + o) * sc_sw : 0.0;
    const R um2c = ld(P.vc, q) * sc_c * r3c, um2w = ld(P.vc, qw + o) * sc_w * r3c;
    const R um2s = srow ? ld(P.vc, qs + o) * sc_s * r3s : 0.0;
    const R um2sw = srow ? ld(P.vc, qsw + o) * sc_sw * r3s : 0.0;
    const R wa1c = srow ? 0.5 * (um1s + um1c) : 0.0, wa1w = srow ? 0.5 * (um1sw + um1w) : 0.0;
    const R wa2c = 0.5 * (um2w + um2c), wa2s = srow ? 0.5 * (um2sw + um2s) : 0.0;
    const R wmk = wm_c, wmk1 = ld(P.wm, q + n2);  // wm has nkp levels
    const R khk = kh_c, khk1 = (k < nk) ? ld(P.kh, q + n2) : 0.0;
    auto adv = [&](const R *var, R xc, R xkm, R xk1) -> R {
      const R xe = ld(var, qe + o), xw = ld(var, qw + o);
      const R xn = nrow ? ld(var, qn + o) : 0.0, xs = srow ? ld(var, qs + o) : 0.0;
      const R w1c = dvr(xe - xc, mx2c, rmx2c), w1w = dvr(xc - xw, mx2w, rmx2w);
      const R wb1 = 0.5 * (wa1w * w1w + wa1c * w1c);
      R ans = dvr(wb1, arh1, rarh1);
      const R w2c = nrow ? dvr(xn - xc, my4c, rmy4c) : 0.0;
      R wb2 = 0.0;
      if (srow) {
        const R w2s = dvr(xc - xs, my4s, rmy4s);
        wb2 = 0.5 * (wa2s * w2s + wa2c * w2c);
      }
      ans = ans + dvr(wb2, arh1, rarh1);
      const R wmp_k = (k >= 2) ? wmk * (xkm - xc) : wmk * 0.0;
      const R wmp_k1 = (k < nk) ? wmk1 * (xc - xk1) : wmk1 * 0.0;
      ans = ans + DIVDP((wmp_k + wmp_k1) * 0.5, k);
      return ans;
    };
    auto dif = [&](const R *var, R xc, R xkm, R xk1) -> R {
      const R xe = ld(var, qe + o), xw = ld(var, qw + o);
      const R xn = nrow ? ld(var, qn + o) : 0.0, xs = srow ? ld(var, qs + o) : 0.0;
      const R w1c = dvr(dvr((xe - xc) * m_e * m_c, mx2c, rmx2c), arh2, rarh2);
      const R w1w = dvr(dvr((xc - xw) * m_c * m_w, mx2w, rmx2w), arh2, rarh2);
      const R A = dvr(c1c * w1c - c1w * w1w, mx1c, rmx1c);
      const R w2c = nrow ? DIVA(dvr((xn - xc) * m_n * m_c, my4c, rmy4c)) : 0.0;
      R B = 0.0;
      if (srow) {
        const R w2s = DIVA(dvr((xc - xs) * m_c * m_s, my4s, rmy4s));
        B = dvr((c2c * w2c) * rh4c - (c2s * w2s) * rh4s, my1c, rmy1c);
      }
      R ans = P.c.ah_c * dvr(A + B, arh1, rarh1);
      R wkp_k = 0.0, wkp_k1 = 0.0;
      if (k >= 2) {
        const R pz = dvr((xkm - xc) * m_km * m_c, P.dz1[k], P.rdz1[k]);
        wkp_k = grho * khk * pz;
      }
      if (k < nk) {
        const R pz = dvr((xc - xk1) * m_c * m_k1, P.dz1[k + 1], P.rdz1[k + 1]);
        wkp_k1 = grho * khk1 * pz;
      }
      ans = ans + DIVDP(wkp_k - wkp_k1, k);
      return ans;
    };
    const R tc_k1 = (k < nk) ? ld(P.tc, q + n2) : 0.0, sc_k1 = (k < nk) ? ld(P.sc, q + n2) : 0.0;
    const R tp_k1 = (k < nk) ? ld(P.tp, q + n2) : 0.0, sp_k1 = (k < nk) ? ld(P.sp, q + n2) : 0.0;
    const R at = adv(P.tc, tc_c, tc_m, tc_k1), as = adv(P.sc, sc_cc, sc_m, sc_k1);
    const R dt_ = dif(P.tp, tp_c, tp_m, tp_k1), ds_ = dif(P.sp, sp_c, sp_m, sp_k1);
    R p1 = -at, p2 = -as;
    p1 = p1 + dt_;
    p2 = p2 + ds_;
    if (k == 1) {
      p1 = p1 + DIVDP(P.c.gamma_t * (ld(P.bnd_t, q2) - tc_c) * m_c, 1);
      p2 = p2 + P.c.gamma_s * (ld(P.bnd_s, q2) - sc_cc) * m_c * mc;
    }
    double tn = (double)tp_c + dvr((double)(p1 * bc * m_c), (double)mc, rmc);
    const double sn = (double)sp_c + dvr((double)(p2 * bc * m_c), (double)mc, rmc);
    if (m_c > 0 && tn < P.c.tice) tn = P.c.tice;
    P.tn_[q] = tn;
    P.sn_[q] = sn;
    // convect's trigger: rhob(k-1) > rhoa(k) for 1 <= k-1 < lev
    if (k >= 2 && k <= lev) {
      const double2 pr = P.prho[q];
      const double rb = pr.x * t_prev + pr.y * s_prev;
      const double ra = pr.x * tn + pr.y * sn;
      if (rb > ra) unstable = true;
    }
    t_prev = tn;
    s_prev = sn;
    tc_m = tc_c; tc_c = tc_k1; sc_m = sc_cc; sc_cc = sc_k1;
    tp_m = tp_c; tp_c = tp_k1; sp_m = sp_c; sp_c = sp_k1;
    wm_c = wmk1; kh_c = khk1;
  }
  if (lev > 1 && unstable) {
    // convect reads prho one level below the adjusted range
    double t[PCOM_MAXK], s_[PCOM_MAXK], p1[PCOM_MAXK], p2[PCOM_MAXK];
    const int np = lev < nk ? lev + 1 : nk;
    for (int k = 1; k <= np; ++k) {
      const long long q = q2 + n2 * (k - 1);
      const double2 pr = P.prho[q];
      p1[k - 1] = pr.x;
      p2[k - 1] = pr.y;
      t[k - 1] = P.tn_[q];
      s_[k - 1] = P.sn_[q];
    }
    ts_convect(P, q2, lev, ColL{t, s_, p1, p2});
    for (int k = 1; k <= lev; ++k) {
      const long long q = q2 + n2 * (k - 1);
      P.tn_[q] = t[k - 1];
      P.sn_[q] = s_[k - 1];
    }
  }
}

template <bool BATCH>
__global__ void __launch_bounds__(512, 2) k_ts_acc(const __grid_constant__ DevT<double> P0,
                                                const DevT<double> *__restrict__ Ps) {
  const DevT<double> &P = BATCH ? Ps[blockIdx.z] : P0;
  int i, j;
  if (!cell(P, i, j, true)) return;
  const long long q2 = I2(P, i, j);
  const int lev = P.lev_t[q2];
  const double chc = ld(P.chc, q2);
  const int ni = P.ni;
  const bool twin = i == 2 || i == ni - 1;
  const long long dq = i == 2 ? (long long)(ni - 2) : -(long long)(ni - 2);
  for (int k = threadIdx.y + 1; k <= P.nk; k += TB_K) {
    const long long q = q2 + P.n2 * (k - 1);
    const double tn = P.tn_[q], sn = P.sn_[q];
    if (twin) {
      P.tn_[q + dq] = tn;
      P.sn_[q + dq] = sn;
    }
    st2(P.act, P, i, q, P.act[q] + tn);
    st2(P.acs, P, i, q, P.acs[q] + sn);
    if (k <= lev) {
      const double w = 1.0 / den_rho(P.c, tn, sn, chc * P.pr2[k]);
      st2(P.acr, P, i, q, P.acr[q] + 1.0 / w);
    }
  }
}

// ----------------------------------------------------------------------------
// den_prho (mod_den.f90:120-153)
template <typename R, bool BATCH>
__global__ void __launch_bounds__(512) k_den_prho(const __grid_constant__ DevT<R> P0, const DevT<R> *__restrict__ Ps) {
  const DevT<R> &P = BATCH ? Ps[blockIdx.z] : P0;
  constexpr bool MIXED = std::is_same<R, float>::value;
  (void)MIXED;
  int i, j;
  if (!cell(P, i, j, false)) return;
  const long long q2 = I2(P, i, j);
  const int lev = P.lev_t[q2];
  const double ch = P.chc[q2];
  const double dt = P.c.deltat, ds = P.c.deltas;
  for (int k = threadIdx.y + 1; k <= lev && k <= P.nk; k += TB_K) {
    const long long q = q2 + P.n2 * (k - 1);
    const double t = P.tc[q], s = P.sc[q], p = ch * P.pr2[k];
    double ra = den_rho(P.c, t + dt, s, p), rb = den_rho(P.c, t - dt, s, p);
    typename Vec2<R>::type r;
    r.x = (ra - rb) / (2 * dt);
    ra = den_rho(P.c, t, s + ds, p);
    rb = den_rho(P.c, t, s - ds, p);
    r.y = (ra - rb) / (2 * ds);
    P.prho[q] = r;
  }
}

}  // namespace

// ---------------------------------------------------------------- launchers
// Single domain: the Dev travels as a kernel parameter.  Batch: Ps[m] in
// device memory describes member m = blockIdx.z; the grid is sized to the
// largest member and CTAs outside a smaller member's domain do nothing.
static const dim3 kBlock3(TB_X, TB_K, 1);
static inline dim3 g3(int nx, int ny, int nz) { return dim3((nx + TB_X - 1) / TB_X, ny, nz); }
// rows of the handle's row window (all rows 1..nj unless the domain is split)
template <typename R>
static inline int wrows(const DevT<R> &P) { return P.j_hi - P.j_lo + 1; }
static inline size_t sm3(int nk, int planes) { return (size_t)planes * nk * TB_X * sizeof(double); }
// k_clin: four level planes (column-sum terms, new u and v) and the two sums
static inline size_t clin_smem(int nk) { return sm3(nk, 4) + 2 * TB_X * sizeof(double); }

template <typename R>
void launch_alpha_tobot(const DevT<R> &P, cudaStream_t s) { k_alpha_tobot<R, false><<<g3(P.ni, wrows(P), 1), kBlock3, sm3(P.nk, 1), s>>>(P, nullptr); }
template <typename R>
void launch_pgra2d(const DevT<R> &P, cudaStream_t s) { k_pgra2d<R, false><<<g3(P.glo_ni, wrows(P), 1), kBlock3, sm3(P.nk, 4), s>>>(P, nullptr); }
template <typename R>
void launch_uv2d(const DevT<R> &P, int mode, cudaStream_t s) {
  k_uv2d<R, false><<<dim3((P.glo_ni + 31) / 32, (P.nj + 3) / 4), dim3(32, 4), 0, s>>>(P, nullptr, mode);
}
template <typename R>
void launch_upwelling(const DevT<R> &P, int with_acw, cudaStream_t s) {
  constexpr int UX = upw_cols<R>();
  k_upwelling<R, false><<<dim3((P.glo_ni + UX - 1) / UX, wrows(P), 1), dim3(UX, TB_K, 1),
                          (size_t)3 * P.nk * UX * sizeof(double), s>>>(P, nullptr, with_acw);
}
template <typename R>
void launch_readyc3d(const DevT<R> &P, cudaStream_t s) {
  if constexpr (std::is_same<R, double>::value)
    k_readyc_col<false><<<dim3((P.glo_ni + kRcX - 1) / kRcX, (wrows(P) + kRcY - 1) / kRcY), dim3(kRcX, kRcY), 0, s>>>(P, nullptr);
  else
    k_readyc3d<R, false><<<g3(P.glo_ni, wrows(P), 1), kBlock3, sm3(P.nk, 2), s>>>(P, nullptr);
}
template <typename R>
void launch_clin(const DevT<R> &P, cudaStream_t s) {
  const size_t smem = clin_smem(P.nk);
  static const cudaError_t attr =
      cudaFuncSetAttribute(k_clin<R, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)clin_smem(PCOM_MAXK));
  (void)attr;
  k_clin<R, false><<<g3(P.glo_ni, wrows(P), 1), kBlock3, smem, s>>>(P, nullptr);
}
template <typename R>
void launch_smag(const DevT<R> &P, cudaStream_t s) {
  const int rows = smag_j1(P) - smag_j0(P) + 1;
  if (rows > 0)
    k_smag<R, false><<<dim3((P.glo_ni + 31) / 32, (rows + 3) / 4, (P.nk + kSmagK - 1) / kSmagK), dim3(32, 4), 0, s>>>(
        P, nullptr);
}
template <typename R>
void launch_ssh(const DevT<R> &P, cudaStream_t s) { k_ssh<R, false><<<g3(P.ni, wrows(P), 1), kBlock3, sm3(P.nk, 1), s>>>(P, nullptr); }
template <typename R>
void launch_ts(const DevT<R> &P, cudaStream_t s) {
  if constexpr (std::is_same<R, double>::value) {
    k_ts_col<false><<<dim3((P.glo_ni + kColX - 1) / kColX, (wrows(P) + kColY - 1) / kColY), dim3(kColX, kColY), 0, s>>>(P, nullptr);
    k_ts_acc<false><<<g3(P.glo_ni, wrows(P), 1), kBlock3, 0, s>>>(P, nullptr);
  } else {
    k_ts<R, false><<<g3(P.glo_ni, wrows(P), 1), kBlock3, sm3(P.nk, 4), s>>>(P, nullptr);
  }
}
template <typename R>
void launch_den_prho(const DevT<R> &P, cudaStream_t s) { k_den_prho<R, false><<<g3(P.ni, wrows(P), 1), kBlock3, 0, s>>>(P, nullptr); }


#define PCOM_INST(R)                                                   \
  template void launch_alpha_tobot<R>(const DevT<R> &, cudaStream_t); \
  template void launch_pgra2d<R>(const DevT<R> &, cudaStream_t);      \
  template void launch_uv2d<R>(const DevT<R> &, int, cudaStream_t);   \
  template void launch_upwelling<R>(const DevT<R> &, int, cudaStream_t); \
  template void launch_readyc3d<R>(const DevT<R> &, cudaStream_t);    \
  template void launch_clin<R>(const DevT<R> &, cudaStream_t);        \
  template void launch_smag<R>(const DevT<R> &, cudaStream_t);        \
  template void launch_ssh<R>(const DevT<R> &, cudaStream_t);         \
  template void launch_ts<R>(const DevT<R> &, cudaStream_t);          \
  template void launch_den_prho<R>(const DevT<R> &, cudaStream_t);
PCOM_INST(double)
PCOM_INST(float)
#undef PCOM_INST

void launch_batch(int kernel, const Dev *dPs, const BatchShape &b, int arg, cudaStream_t s) {
  Dev none{};  // the by-value parameter is unused in the batched form
  const int n = b.n;
  switch (kernel) {
  case BK_ALPHA_TOBOT: k_alpha_tobot<double, true><<<g3(b.ni, b.nj, n), kBlock3, sm3(b.nk, 1), s>>>(none, dPs); break;
  case BK_PGRA2D: k_pgra2d<double, true><<<g3(b.glo_ni, b.nj, n), kBlock3, sm3(b.nk, 4), s>>>(none, dPs); break;
  case BK_UV2D: k_uv2d<double, true><<<dim3((b.glo_ni + 31) / 32, (b.nj + 3) / 4, n), dim3(32, 4), 0, s>>>(none, dPs, arg); break;
  case BK_UPWELLING: {
    constexpr int UX = upw_cols<double>();
    k_upwelling<double, true><<<dim3((b.glo_ni + UX - 1) / UX, b.nj, n), dim3(UX, TB_K, 1),
                                (size_t)3 * b.nk * UX * sizeof(double), s>>>(none, dPs, arg);
    break;
  }
  case BK_READYC3D:
    k_readyc_col<true><<<dim3((b.glo_ni + kRcX - 1) / kRcX, (b.nj + kRcY - 1) / kRcY, n), dim3(kRcX, kRcY), 0, s>>>(none, dPs);
    break;
  case BK_CLIN: {
    static const cudaError_t attr = cudaFuncSetAttribute(k_clin<double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                         (int)clin_smem(PCOM_MAXK));
    (void)attr;
    k_clin<double, true><<<g3(b.glo_ni, b.nj, n), kBlock3, clin_smem(b.nk), s>>>(none, dPs);
    break;
  }
  case BK_SMAG: k_smag<double, true><<<dim3((b.glo_ni + 31) / 32, (b.nj + 3) / 4, n), dim3(32, 4), 0, s>>>(none, dPs); break;
  case BK_SSH: k_ssh<double, true><<<g3(b.ni, b.nj, n), kBlock3, sm3(b.nk, 1), s>>>(none, dPs); break;
  case BK_TS:
    k_ts_col<true><<<dim3((b.glo_ni + kColX - 1) / kColX, (b.nj + kColY - 1) / kColY, n), dim3(kColX, kColY), 0, s>>>(none, dPs);
    k_ts_acc<true><<<g3(b.glo_ni, b.nj, n), kBlock3, 0, s>>>(none, dPs);
    break;
  case BK_DEN_PRHO: k_den_prho<double, true><<<g3(b.ni, b.nj, n), kBlock3, 0, s>>>(none, dPs); break;
  default: break;
  }
}
