// pcom_gpu.cu -- implementation of the C ABI in include/pcom_gpu.h.
//
// A handle owns the device mirrors of one domain (all FP64, Fortran order,
// padded ni x nj planes), one CUDA stream and the step orchestration:
//   den_alpha+int_tobot, int_pgra, int_readyc, int_trop, int_clin+smag,
//   int_ssh, int_ts  (main.f90:205-223)
// Ring buffers replace the reference's array copies: the AB3 history
// (mod_int.f90:115-118) rotates three buffers per component, and int_ts
// writes the new T/S into a free buffer that then becomes both tc and tp
// (mod_int.f90:496-497).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/pcom_gpu.h"
#include "pcom_dev.cuh"
#include "pcom_kernels.h"

namespace {

thread_local std::string g_last_error;

int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

#define CK(call)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) return fail(PCOM_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

// ------------------------------------------------------------------ constants
// Default-REAL literals of mod_con.f90:16-36, mod_den.f90:91-115 and
// mod_int.f90:314-316 as the reference's compiler stores them.
struct LitMode {
  bool r8;
  double operator()(float f, double d) const { return r8 ? d : (double)f; }
};
#define LIT(x) lit((float)(x##f), (double)(x))

void make_consts(bool r8, DevConsts &c) {
  LitMode lit{r8};
  c.rho0 = LIT(1029.0);
  c.a0 = 1.0 / c.rho0;
  c.g = LIT(9.8);
  c.a = LIT(6370e3);
  c.pi = LIT(3.141592653589793);
  c.gamma_t = c.g * LIT(40.0) / LIT(3901.0);
  c.gamma_s = r8 ? 1.0 / (double)(120 * 24 * 60 * 60) : (double)(1.0f / (float)(120 * 24 * 60 * 60));
  c.gamma_b = LIT(0.2);
  c.deltat = LIT(1.0e-2);
  c.deltas = LIT(1.0e-3);
  c.cdbot = LIT(2.6);
  c.tice = LIT(-1.5);
  c.smag_c = LIT(0.56);
  c.ah_c = LIT(1.0e3);
  c.c_tc = r8 ? 23.0 / 12 : (double)(23.0f / 12);
  c.c_tp = r8 ? -16.0 / 12 : (double)(-16.0f / 12);
  c.c_tpp = r8 ? 5.0 / 12 : (double)(5.0f / 12);
  const double e[42] = {
      LIT(999.842594), LIT(6.793952e-2), LIT(9.095290e-3), LIT(1.001685e-4), LIT(1.120083e-6), LIT(6.536336e-9),
      LIT(8.24493e-1), LIT(4.0899e-3),   LIT(7.6438e-5),   LIT(8.2467e-7),   LIT(5.3875e-9),
      LIT(5.72466e-3), LIT(1.0227e-4),   LIT(1.6546e-6),
      LIT(4.8314e-4),
      LIT(1.965933e4), LIT(1.444304e2),  LIT(1.706103),    LIT(9.648704e-3), LIT(4.190253e-5),
      LIT(5.284855e1), LIT(3.101089e-1), LIT(6.283263e-3), LIT(5.084188e-5),
      LIT(3.886640e-1), LIT(9.085835e-3), LIT(4.619924e-4),
      LIT(3.186519),   LIT(2.212276e-2), LIT(2.984642e-4), LIT(1.956415e-6),
      LIT(6.704388e-3), LIT(1.847318e-4), LIT(2.059331e-7),
      LIT(1.480266e-4),
      LIT(2.102898e-4), LIT(1.202016e-5), LIT(1.394680e-7),
      LIT(2.040237e-6), LIT(6.128773e-8), LIT(6.207323e-10),
      LIT(1e-5)};
  memcpy(c.eos, e, sizeof e);
}

// ------------------------------------------------------------------- kernels
template <typename T>
__global__ void k_nonfinite(const T *f, const int *lev, int nk, long long n2, int planes,
                            unsigned long long *count) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long n = n2 * planes;
  unsigned long long c = 0;
  for (; p < n; p += (long long)gridDim.x * blockDim.x) {
    const long long q2 = p % n2;
    const int k = (int)(p / n2) + 1;
    const bool wet = planes == 1 ? lev[q2] >= 1 : lev[q2] >= k;
    if (wet && !isfinite(f[p])) ++c;
  }
  if (c) atomicAdd(count, c);
}

// mixed path: conversions between the FP64 host layout and FP32 device
// storage; kind 1 subtracts / adds a per-level profile (alpha, adp anomalies)
// (kind 1: alpha, a per-level profile; kind 2: adp, the profile's int_tobot
// over each column's wet levels, which needs lev)
struct Profile {
  double alpha_r[PCOM_MAXK], dpr2[PCOM_MAXK], cum[PCOM_MAXK + 1];
  const int *lev;
};
__device__ double profile_at(const Profile &pr, long long p, long long n2, int per, int kind) {
  const long long pt = p / per;
  const int k = (int)(pt / n2) + 1;
  if (kind == 1) return pr.alpha_r[k];
  if (kind == 2) return adp_ref(pr.alpha_r, pr.dpr2, pr.cum, k, pr.lev[pt % n2]);
  return 0.0;
}
__global__ void k_to_f32(const double *src, float *dst, long long n, long long n2, int per, int kind,
                         const __grid_constant__ Profile pr) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    double v = src[p];
    if (kind) v -= profile_at(pr, p, n2, per, kind);
    dst[p] = (float)v;
  }
}
__global__ void k_to_f64(const float *src, double *dst, long long n, long long n2, int per, int kind,
                         const __grid_constant__ Profile pr) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    double v = (double)src[p];
    if (kind) v += profile_at(pr, p, n2, per, kind);
    dst[p] = v;
  }
}

// reference profile of the mixed path: alpha_r(k) = 1/rho(T_r, S_r, pr(k))
__global__ void k_ref_profile(DevConsts c, const double *tr, const double *sr, const double *pr, int nk, double *out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int k = 1; k <= nk; ++k) out[k] = 1.0 / den_rho(c, tr[k], sr[k], pr[k]);
}

// global sums: wet volume, and the volume integrals of T and S over T cells
// of interior columns and rows; fixed-order reduction (deterministic)
template <typename R>
__global__ void k_sums(const __grid_constant__ DevT<R> P, double *part) {
  __shared__ double sh[3][256];
  double v = 0.0, t = 0.0, s = 0.0;
  const long long nint = (long long)P.glo_ni * (P.nj - 2) * P.nk;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < nint; p += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(p % P.glo_ni);
    const int j = (int)((p / P.glo_ni) % (P.nj - 2)) + 2;
    const int k = (int)(p / ((long long)P.glo_ni * (P.nj - 2))) + 1;
    const long long q2 = (long long)(x + 1) + (long long)P.ni * (j - 1);
    if (P.lev_t[q2] < k) continue;
    const double area = (P.c.a * P.rh[1][q2] * P.dxx[1][q2]) * (P.c.a * P.dxy[1][q2]);
    const double dv = area * P.dz2[k];
    const long long q = q2 + P.n2 * (k - 1);
    v += dv;
    t += (double)P.tc[q] * dv;
    s += (double)P.sc[q] * dv;
  }
  sh[0][threadIdx.x] = v;
  sh[1][threadIdx.x] = t;
  sh[2][threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      for (int c = 0; c < 3; ++c) sh[c][threadIdx.x] += sh[c][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int c = 0; c < 3; ++c) part[3 * blockIdx.x + c] = sh[c][0];
}
__global__ void k_sums_final(const double *part, int nb, double *out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double a[3] = {0.0, 0.0, 0.0};
  for (int b = 0; b < nb; ++b)
    for (int c = 0; c < 3; ++c) a[c] += part[3 * b + c];
  for (int c = 0; c < 3; ++c) out[c] = a[c];
}

// int_bnd (mod_int.f90:649-691): bnd = (frc(m2) - frc(m1)) f + frc(m1)
__global__ void k_int_bnd(const double *frc, double *taux, double *tauy, double *t, double *s, double *pa,
                          long long n2, int m1, int m2, double f) {
  double *dst[5] = {taux, tauy, t, s, pa};
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < 5 * n2; p += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(p / n2);
    const long long r = p % n2;
    const double *F = frc + (long long)q * 12 * n2;
    const double a = F[(long long)(m1 - 1) * n2 + r], b = F[(long long)(m2 - 1) * n2 + r];
    dst[q][r] = (b - a) * f + a;
  }
}


// ---- closure coupling (FP64 handles)
struct Grid2 {
  int ni, glo_ni, glo_nj, nk;
  long long n2;
};
template <typename T>
__device__ __forceinline__ void put_twin(T *f, const Grid2 &g, int i, long long q, T v) {
  f[q] = v;
  if (i == 2) f[q + (g.ni - 2)] = v;
  else if (i == g.ni - 1) f[q - (g.ni - 2)] = v;
}
// block mean over wet fine cells (all cells when none is wet) of nlev planes
// levc (optional): the coarse grid's levels; the value is 0 where the
// coarse point is land (U-grid velocities must vanish there)
__global__ void k_coarsen(const double *f, double *c, const int *levf, const int *levc, Grid2 F, Grid2 Cg, int nlev,
                          int factor, int plane_lev) {
  const long long n = (long long)Cg.glo_ni * Cg.glo_nj * nlev;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    const int I = (int)(p % Cg.glo_ni), J = (int)((p / Cg.glo_ni) % Cg.glo_nj), k = (int)(p / ((long long)Cg.glo_ni * Cg.glo_nj)) + 1;
    const int kl = plane_lev ? k : 1;
    double sw = 0.0, sa = 0.0;
    int nw = 0;
    for (int b = 0; b < factor; ++b)
      for (int a = 0; a < factor; ++a) {
        const long long q2 = (long long)(1 + factor * I + a) + (long long)F.ni * (1 + factor * J + b);
        const double v = f[q2 + F.n2 * (k - 1)];
        sa += v;
        if (levf[q2] >= kl) { sw += v; ++nw; }
      }
    double m = nw ? sw / nw : sa / (factor * factor);
    const int i = I + 2;
    const long long q2c = (long long)(i - 1) + (long long)Cg.ni * (J + 1);
    if (levc && levc[q2c] < kl) m = 0.0;
    put_twin(c, Cg, i, q2c + Cg.n2 * (k - 1), m);
  }
}
struct CnnStatsDev {
  float in_mean[5], in_std[5], out_std[4], out_gain[4], out_clip;
  double alpha_ref[64];
};
__device__ __forceinline__ float clip_y(float y, float c) { return c > 0.f ? fminf(fmaxf(y, -c), c) : y; }
__device__ __forceinline__ uint32_t bf16x2_bits(float lo, float hi) {
  const __nv_bfloat162 b = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t *>(&b);
}
// The network's input at pixel (I, J, level k): grid (ceil(glo_ni / 128),
// glo_nj, nk), one thread per pixel, its 16 BF16 channels written as two
// 16-byte stores (16 separate 2-byte stores touched 32 sectors per warp
// store).  R: the handle's 3-D storage (the mixed path stores alpha as
// alpha - alpha_r(k)).
template <typename R>
__global__ void k_cnn_features(const __grid_constant__ DevT<R> P, __nv_bfloat16 *x, CnnStatsDev st) {
  constexpr bool MIXED = std::is_same<R, float>::value;
  const int I = blockIdx.x * blockDim.x + threadIdx.x, J = blockIdx.y, k = blockIdx.z + 1;
  if (I >= P.glo_ni) return;
  const long long p = ((long long)(k - 1) * P.glo_nj + J) * P.glo_ni + I;
  const long long q2 = (long long)(I + 1) + (long long)P.ni * (J + 1), q = q2 + P.n2 * (k - 1);
  const bool wu = P.lev_u[q2] >= k, wt = P.lev_t[q2] >= k;
  float v[5];
  const double al = MIXED ? (double)P.alpha[q] + P.alpha_r[k] : (double)P.alpha[q];
  v[0] = wu ? (float)(((double)P.uc[q] - st.in_mean[0]) / st.in_std[0]) : 0.f;
  v[1] = wu ? (float)(((double)P.vc[q] - st.in_mean[1]) / st.in_std[1]) : 0.f;
  v[2] = wt ? (float)(((double)P.tc[q] - st.in_mean[2]) / st.in_std[2]) : 0.f;
  v[3] = wt ? (float)(((double)P.sc[q] - st.in_mean[3]) / st.in_std[3]) : 0.f;
  v[4] = wt ? (float)((al - st.alpha_ref[k - 1] - st.in_mean[4]) / st.in_std[4]) : 0.f;
  uint4 *o = reinterpret_cast<uint4 *>(x + p * 16);
  o[0] = make_uint4(bf16x2_bits(v[0], v[1]), bf16x2_bits(v[2], v[3]), bf16x2_bits(v[4], 0.f), 0u);
  o[1] = make_uint4(0u, 0u, 0u, 0u);
}
__global__ void k_cnn_target(const __grid_constant__ Dev Pp, const __grid_constant__ Dev Pt, float *target, float *mask,
                             CnnStatsDev st, double rdt) {
  const long long n = (long long)Pp.glo_ni * Pp.glo_nj * Pp.nk;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    const int I = (int)(p % Pp.glo_ni), J = (int)((p / Pp.glo_ni) % Pp.glo_nj), k = (int)(p / ((long long)Pp.glo_ni * Pp.glo_nj)) + 1;
    const long long q2 = (long long)(I + 1) + (long long)Pp.ni * (J + 1), q = q2 + Pp.n2 * (k - 1);
    const float mu = Pp.lev_u[q2] >= k ? 1.f : 0.f, mt = Pp.lev_t[q2] >= k ? 1.f : 0.f;
    if (target) {  // an output with scale 0 carries no signal: target 0
      const double d[4] = {Pt.uc[q] - Pp.uc[q], Pt.vc[q] - Pp.vc[q], Pt.tc[q] - Pp.tc[q], Pt.sc[q] - Pp.sc[q]};
      const float m[4] = {mu, mu, mt, mt};
      for (int c = 0; c < 4; ++c)
        target[p * 4 + c] = st.out_std[c] > 0.f ? m[c] * (float)(d[c] * rdt / st.out_std[c]) : 0.f;
    }
    if (mask) {
      mask[p * 4 + 0] = mu;
      mask[p * 4 + 1] = mu;
      mask[p * 4 + 2] = mt;
      mask[p * 4 + 3] = mt;
    }
  }
}
// the network's tendency applied at pixel (I, J, level k), the same grid
template <typename R>
__global__ void k_cnn_apply(const __grid_constant__ DevT<R> P, const float *y, CnnStatsDev st, double dt, int tp_distinct) {
  const Grid2 G{P.ni, P.glo_ni, P.glo_nj, P.nk, P.n2};
  const int I = blockIdx.x * blockDim.x + threadIdx.x, J = blockIdx.y, k = blockIdx.z + 1;
  if (I >= P.glo_ni) return;
  const long long p = ((long long)(k - 1) * P.glo_nj + J) * P.glo_ni + I;
  const int i = I + 2;
  const long long q2 = (long long)(i - 1) + (long long)P.ni * (J + 1), q = q2 + P.n2 * (k - 1);
  const float4 yv = reinterpret_cast<const float4 *>(y)[p];
  if (P.lev_u[q2] >= k) {
    const double du = dt * st.out_gain[0] * st.out_std[0] * clip_y(yv.x, st.out_clip);
    const double dv = dt * st.out_gain[1] * st.out_std[1] * clip_y(yv.y, st.out_clip);
    put_twin(P.uc, G, i, q, (R)(P.uc[q] + du));
    put_twin(P.vc, G, i, q, (R)(P.vc[q] + dv));
    put_twin(P.up, G, i, q, (R)(P.up[q] + du));
    put_twin(P.vp, G, i, q, (R)(P.vp[q] + dv));
  }
  if (P.lev_t[q2] >= k) {
    const double dT = dt * st.out_gain[2] * st.out_std[2] * clip_y(yv.z, st.out_clip);
    const double dS = dt * st.out_gain[3] * st.out_std[3] * clip_y(yv.w, st.out_clip);
    put_twin(P.tc, G, i, q, (R)(P.tc[q] + dT));
    put_twin(P.sc, G, i, q, (R)(P.sc[q] + dS));
    if (tp_distinct) {
      put_twin(P.tp, G, i, q, (R)(P.tp[q] + dT));
      put_twin(P.sp, G, i, q, (R)(P.sp[q] + dS));
    }
  }
}

struct ProfEntry {
  long long launches = 0;
  double ms = 0.0;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending;
};

}  // namespace

void launch_nonfinite(const double *f, const int *lev, int nk, long long n2, int planes, unsigned long long *count,
                      cudaStream_t s) {
  k_nonfinite<double><<<592, 256, 0, s>>>(f, lev, nk, n2, planes, count);
}

struct pcom_handle {
  pcom_dims dims{};
  int ni = 0, nj = 0, nk = 0, nkp = 0;
  long long n2 = 0, n3 = 0, n3p = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int device = 0;
  Dev D{};
  // mixed path: the 3-D fields live in DM (FP32); D keeps the shared FP64
  // part and serves the barotropic kernel (its am is the FP64 level-1 copy)
  bool mixed = false;
  DevM DM{};
  float *ab_uf[3] = {}, *ab_vf[3] = {}, *t_poolf[3] = {}, *s_poolf[3] = {};
  double *stage = nullptr;     // FP64 staging for host copies of FP32 fields
  bool ref_set = false;        // reference profile of the anomalies fixed
  double *d_sums = nullptr;    // global-sum partials and result
  std::vector<int> lev_t_host;
  std::vector<void *> allocs;
  double *ab_u[3] = {}, *ab_v[3] = {};  // AB3 ring buffers: [ic], [ip], [ipp]
  int ic = 0, ip = 1, ipp = 2;
  double *t_pool[3] = {}, *s_pool[3] = {};
  int itc = 0, itp = 0;  // indices of tc/tp (and sc/sp) in the pools
  double *dxx_h[5] = {}, *dxy_h[5] = {};
  bool static_ok = false;
  int n_ts = 0, n_uv = 0, n_w = 0, n_ch = 0, n_ssh = 0;
  int trop_tx = 24, trop_ty = 18, trop_blocks = 0;
  bool trop_resident = false;
  // domains too large for the resident kernel: the multi-tile kernel over
  // this domain's tile list (its Dev passed by value per launch)
  bool trop_multi = false;
  // mixed handles on the multi-tile path: FP32 coefficients and velocities
  unsigned char *mm_scratch = nullptr;
  MultiMixed mm{};
  int trop_force = 0;  // 0 automatic, 1 resident, 2 multi-tile, 3 generic
  TileRef *d_tiles1 = nullptr;
  int ntiles1 = 0;
  unsigned long long *d_cnt1 = nullptr;
  double *frc_months = nullptr;  // taux, tauy, t, s, pa: [5][12][nj][ni]
  unsigned long long trop_epoch = 0;  // barrier arrivals of the barotropic kernel so far
  // second stream of the full step: phases that share no array with the
  // main stream's concurrent phases run on it, forked and joined by events
  bool overlap = true;
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork[2] = {}, ev_join[2] = {};
  // host transfers of the asynchronous calls: forcing on `copy` into a
  // second set of forcing fields (taux, tauy, bnd_t, bnd_s, bnd_pa) that the
  // next step switches to; state on `copy_out` from device snapshots taken
  // on `stream` (two streams, so an upload never queues behind a download
  // that waits for a step)
  cudaStream_t copy = nullptr, copy_out = nullptr;
  cudaEvent_t ev_frc = nullptr, ev_snap = nullptr, ev_d2h = nullptr, ev_frc_free[2] = {};
  double *frc_buf[2][5] = {};
  int frc_cur = 0, frc_pending = -1;
  std::map<std::string, double *> snap;
  bool prof = false;
  std::map<std::string, ProfEntry> prof_tab;
  long long launches = 0;
  unsigned long long *d_count = nullptr;

  template <class T>
  int alloc(T **p, size_t n) {
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, n * sizeof(T));
    if (e != cudaSuccess) return fail(PCOM_ERR_CUDA, "cudaMalloc(%zu bytes): %s", n * sizeof(T), cudaGetErrorString(e));
    // zeroed on the owning stream and finished before the buffer is handed
    // out: a plain cudaMemset would run on the legacy stream, which
    // non-blocking streams are not ordered after, and synchronous copies on
    // the legacy stream are not ordered after the owning stream either
    cudaMemsetAsync(q, 0, n * sizeof(T), stream);
    cudaStreamSynchronize(stream);
    allocs.push_back(q);
    *p = (T *)q;
    return PCOM_OK;
  }
};

namespace {

// time a launch with events when profiling is on
struct Prof {
  pcom_handle *h;
  const char *name;
  cudaStream_t st;
  cudaEvent_t a = nullptr, b = nullptr;
  Prof(pcom_handle *h_, const char *n, cudaStream_t s = nullptr) : h(h_), name(n), st(s ? s : h_->stream) {
    h->launches++;
    if (h->prof) {
      cudaEventCreate(&a);
      cudaEventCreate(&b);
      cudaEventRecord(a, st);
    }
  }
  ~Prof() {
    if (h->prof) {
      cudaEventRecord(b, st);
      ProfEntry &e = h->prof_tab[name];
      e.launches++;
      e.pending.emplace_back(a, b);
    }
  }
};

int sync_check(pcom_handle *h) {
  CK(cudaStreamSynchronize(h->stream));
  if (h->side) CK(cudaStreamSynchronize(h->side));
  if (h->copy) CK(cudaStreamSynchronize(h->copy));
  if (h->copy_out) CK(cudaStreamSynchronize(h->copy_out));
  CK(cudaGetLastError());
  int err[2] = {0, 0};
  CK(cudaMemcpy(err, h->D.err, sizeof err, cudaMemcpyDeviceToHost));
  if (err[0]) {
    cudaMemsetAsync(h->D.err, 0, sizeof err, h->stream);
    cudaMemsetAsync(h->D.bar, 0, 2 * sizeof(unsigned), h->stream);
    cudaMemsetAsync(h->D.tile_flag, 0, sizeof(unsigned long long), h->stream);
    cudaStreamSynchronize(h->stream);
    h->trop_epoch = 0;
    return fail(PCOM_ERR_TIMEOUT, "a device-side grid barrier gave up waiting (bounded spin)");
  }
  return PCOM_OK;
}

template <typename R>
void bind_ring(pcom_handle *h, DevT<R> &D, R *const *abu, R *const *abv, R *const *tp, R *const *sp) {
  D.auc = abu[h->ic]; D.aup = abu[h->ip]; D.aupp = abu[h->ipp];
  D.avc = abv[h->ic]; D.avp = abv[h->ip]; D.avpp = abv[h->ipp];
  D.tc = tp[h->itc]; D.tp = tp[h->itp];
  D.sc = sp[h->itc]; D.sp = sp[h->itp];
  int fr = 0;
  while (fr == h->itc || fr == h->itp) ++fr;
  D.tn_ = tp[fr];
  D.sn_ = sp[fr];
}
void bind_rotating(pcom_handle *h) {
  if (h->mixed) bind_ring(h, h->DM, h->ab_uf, h->ab_vf, h->t_poolf, h->s_poolf);
  else bind_ring(h, h->D, h->ab_u, h->ab_v, h->t_pool, h->s_pool);
}
// the mixed path's DM shares every FP64 field of D
void sync_common(pcom_handle *h) {
  if (h->mixed) static_cast<DevCommon &>(h->DM) = static_cast<const DevCommon &>(h->D);
}

// a forcing staged by pcom_gpu_set_forcing_async becomes the step's forcing:
// the handle's stream waits for its upload, the set in use so far is free
// once the work enqueued until now has run, and D points at the staged set
int apply_staged_forcing(pcom_handle *h) {
  if (h->frc_pending < 0) return PCOM_OK;
  CK(cudaStreamWaitEvent(h->stream, h->ev_frc, 0));
  CK(cudaEventRecord(h->ev_frc_free[h->frc_cur], h->stream));
  h->frc_cur = h->frc_pending;
  h->frc_pending = -1;
  double *const *b = h->frc_buf[h->frc_cur];
  h->D.taux = b[0]; h->D.tauy = b[1]; h->D.bnd_t = b[2]; h->D.bnd_s = b[3]; h->D.bnd_pa = b[4];
  sync_common(h);
  return PCOM_OK;
}

int pick_trop_config(pcom_handle *h) {
  // resident kernel: one tile per CTA, one region point per thread; pick the
  // tiling with the fewest tiles (fewest CTAs at the grid barrier)
  h->trop_resident = false;
  h->trop_multi = false;
  if (h->D.separable && (h->trop_force == 0 || h->trop_force == 1)) {
    int best_n = 1 << 30, bx = 0, by = 0;
    const int mb = trop_fast_max_blocks(24, 18);
    for (int ty = 6; ty <= 40; ++ty)
      for (int tx = 6; tx <= 60; ++tx) {
        if (!trop_res_fits(tx, ty)) continue;
        const int nt = ((h->dims.glo_ni + tx - 1) / tx) * ((h->nj + ty - 1) / ty);
        if (nt > mb) continue;
        if (nt < best_n || (nt == best_n && (tx + 4) * (ty + 4) < (bx + 4) * (by + 4))) { best_n = nt; bx = tx; by = ty; }
      }
    if (bx > 0 && trop_fast_max_blocks(bx, by) >= best_n) {
      h->trop_resident = true;
      h->trop_tx = bx;
      h->trop_ty = by;
      h->trop_blocks = best_n;
      return PCOM_OK;
    }
  }
  // too large to be resident: the multi-tile kernel (several tiles per CTA,
  // coefficients from L2) over this domain's tiles
  if (h->trop_force == 1) return fail(PCOM_ERR_ARG, "the domain does not fit the resident barotropic kernel");
  if (h->D.separable && (h->trop_force == 0 || h->trop_force == 2)) {
    const int tx = 32, ty = 10;
    const int mb = trop_batch_max_blocks(tx, ty);
    if (mb > 0) {
      std::vector<TileRef> t;
      const int G = h->dims.glo_ni, nj = h->nj;
      for (int j0 = 1; j0 <= nj; j0 += ty)
        for (int r0 = 0; r0 < G; r0 += tx) t.push_back({0, r0, j0, std::min(tx, G - r0), std::min(ty, nj - j0 + 1)});
      if (!h->d_cnt1) {
        int rc = h->alloc(&h->d_cnt1, 1);
        if (rc) return rc;
      }
      int rc = h->alloc(&h->d_tiles1, t.size());
      if (rc) return rc;
      CK(cudaMemcpy(h->d_tiles1, t.data(), t.size() * sizeof(TileRef), cudaMemcpyHostToDevice));
      h->ntiles1 = (int)t.size();
      h->trop_multi = true;
      h->trop_tx = tx;
      h->trop_ty = ty;
      h->trop_blocks = std::min(h->ntiles1, mb);
      if (h->mixed) {
        const int mmb = trop_multi_mixed_max_blocks(tx, ty);
        if (mmb <= 0) return fail(PCOM_ERR_CUDA, "the mixed multi-tile barotropic kernel cannot be launched");
        if (!h->mm_scratch) {
          rc = h->alloc(&h->mm_scratch, trop_multi_mixed_scratch_bytes(h->n2));
          if (rc) return rc;
          trop_multi_mixed_bind(h->mm, h->mm_scratch, h->n2);
        }
        h->trop_blocks = std::min(h->ntiles1, mmb);
      }
      return PCOM_OK;
    }
  }
  // largest co-resident grid for the candidate tiles; prefer a tiling with at
  // most one tile per CTA (the whole subcycle then stays one wave)
  static const int cand[][2] = {{24, 18}, {32, 16}, {32, 24}, {32, 32}, {48, 32}, {64, 32}};
  for (auto &c : cand) {
    const int tx = c[0], ty = c[1];
    const int nt = ((h->dims.glo_ni + tx - 1) / tx) * ((h->nj + ty - 1) / ty);
    const int mb = trop_max_blocks(tx, ty);
    if (mb <= 0) continue;
    h->trop_tx = tx;
    h->trop_ty = ty;
    h->trop_blocks = nt < mb ? nt : mb;
    if (nt <= mb) return PCOM_OK;
  }
  if (h->trop_blocks <= 0) return fail(PCOM_ERR_CUDA, "no launchable configuration for the barotropic kernel");
  return PCOM_OK;
}

// ---- the pieces of the step (FP64 handle: D; mixed handle: DM)
#define ON_DEV(call_on) \
  do {                  \
    if (h->mixed) {     \
      auto &X = h->DM;  \
      call_on;          \
    } else {            \
      auto &X = h->D;   \
      call_on;          \
    }                   \
  } while (0)
int do_den_alpha(pcom_handle *h) {
  Prof p(h, "den_alpha+int_tobot");
  ON_DEV(launch_alpha_tobot(X, h->stream));
  return PCOM_OK;
}
int do_pgra(pcom_handle *h) {
  Prof p(h, "int_pgra");
  ON_DEV(launch_pgra2d(X, h->stream));
  return PCOM_OK;
}
// int_readyc's 2-D prep and upwelling (read bnd_pa, chc, chp, uc, vc, wm;
// write pax, pay, sch_r, sch_w, rsch, rsch2, rchc, wm)
int do_readyc_2d(pcom_handle *h, cudaStream_t s) {
  {
    Prof p(h, "readyc_2d", s);
    ON_DEV(launch_uv2d(X, 0, s));
  }
  {
    Prof p(h, "upwelling", s);
    ON_DEV(launch_upwelling(X, 0, s));
  }
  return PCOM_OK;
}
int do_readyc_3d(pcom_handle *h, int64_t iter) {
  // AB3 history: aupp <- aup <- auc (mod_int.f90:115-118) by rotation
  int old_pp = h->ipp;
  h->ipp = h->ip;
  h->ip = h->ic;
  h->ic = old_pp;
  bind_rotating(h);
  const bool fresh = h->dims.rst != 1;
  h->D.ab3_mode = h->DM.ab3_mode = (fresh && iter == 1) ? 1 : 0;
  if (fresh && iter == 2) {
    // aupp = aup (mod_int.f90:128-130)
    if (h->mixed) {
      CK(cudaMemcpyAsync(h->DM.aupp, h->DM.aup, h->n3 * sizeof(float), cudaMemcpyDeviceToDevice, h->stream));
      CK(cudaMemcpyAsync(h->DM.avpp, h->DM.avp, h->n3 * sizeof(float), cudaMemcpyDeviceToDevice, h->stream));
    } else {
      CK(cudaMemcpyAsync(h->D.aupp, h->D.aup, h->n3 * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
      CK(cudaMemcpyAsync(h->D.avpp, h->D.avp, h->n3 * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    }
  }
  {
    Prof p(h, "readyc_3d");
    ON_DEV(launch_readyc3d(X, h->stream));
  }
  h->D.ab3_mode = h->DM.ab3_mode = 0;
  return PCOM_OK;
}
int do_trop(pcom_handle *h) {
  if (h->trop_blocks <= 0) {
    int rc = pick_trop_config(h);
    if (rc) return rc;
  }
  Prof p(h, "int_trop");
  cudaError_t e;
  if (h->trop_resident) {
    // the kernel's barrier counter is monotone: pass the arrivals so far
    if (h->mixed && trop_mixed_max_blocks(h->trop_tx, h->trop_ty) >= h->trop_blocks)
      e = launch_trop_mixed(h->D, h->trop_tx, h->trop_ty, h->trop_epoch, h->stream);
    else
      e = launch_trop_fast(h->D, h->trop_tx, h->trop_ty, h->trop_epoch, h->stream);
    h->trop_epoch += (unsigned long long)h->D.nstep * (unsigned long long)h->trop_blocks;
  } else if (h->trop_multi && h->mixed) {
    e = launch_trop_multi_mixed(h->D, h->mm, h->d_tiles1, h->ntiles1, h->trop_tx, h->trop_ty, h->trop_blocks,
                                h->d_cnt1, h->D.err, h->stream);
  } else if (h->trop_multi) {
    e = launch_trop_multi(h->D, h->d_tiles1, h->ntiles1, h->trop_tx, h->trop_ty, h->trop_blocks, h->d_cnt1, h->D.err,
                          h->stream);
  } else {
    e = launch_trop(h->D, h->trop_tx, h->trop_ty, h->trop_blocks, h->stream);
  }
  if (e != cudaSuccess) return fail(PCOM_ERR_CUDA, "barotropic kernel launch: %s", cudaGetErrorString(e));
  h->n_ch++;
  return PCOM_OK;
}
// with_ts2d: the 2-D prep of int_ts (its sch, reciprocals of mch, mch2) in
// the same launch as int_clin's (both read only int_trop's outputs)
int do_clin_uv(pcom_handle *h, bool with_ts2d = false) {
  {
    Prof p(h, "clin_2d");
    ON_DEV(launch_uv2d(X, with_ts2d ? 3 : 2, h->stream));
  }
  {
    Prof p(h, "int_clin");
    ON_DEV(launch_clin(X, h->stream));
  }
  h->n_uv++;
  return PCOM_OK;
}
// Smagorinsky viscosity (reads uu, vv, dxs, tn3; writes am, am1)
int do_smag(pcom_handle *h, cudaStream_t s) {
  Prof p(h, "smag", s);
  ON_DEV(launch_smag(X, s));
  return PCOM_OK;
}
int do_ssh(pcom_handle *h) {
  Prof p(h, "int_ssh");
  ON_DEV(launch_ssh(X, h->stream));
  h->n_ssh++;
  return PCOM_OK;
}
int do_ts(pcom_handle *h, bool with_2d = true) {
  if (with_2d) {
    Prof p(h, "ts_2d");
    ON_DEV(launch_uv2d(X, 1, h->stream));
  }
  {
    Prof p(h, "upwelling+acw");
    ON_DEV(launch_upwelling(X, 1, h->stream));
  }
  h->n_w++;
  {
    Prof p(h, "int_ts");
    ON_DEV(launch_ts(X, h->stream));
    if (!h->mixed) h->launches++;  // FP64: the column kernel and the accumulation kernel
  }
  // tc = tp = the buffer just written (mod_int.f90:496-497)
  int fr = 0;
  while (fr == h->itc || fr == h->itp) ++fr;
  h->itc = h->itp = fr;
  bind_rotating(h);
  h->n_ts++;
  return PCOM_OK;
}

int run_phase(pcom_handle *h, int phase, int64_t iter) {
  switch (phase) {
  case 0: return do_den_alpha(h);
  case 1: return do_pgra(h);
  case 2: {
    int rc = do_readyc_2d(h, h->stream);
    return rc ? rc : do_readyc_3d(h, iter);
  }
  case 3: return do_trop(h);
  case 4: {
    int rc = do_clin_uv(h);
    return rc ? rc : do_smag(h, h->stream);
  }
  case 5: return do_ssh(h);
  case 6: return do_ts(h);
  default: return fail(PCOM_ERR_ARG, "unknown phase %d", phase);
  }
}

int enqueue_step(pcom_handle *h, int64_t iter) {
  if (!h) return fail(PCOM_ERR_ARG, "null handle");
  if (!h->static_ok) return fail(PCOM_ERR_STATE, "step before pcom_gpu_upload_static");
  if (iter < 1) return fail(PCOM_ERR_ARG, "tctr_i must be >= 1");
  if (int rc = apply_staged_forcing(h)) return rc;
  if (!h->overlap) {
    for (int ph = 0; ph <= 6; ++ph) {
      int rc = run_phase(h, ph, iter);
      if (rc) return rc;
    }
    CK(cudaGetLastError());
    return PCOM_OK;
  }
  // The same launches in the same per-stream order, with two pairs of
  // phases that touch no common array run concurrently on the side stream:
  //  - int_readyc's 2-D prep and upwelling beside den_alpha/int_tobot
  //    (read tc, sc, chc, alpha; write alpha, adp) and int_pgra (reads
  //    adp, alpha; writes bphi, bgraphi); joined before int_readyc's 3-D
  //    part, which reads both sides' results;
  //  - smag (reads uu, vv; writes am, used by the next step's int_readyc
  //    and int_trop only) beside int_ssh and int_ts; joined at the end of
  //    the step.
  int rc;
  CK(cudaEventRecord(h->ev_fork[0], h->stream));
  CK(cudaStreamWaitEvent(h->side, h->ev_fork[0], 0));
  if ((rc = do_readyc_2d(h, h->side))) return rc;
  CK(cudaEventRecord(h->ev_join[0], h->side));
  if ((rc = do_den_alpha(h))) return rc;
  if ((rc = do_pgra(h))) return rc;
  CK(cudaStreamWaitEvent(h->stream, h->ev_join[0], 0));
  if ((rc = do_readyc_3d(h, iter))) return rc;
  if ((rc = do_trop(h))) return rc;
  if ((rc = do_clin_uv(h, true))) return rc;
  CK(cudaEventRecord(h->ev_fork[1], h->stream));
  CK(cudaStreamWaitEvent(h->side, h->ev_fork[1], 0));
  if ((rc = do_smag(h, h->side))) return rc;
  CK(cudaEventRecord(h->ev_join[1], h->side));
  if ((rc = do_ssh(h))) return rc;
  if ((rc = do_ts(h, false))) return rc;
  CK(cudaStreamWaitEvent(h->stream, h->ev_join[1], 0));
  CK(cudaGetLastError());
  return PCOM_OK;
}

int copy_in(pcom_handle *h, double *dst, const double *src, long long n) {
  if (!src) return PCOM_OK;
  CK(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  return PCOM_OK;
}
int copy_out(pcom_handle *h, double *dst, const double *src, long long n) {
  if (!dst) return PCOM_OK;
  CK(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  return PCOM_OK;
}

// the 3-D fields of one storage type
template <typename R>
int alloc_3d(pcom_handle *h, DevT<R> &X, R **abu, R **abv, R **tpool, R **spool) {
  const long long n3 = h->n3, n3p = h->n3p;
  int rc = 0;
  auto A = [&](R **p, long long n) { if (!rc) rc = h->alloc(p, (size_t)n); };
  R *p = nullptr;
  A(&p, n3p); X.km = p; A(&p, n3p); X.kh = p;
  for (int q = 0; q < 3; ++q) { A(&tpool[q], n3); A(&spool[q], n3); A(&abu[q], n3); A(&abv[q], n3); }
  A(&X.uc, n3); A(&X.vc, n3); A(&X.up, n3); A(&X.vp, n3);
  A(&X.am, n3); A(&X.alpha, n3); A(&X.adp, n3); A(&X.wm, n3p);
  {
    typename Vec2<R>::type *pr = nullptr;
    if (!rc) rc = h->alloc(&pr, (size_t)n3);
    X.prho = pr;
  }
  A(&X.fx, n3); A(&X.fy, n3); A(&X.uu, n3); A(&X.vv, n3);
  A(&X.act, n3); A(&X.acs, n3); A(&X.acr, n3); A(&X.acu, n3); A(&X.acv, n3); A(&X.acw, n3);
  return rc;
}

// host FP64 array -> FP32 device array through the staging buffer
Profile profile_of(const DevCommon &D) {
  Profile pr{};
  memcpy(pr.alpha_r, D.alpha_r, sizeof pr.alpha_r);
  memcpy(pr.dpr2, D.dpr2, sizeof pr.dpr2);
  memcpy(pr.cum, D.adp_cum, sizeof pr.cum);
  pr.lev = D.lev_t;
  return pr;
}
int put_f32(pcom_handle *h, float *dst, const double *src, long long n, int kind, int per = 1) {
  CK(cudaMemcpyAsync(h->stage, src, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  const Profile pr = profile_of(h->D);
  k_to_f32<<<592, 256, 0, h->stream>>>(h->stage, dst, n, h->n2, per, kind, pr);
  CK(cudaGetLastError());
  return PCOM_OK;
}
// FP32 device array -> host FP64 array through the staging buffer
int get_f32(pcom_handle *h, double *dst, const float *src, long long n, int kind, int per = 1) {
  const Profile pr = profile_of(h->D);
  k_to_f64<<<592, 256, 0, h->stream>>>(src, h->stage, n, h->n2, per, kind, pr);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(dst, h->stage, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  return PCOM_OK;
}

// a named device array: FP64, or FP32 (mixed path) with its profile kind
struct Named {
  const double *p;
  long long n;
  const float *pf = nullptr;  // FP32 storage (then p is null)
  int kind = 0;               // 1: alpha anomaly, 2: adp anomaly
  int per = 1;                // values per point (prho: 2)
};

Named lookup(pcom_handle *h, const std::string &s) {
  Dev &D = h->D;
  const long long n2 = h->n2, n3 = h->n3, n3p = h->n3p;
  static const char *b4[4] = {"xn", "xs", "ye", "yw"};
  for (int q = 0; q < 4; ++q) {
    if (s == std::string("bphi_") + b4[q]) return {D.bphi[q], n2};
    if (s == std::string("bgraphi_") + b4[q]) return {D.bgra[q], n2};
  }
  const std::map<std::string, Named> m2 = {
      {"ubc", {D.ubc, n2}},   {"vbc", {D.vbc, n2}},     {"ubp", {D.ubp, n2}},   {"vbp", {D.vbp, n2}},
      {"chc", {D.chc, n2}},   {"chp", {D.chp, n2}},     {"mch", {D.mch, n2}},   {"mch2", {D.mch2, n2}},
      {"pax", {D.pax, n2}},   {"pay", {D.pay, n2}},     {"ut", {D.ut, n2}},     {"vt", {D.vt, n2}},
      {"acch", {D.acch, n2}}, {"acssh", {D.acssh, n2}}, {"cor", {D.cor, n2}},   {"cv1", {D.cv1, n2}},
      {"cv2", {D.cv2, n2}},   {"graphihx", {D.graphihx, n2}}, {"graphihy", {D.graphihy, n2}},
      {"sch_r", {D.sch_r, n2}}, {"sch_w", {D.sch_w, n2}}, {"bnd_taux", {D.taux, n2}}, {"bnd_tauy", {D.tauy, n2}},
      {"bnd_t", {D.bnd_t, n2}}, {"bnd_s", {D.bnd_s, n2}}, {"bnd_pa", {D.bnd_pa, n2}}, {"am1", {D.am1, n2}}};
  auto it2 = m2.find(s);
  if (it2 != m2.end()) return it2->second;
  // 3-D fields: FP64, or FP32 on the mixed path
  struct E {
    const void *p;
    long long n;
    int kind, per;
  };
  auto table = [&](const auto &X) {
    return std::map<std::string, E>{
        {"tc", {X.tc, n3, 0, 1}},     {"sc", {X.sc, n3, 0, 1}},     {"tp", {X.tp, n3, 0, 1}},
        {"sp", {X.sp, n3, 0, 1}},     {"uc", {X.uc, n3, 0, 1}},     {"vc", {X.vc, n3, 0, 1}},
        {"up", {X.up, n3, 0, 1}},     {"vp", {X.vp, n3, 0, 1}},     {"auc", {X.auc, n3, 0, 1}},
        {"aup", {X.aup, n3, 0, 1}},   {"aupp", {X.aupp, n3, 0, 1}}, {"avc", {X.avc, n3, 0, 1}},
        {"avp", {X.avp, n3, 0, 1}},   {"avpp", {X.avpp, n3, 0, 1}}, {"am", {X.am, n3, 0, 1}},
        {"alpha", {X.alpha, n3, 1, 1}}, {"adp", {X.adp, n3, 2, 1}}, {"wm", {X.wm, n3p, 0, 1}},
        {"prho", {X.prho, 2 * n3, 0, 2}}, {"fx", {X.fx, n3, 0, 1}}, {"fy", {X.fy, n3, 0, 1}},
        {"act", {X.act, n3, 0, 1}},   {"acs", {X.acs, n3, 0, 1}},   {"acr", {X.acr, n3, 0, 1}},
        {"acu", {X.acu, n3, 0, 1}},   {"acv", {X.acv, n3, 0, 1}},   {"acw", {X.acw, n3, 0, 1}},
        {"km", {X.km, n3p, 0, 1}},    {"kh", {X.kh, n3p, 0, 1}},    {"uu", {X.uu, n3, 0, 1}},
        {"vv", {X.vv, n3, 0, 1}}};
  };
  if (h->mixed) {
    auto m3 = table(h->DM);
    auto it = m3.find(s);
    if (it == m3.end()) return {nullptr, 0};
    Named r{nullptr, it->second.n};
    r.pf = (const float *)it->second.p;
    r.kind = it->second.kind;
    r.per = it->second.per;
    return r;
  }
  auto m3 = table(D);
  auto it = m3.find(s);
  if (it == m3.end()) return {nullptr, 0};
  return {(const double *)it->second.p, it->second.n};
}

// copy a named array to the host as FP64
int fetch(pcom_handle *h, const char *name, double *dst) {
  if (!dst) return PCOM_OK;
  Named f = lookup(h, name);
  if (f.p) return copy_out(h, dst, f.p, f.n);
  if (!f.pf) return fail(PCOM_ERR_ARG, "unknown field '%s'", name);
  return get_f32(h, dst, f.pf, f.n, f.kind, f.per);
}

}  // namespace

namespace {

// mixed path: fix the reference profile of the alpha/adp anomalies from the
// level means of T and S over wet points, and re-express stored anomalies
int set_reference_profile(pcom_handle *h, const double *tc, const double *sc) {
  const int nk = h->nk;
  const long long n2 = h->n2;
  std::vector<double> tr(PCOM_MAXK, 0.0), sr(PCOM_MAXK, 0.0), pr(PCOM_MAXK, 0.0), al(PCOM_MAXK, 0.0);
  for (int k = 1; k <= nk; ++k) {
    double st = 0.0, ss = 0.0;
    long long c = 0;
    for (long long q = 0; q < n2; ++q) {
      const bool wet = h->lev_t_host.empty() ? true : h->lev_t_host[q] >= k;
      if (!wet) continue;
      st += tc[q + n2 * (k - 1)];
      ss += sc[q + n2 * (k - 1)];
      ++c;
    }
    tr[k] = c ? st / c : (k > 1 ? tr[k - 1] : 10.0);
    sr[k] = c ? ss / c : (k > 1 ? sr[k - 1] : 35.0);
    pr[k] = h->D.pr2[k];
  }
  double *d = h->stage;
  CK(cudaMemcpyAsync(d, tr.data(), PCOM_MAXK * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(d + PCOM_MAXK, sr.data(), PCOM_MAXK * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(d + 2 * PCOM_MAXK, pr.data(), PCOM_MAXK * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  k_ref_profile<<<1, 32, 0, h->stream>>>(h->D.c, d, d + PCOM_MAXK, d + 2 * PCOM_MAXK, nk, d + 3 * PCOM_MAXK);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(al.data(), d + 3 * PCOM_MAXK, PCOM_MAXK * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  // stored anomalies were relative to the old profile: re-express them
  Dev &D = h->D;
  const Profile old_pr = profile_of(D);
  for (int k = 1; k <= nk; ++k) D.alpha_r[k] = al[k];
  D.adp_cum[nk + 1] = 0.0;
  for (int k = nk; k >= 1; --k) D.adp_cum[k] = D.adp_cum[k + 1] + D.alpha_r[k] * D.dpr2[k];
  const Profile new_pr = profile_of(D);
  const long long n3 = h->n3;
  for (int f = 1; f <= 2; ++f) {
    float *p = f == 1 ? h->DM.alpha : h->DM.adp;
    k_to_f64<<<592, 256, 0, h->stream>>>(p, h->stage, n3, n2, 1, f, old_pr);
    k_to_f32<<<592, 256, 0, h->stream>>>(h->stage, p, n3, n2, 1, f, new_pr);
    CK(cudaGetLastError());
  }
  sync_common(h);
  h->ref_set = true;
  CK(cudaStreamSynchronize(h->stream));
  return PCOM_OK;
}

int set_state_mixed(pcom_handle *h, const pcom_state *s) {
  const long long n2 = h->n2, n3 = h->n3, n3p = h->n3p;
  Dev &D = h->D;
  DevM &M = h->DM;
  int rc = 0;
  if (!h->ref_set && s->tc && s->sc) rc = set_reference_profile(h, s->tc, s->sc);
  auto in2 = [&](double *dst, const double *src) { if (!rc) rc = copy_in(h, dst, src, n2); };
  auto in3 = [&](float *dst, const double *src, long long n, int kind, const double *, int per) {
    if (!rc && src) rc = put_f32(h, dst, src, n, kind, per);
  };
  in3(M.tc, s->tc, n3, 0, nullptr, 1); in3(M.sc, s->sc, n3, 0, nullptr, 1);
  in3(M.tp, s->tp, n3, 0, nullptr, 1); in3(M.sp, s->sp, n3, 0, nullptr, 1);
  in3(M.uc, s->uc, n3, 0, nullptr, 1); in3(M.vc, s->vc, n3, 0, nullptr, 1);
  in3(M.up, s->up, n3, 0, nullptr, 1); in3(M.vp, s->vp, n3, 0, nullptr, 1);
  in3(M.auc, s->auc, n3, 0, nullptr, 1); in3(M.aup, s->aup, n3, 0, nullptr, 1); in3(M.aupp, s->aupp, n3, 0, nullptr, 1);
  in3(M.avc, s->avc, n3, 0, nullptr, 1); in3(M.avp, s->avp, n3, 0, nullptr, 1); in3(M.avpp, s->avpp, n3, 0, nullptr, 1);
  in2(D.ubc, s->ubc); in2(D.vbc, s->vbc); in2(D.ubp, s->ubp); in2(D.vbp, s->vbp);
  in2(D.chc, s->chc); in2(D.chp, s->chp); in2(D.mch, s->mch); in2(D.mch2, s->mch2);
  in3(M.am, s->am, n3, 0, nullptr, 1);
  if (!rc && s->am) rc = copy_in(h, D.am1, s->am, n2);
  in3((float *)M.prho, s->prho, 2 * n3, 0, nullptr, 2);
  in3(M.alpha, s->alpha, n3, 1, nullptr, 1);
  in3(M.adp, s->adp, n3, 2, nullptr, 1);
  in3(M.wm, s->wm, n3p, 0, nullptr, 1);
  if (rc) return rc;
  CK(cudaStreamSynchronize(h->stream));
  return PCOM_OK;
}

}  // namespace

// =============================================================== C ABI
extern "C" {

int pcom_gpu_last_error(char *buf, int32_t len) {
  if (buf && len > 0) {
    strncpy(buf, g_last_error.c_str(), (size_t)len - 1);
    buf[len - 1] = 0;
  }
  return (int)g_last_error.size();
}

int pcom_gpu_create(const pcom_dims *dims, pcom_handle **out) {
  if (!dims || !out) return fail(PCOM_ERR_ARG, "null argument");
  const pcom_dims &d = *dims;
  if (d.glo_ni < 2 || d.glo_nj < 2 || d.nk < 2) return fail(PCOM_ERR_ARG, "domain too small (%d x %d x %d)", d.glo_ni, d.glo_nj, d.nk);
  if (d.nk > PCOM_MAXK - 1) return fail(PCOM_ERR_ARG, "nk = %d exceeds the supported %d levels", d.nk, PCOM_MAXK - 1);
  if (d.ni != d.glo_ni + 2 || d.nj != d.glo_nj + 2) return fail(PCOM_ERR_ARG, "ni, nj must be glo_ni + 2, glo_nj + 2");
  if (d.dtbt <= 0 || d.dtbc <= 0 || d.dtbc % d.dtbt != 0) return fail(PCOM_ERR_ARG, "dtbc must be a positive multiple of dtbt");
  pcom_handle *h = new pcom_handle();
  h->mixed = (d.flags & PCOM_PREC_MIXED) != 0;
  h->dims = d;
  h->ni = d.ni; h->nj = d.nj; h->nk = d.nk; h->nkp = d.nk + 1;
  h->n2 = (long long)d.ni * d.nj;
  h->n3 = h->n2 * d.nk;
  h->n3p = h->n2 * (d.nk + 1);
  cudaGetDevice(&h->device);
  cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { delete h; return fail(PCOM_ERR_CUDA, "stream: %s", cudaGetErrorString(e)); }
  h->own_stream = true;
  // the side stream and fork/join events of the overlapped step (created
  // here, not in the step, which may be enqueued into a graph capture)
  e = cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking);
  for (int q = 0; q < 2 && e == cudaSuccess; ++q) {
    e = cudaEventCreateWithFlags(&h->ev_fork[q], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_join[q], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_frc_free[q], cudaEventDisableTiming);
  }
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->copy, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->copy_out, cudaStreamNonBlocking);
  for (cudaEvent_t *ev : {&h->ev_frc, &h->ev_snap, &h->ev_d2h})
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
  if (e != cudaSuccess) { pcom_gpu_destroy(h); return fail(PCOM_ERR_CUDA, "side stream: %s", cudaGetErrorString(e)); }
  Dev &D = h->D;
  D.ni = d.ni; D.nj = d.nj; D.nk = d.nk; D.nkp = d.nk + 1; D.nim = d.ni - 1; D.njm = d.nj - 1;
  D.j_lo = 1; D.j_hi = d.nj;
  D.glo_ni = d.glo_ni; D.glo_nj = d.glo_nj;
  D.bt = d.dtbt; D.bc = d.dtbc; D.nstep = d.dtbc / d.dtbt * 2; D.rst = d.rst;
  D.n2 = h->n2; D.n3 = h->n3; D.n3p = h->n3p;
  make_consts((d.flags & PCOM_LIT_R8) != 0, D.c);
  const long long n2 = h->n2, n3 = h->n3, n3p = h->n3p;
  int rc = 0;
  auto A = [&](double **p, long long n) { if (!rc) rc = h->alloc(p, (size_t)n); };
  for (int g = 1; g <= 4; ++g) {
    double *r, *x, *y;
    A(&r, n2); A(&x, n2); A(&y, n2);
    D.rh[g] = r; D.dxx[g] = x; D.dxy[g] = y;
  }
  double *tn3; A(&tn3, n2); D.tn3 = tn3;
  for (int g = 1; g <= 4; ++g) {
    double *x, *y, *r, *rx, *ry, *rr, *ar, *rar;
    A(&x, d.ni); A(&y, d.nj); A(&r, d.nj);
    A(&rx, d.ni); A(&ry, d.nj); A(&rr, d.nj); A(&ar, d.nj); A(&rar, d.nj);
    D.dxx1d[g] = x; D.dxy1d[g] = y; D.rh1d[g] = r;
    D.rdxx1d[g] = rx; D.rdxy1d[g] = ry; D.rrh1d[g] = rr; D.arh1d[g] = ar; D.rarh1d[g] = rar;
  }
  {
    double *x, *y;
    A(&x, d.nj); A(&y, d.nj); D.aarh3 = x; D.raarh3 = y;
    A(&x, d.nj); A(&y, d.nj); D.dys1d = x; D.rdys1d = y;
    A(&x, n2); D.rprh_t = x; A(&x, n2); D.rprh_u = x; A(&x, n2); D.rwc = x; A(&x, n2); D.rwt = x;
    A(&x, n2); D.dxs = x; A(&x, n2); D.rdxs = x;
  }
  A(&D.rsch, n2); A(&D.rsch2, n2); A(&D.rchc, n2); A(&D.rmch, n2); A(&D.rgm2, n2);
  A(&D.schc, n2); A(&D.schu, n2); A(&D.rmch2, n2);
  int *lt = nullptr, *lu = nullptr;
  if (!rc) rc = h->alloc(&lt, (size_t)n2);
  if (!rc) rc = h->alloc(&lu, (size_t)n2);
  D.lev_t = lt; D.lev_u = lu;
  double *p;
  A(&p, n2); D.prh_t = p; A(&p, n2); D.phih_t = p; A(&p, n2); D.prh_u = p;
  A(&p, n2); D.cv1 = p; A(&p, n2); D.cv2 = p; A(&p, n2); D.cor = p;
  A(&p, n2); D.graphihx = p; A(&p, n2); D.graphihy = p;
  A(&p, n2); D.taux = p; A(&p, n2); D.tauy = p; A(&p, n2); D.bnd_t = p; A(&p, n2); D.bnd_s = p; A(&p, n2); D.bnd_pa = p;
  if (!rc) {
    if (h->mixed) rc = alloc_3d(h, h->DM, h->ab_uf, h->ab_vf, h->t_poolf, h->s_poolf);
    else rc = alloc_3d(h, D, h->ab_u, h->ab_v, h->t_pool, h->s_pool);
  }
  A(&D.ubc, n2); A(&D.vbc, n2); A(&D.ubp, n2); A(&D.vbp, n2);
  A(&D.chc, n2); A(&D.chp, n2); A(&D.mch, n2); A(&D.mch2, n2);
  A(&D.pax, n2); A(&D.pay, n2); A(&D.ut, n2); A(&D.vt, n2);
  for (int q = 0; q < 4; ++q) { A(&D.bphi[q], n2); A(&D.bgra[q], n2); }
  A(&D.sch_r, n2); A(&D.sch_w, n2);
  A(&D.acch, n2); A(&D.acssh, n2);
  for (int q = 0; q < 2; ++q) { A(&D.tr_ch[q], n2); A(&D.tr_ub[q], n2); A(&D.tr_vb[q], n2); }
  for (int q = 0; q < 6; ++q) A(&D.tr_acc[q], n2);
  A(&D.am1, n2);
  if (h->mixed) {
    D.am = D.am1;  // the barotropic kernel reads am at level 1 only
    A(&h->stage, std::max(n3p, 2 * n3));
  }
  A(&h->d_sums, 3 * 1024 + 3);
  unsigned *bar = nullptr;
  int *err = nullptr;
  if (!rc) rc = h->alloc(&bar, 4);
  if (!rc) rc = h->alloc(&err, 4);
  if (!rc) rc = h->alloc(&h->d_count, 1);
  {
    unsigned long long *tf = nullptr;
    if (!rc) rc = h->alloc(&tf, 4096);
    D.tile_flag = tf;
  }
  D.bar = bar; D.err = err;
  if (rc) { pcom_gpu_destroy(h); return rc; }
  // reference initial values (mod_arrays.f90:298-313): alpha = 1/1000.0, am = am_c, ch = 1
  {
    LitMode lit{(d.flags & PCOM_LIT_R8) != 0};
    std::vector<double> v((size_t)n3, lit(1.0f / 1000.0f, 1.0 / 1000.0));
    if (h->mixed) {
      // the anomaly profile is zero until the first state arrives
      std::vector<float> f((size_t)n3, (float)v[0]);
      cudaMemcpy(h->DM.alpha, f.data(), n3 * sizeof(float), cudaMemcpyHostToDevice);
      std::fill(f.begin(), f.end(), (float)LIT(1.0e3));
      cudaMemcpy(h->DM.am, f.data(), n3 * sizeof(float), cudaMemcpyHostToDevice);
      std::fill(v.begin(), v.end(), LIT(1.0e3));
      cudaMemcpy(D.am1, v.data(), n2 * sizeof(double), cudaMemcpyHostToDevice);
    } else {
      cudaMemcpy(D.alpha, v.data(), n3 * sizeof(double), cudaMemcpyHostToDevice);
      std::fill(v.begin(), v.end(), LIT(1.0e3));
      cudaMemcpy(D.am, v.data(), n3 * sizeof(double), cudaMemcpyHostToDevice);
    }
    std::vector<double> one((size_t)n2, 1.0);
    for (double *c : {D.chc, D.chp, D.mch, D.mch2}) cudaMemcpy(c, one.data(), n2 * sizeof(double), cudaMemcpyHostToDevice);
  }
  h->itc = h->itp = 0;
  h->ic = 0; h->ip = 1; h->ipp = 2;
  sync_common(h);
  bind_rotating(h);
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) { pcom_gpu_destroy(h); return fail(PCOM_ERR_CUDA, "init: %s", cudaGetErrorString(e)); }
  *out = h;
  return PCOM_OK;
}

int pcom_gpu_destroy(pcom_handle *h) {
  if (!h) return PCOM_OK;
  cudaStreamSynchronize(h->stream);
  for (auto &kv : h->prof_tab)
    for (auto &pe : kv.second.pending) { cudaEventDestroy(pe.first); cudaEventDestroy(pe.second); }
  if (h->side) {
    cudaStreamSynchronize(h->side);
    cudaStreamDestroy(h->side);
  }
  for (int q = 0; q < 2; ++q) {
    if (h->ev_fork[q]) cudaEventDestroy(h->ev_fork[q]);
    if (h->ev_join[q]) cudaEventDestroy(h->ev_join[q]);
    if (h->ev_frc_free[q]) cudaEventDestroy(h->ev_frc_free[q]);
  }
  for (cudaStream_t cs : {h->copy, h->copy_out})
    if (cs) {
      cudaStreamSynchronize(cs);
      cudaStreamDestroy(cs);
    }
  for (cudaEvent_t ev : {h->ev_frc, h->ev_snap, h->ev_d2h})
    if (ev) cudaEventDestroy(ev);
  for (void *p : h->allocs) cudaFree(p);
  if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return PCOM_OK;
}

int pcom_gpu_upload_static(pcom_handle *h, const pcom_static *s) {
  if (!h || !s) return fail(PCOM_ERR_ARG, "null argument");
  const int ni = h->ni, nj = h->nj, nk = h->nk, nkp = h->nkp;
  const long long n2 = h->n2;
  Dev &D = h->D;
  // masks must be lev >= k (set_grid, main.f90:601-625)
  if (!s->msk_t || !s->lev_t || !s->msk_u || !s->lev_u) return fail(PCOM_ERR_ARG, "masks and levels are required");
  for (int k = 1; k <= nk; ++k)
    for (long long q = 0; q < n2; ++q) {
      const int mt = s->lev_t[q] >= k, mu = s->lev_u[q] >= k;
      if (s->msk_t[q + n2 * (k - 1)] != mt || s->msk_u[q + n2 * (k - 1)] != mu)
        return fail(PCOM_ERR_ARG, "msk is not (lev >= k) at point %lld level %d", q, k);
    }
  std::vector<double> bx((size_t)n2), by((size_t)n2);
  for (int g = 1; g <= 4; ++g) {
    if (!s->rh[g - 1] || !s->dx[g - 1]) return fail(PCOM_ERR_ARG, "grid %d arrays missing", g);
    for (long long q = 0; q < n2; ++q) { bx[q] = s->dx[g - 1][2 * q]; by[q] = s->dx[g - 1][2 * q + 1]; }
    CK(cudaMemcpy((void *)D.rh[g], s->rh[g - 1], n2 * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy((void *)D.dxx[g], bx.data(), n2 * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy((void *)D.dxy[g], by.data(), n2 * sizeof(double), cudaMemcpyHostToDevice));
  }
  // lat-lon metrics: dx?x(i, j) = dx?x(i), dx?y(i, j) = dx?y(j), rh?(i, j) = rh?(j),
  // as set_hgrid builds them from 1-D lon/lat (main.f90:408-493).  Kept as
  // 1-D vectors with the correctly rounded reciprocal of every divisor the
  // step uses (IEEE division on the host), so kernels divide with dvr.
  {
    const double a = D.c.a;
    std::vector<double> x1((size_t)ni), y1((size_t)nj), r1((size_t)nj), v((size_t)std::max(ni, nj));
    for (int g = 1; g <= 4; ++g) {
      const double *dx = s->dx[g - 1], *rh = s->rh[g - 1];
      for (int j = 0; j < nj; ++j)
        for (int i = 0; i < ni; ++i) {
          const long long q = i + (long long)ni * j;
          if (dx[2 * q] != dx[2 * (long long)i] || dx[2 * q + 1] != dx[2 * ((long long)ni * j) + 1] ||
              rh[q] != rh[(long long)ni * j])
            return fail(PCOM_ERR_ARG, "grid %d metrics are not those of a lat-lon grid (point %d, %d)", g, i + 1, j + 1);
        }
      for (int i = 0; i < ni; ++i) x1[i] = dx[2 * (long long)i];
      for (int j = 0; j < nj; ++j) { y1[j] = dx[2 * ((long long)ni * j) + 1]; r1[j] = rh[(long long)ni * j]; }
      auto up = [&](const double *dst, const std::vector<double> &src, int n) -> int {
        CK(cudaMemcpy((void *)dst, src.data(), n * sizeof(double), cudaMemcpyHostToDevice));
        return PCOM_OK;
      };
      int rc = 0;
      rc |= up(D.dxx1d[g], x1, ni);
      rc |= up(D.dxy1d[g], y1, nj);
      rc |= up(D.rh1d[g], r1, nj);
      for (int i = 0; i < ni; ++i) v[i] = 1.0 / x1[i];
      rc |= up(D.rdxx1d[g], v, ni);
      for (int j = 0; j < nj; ++j) v[j] = 1.0 / y1[j];
      rc |= up(D.rdxy1d[g], v, nj);
      for (int j = 0; j < nj; ++j) v[j] = 1.0 / r1[j];
      rc |= up(D.rrh1d[g], v, nj);
      for (int j = 0; j < nj; ++j) v[j] = a * r1[j];
      rc |= up(D.arh1d[g], v, nj);
      for (int j = 0; j < nj; ++j) v[j] = 1.0 / (a * r1[j]);
      rc |= up(D.rarh1d[g], v, nj);
      if (g == 3) {
        for (int j = 0; j < nj; ++j) v[j] = a * a * r1[j];
        rc |= up(D.aarh3, v, nj);
        for (int j = 0; j < nj; ++j) v[j] = 1.0 / (a * a * r1[j]);
        rc |= up(D.raarh3, v, nj);
      }
      if (rc) return rc;
    }
    D.separable = 1;
    h->trop_blocks = 0;  // re-pick the barotropic kernel configuration
    // smag's dy (j) and dx (i, j) (mod_int.f90:416-418) and their reciprocals
    const double *dx2 = s->dx[1], *dx4 = s->dx[3], *rh4 = s->rh[3];
    for (int j = 0; j < nj; ++j) v[j] = (j + 1 < nj) ? a * (dx2[2 * ((long long)ni * j) + 1] + dx2[2 * ((long long)ni * (j + 1)) + 1]) : 1.0;
    CK(cudaMemcpy((void *)D.dys1d, v.data(), nj * sizeof(double), cudaMemcpyHostToDevice));
    for (int j = 0; j < nj; ++j) v[j] = 1.0 / v[j];
    CK(cudaMemcpy((void *)D.rdys1d, v.data(), nj * sizeof(double), cudaMemcpyHostToDevice));
    std::vector<double> w2((size_t)n2, 1.0), rw2((size_t)n2, 1.0);
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i + 1 < ni; ++i) {
        const long long q = i + (long long)ni * j;
        w2[q] = a * (rh4[q] * dx4[2 * q] + rh4[q + 1] * dx4[2 * (q + 1)]);
        rw2[q] = 1.0 / w2[q];
      }
    CK(cudaMemcpy((void *)D.dxs, w2.data(), n2 * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy((void *)D.rdxs, rw2.data(), n2 * sizeof(double), cudaMemcpyHostToDevice));
    // 1/prh, and the Coriolis-adjustment denominators 1 + (0.5 cor dt)^2
    // (mod_int.f90:246, 358-361) for dtbt and dtbc
    for (long long q = 0; q < n2; ++q) { w2[q] = 1.0 / s->prh_t[q]; rw2[q] = 1.0 / s->prh_u[q]; }
    CK(cudaMemcpy((void *)D.rprh_t, w2.data(), n2 * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy((void *)D.rprh_u, rw2.data(), n2 * sizeof(double), cudaMemcpyHostToDevice));
    for (long long q = 0; q < n2; ++q) {
      const double wc = 0.5 * s->cor[q] * (double)D.bc, wt = 0.5 * s->cor[q] * (double)D.bt;
      w2[q] = 1.0 / (1 + wc * wc);
      rw2[q] = 1.0 / (1 + wt * wt);
    }
    CK(cudaMemcpy((void *)D.rwc, w2.data(), n2 * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy((void *)D.rwt, rw2.data(), n2 * sizeof(double), cudaMemcpyHostToDevice));
    D.ra = 1.0 / a;
    D.rg = 1.0 / D.c.g;
    D.rbc32 = 1.0 / (double)(4 * 8 * D.bc);
  }
  if (!s->tn[2]) return fail(PCOM_ERR_ARG, "tn of grid 3 missing");
  CK(cudaMemcpy((void *)D.tn3, s->tn[2], n2 * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy((void *)D.lev_t, s->lev_t, n2 * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy((void *)D.lev_u, s->lev_u, n2 * sizeof(int), cudaMemcpyHostToDevice));
  const double *src2[8] = {s->prh_t, s->phih_t, s->prh_u, s->cv1, s->cv2, s->cor, s->graphihx, s->graphihy};
  const double *dst2[8] = {D.prh_t, D.phih_t, D.prh_u, D.cv1, D.cv2, D.cor, D.graphihx, D.graphihy};
  for (int q = 0; q < 8; ++q) {
    if (!src2[q]) return fail(PCOM_ERR_ARG, "static 2-D array %d missing", q);
    CK(cudaMemcpy((void *)dst2[q], src2[q], n2 * sizeof(double), cudaMemcpyHostToDevice));
  }
  if (!s->km || !s->kh) return fail(PCOM_ERR_ARG, "km/kh missing");
  if (h->mixed) {
    int rc2 = put_f32(h, (float *)h->DM.km, s->km, h->n3p, 0);
    if (!rc2) rc2 = put_f32(h, (float *)h->DM.kh, s->kh, h->n3p, 0);
    if (rc2) return rc2;
    CK(cudaStreamSynchronize(h->stream));
  } else {
    CK(cudaMemcpy((void *)D.km, s->km, h->n3p * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy((void *)D.kh, s->kh, h->n3p * sizeof(double), cudaMemcpyHostToDevice));
  }
  h->lev_t_host.assign(s->lev_t, s->lev_t + n2);
  if (!s->pr2 || !s->dpr2 || !s->dz1) return fail(PCOM_ERR_ARG, "vertical grid missing");
  for (int k = 1; k <= nk; ++k) { D.pr2[k] = s->pr2[k - 1]; D.dpr2[k] = s->dpr2[k - 1]; D.rdpr2[k] = 1.0 / s->dpr2[k - 1]; }
  for (int k = 1; k <= nkp; ++k) { D.dz1[k] = s->dz1[k - 1]; D.rdz1[k] = 1.0 / s->dz1[k - 1]; }
  for (int k = 1; k <= nk; ++k) D.dz2[k] = s->dz2 ? s->dz2[k - 1] : 0.0;
  (void)ni; (void)nj;
  sync_common(h);
  h->static_ok = true;
  return PCOM_OK;
}

int pcom_gpu_set_state(pcom_handle *h, const pcom_state *s) {
  if (!h || !s) return fail(PCOM_ERR_ARG, "null argument");
  const long long n2 = h->n2, n3 = h->n3;
  Dev &D = h->D;
  // tracers: keep tc and tp in distinct buffers when both are given
  if (s->tp || s->sp) {
    if (h->itc == h->itp) {
      int fr = 0;
      while (fr == h->itc) ++fr;
      // preserve the current tc/sc contents in the new tp buffer first
      if (h->mixed) {
        CK(cudaMemcpyAsync(h->t_poolf[fr], h->t_poolf[h->itc], n3 * sizeof(float), cudaMemcpyDeviceToDevice, h->stream));
        CK(cudaMemcpyAsync(h->s_poolf[fr], h->s_poolf[h->itc], n3 * sizeof(float), cudaMemcpyDeviceToDevice, h->stream));
      } else {
        CK(cudaMemcpyAsync(h->t_pool[fr], h->t_pool[h->itc], n3 * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        CK(cudaMemcpyAsync(h->s_pool[fr], h->s_pool[h->itc], n3 * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
      }
      h->itp = fr;
      bind_rotating(h);
    }
  }
  if (h->mixed) return set_state_mixed(h, s);
  int rc = 0;
  auto in = [&](double *dst, const double *src, long long n) { if (!rc) rc = copy_in(h, dst, src, n); };
  in(D.tc, s->tc, n3); in(D.sc, s->sc, n3); in(D.tp, s->tp, n3); in(D.sp, s->sp, n3);
  in(D.uc, s->uc, n3); in(D.vc, s->vc, n3); in(D.up, s->up, n3); in(D.vp, s->vp, n3);
  in(D.auc, s->auc, n3); in(D.aup, s->aup, n3); in(D.aupp, s->aupp, n3);
  in(D.avc, s->avc, n3); in(D.avp, s->avp, n3); in(D.avpp, s->avpp, n3);
  in(D.ubc, s->ubc, n2); in(D.vbc, s->vbc, n2); in(D.ubp, s->ubp, n2); in(D.vbp, s->vbp, n2);
  in(D.chc, s->chc, n2); in(D.chp, s->chp, n2); in(D.mch, s->mch, n2); in(D.mch2, s->mch2, n2);
  in(D.am, s->am, n3); in((double *)D.prho, s->prho, 2 * n3);
  in(D.alpha, s->alpha, n3); in(D.adp, s->adp, n3); in(D.wm, s->wm, h->n3p);
  if (rc) return rc;
  CK(cudaStreamSynchronize(h->stream));
  return PCOM_OK;
}

int pcom_gpu_get_state(pcom_handle *h, pcom_state *s) {
  if (!h || !s) return fail(PCOM_ERR_ARG, "null argument");
  int rc = 0;
  auto out = [&](double *dst, const char *name) { if (!rc) rc = fetch(h, name, dst); };
  out(s->tc, "tc"); out(s->sc, "sc"); out(s->tp, "tp"); out(s->sp, "sp");
  out(s->uc, "uc"); out(s->vc, "vc"); out(s->up, "up"); out(s->vp, "vp");
  out(s->auc, "auc"); out(s->aup, "aup"); out(s->aupp, "aupp");
  out(s->avc, "avc"); out(s->avp, "avp"); out(s->avpp, "avpp");
  out(s->ubc, "ubc"); out(s->vbc, "vbc"); out(s->ubp, "ubp"); out(s->vbp, "vbp");
  out(s->chc, "chc"); out(s->chp, "chp"); out(s->mch, "mch"); out(s->mch2, "mch2");
  out(s->am, "am"); out(s->prho, "prho");
  out(s->alpha, "alpha"); out(s->adp, "adp"); out(s->wm, "wm");
  if (rc) return rc;
  return sync_check(h);
}

int pcom_gpu_set_forcing(pcom_handle *h, const pcom_forcing *f) {
  if (!h || !f) return fail(PCOM_ERR_ARG, "null argument");
  const long long n2 = h->n2;
  int rc = apply_staged_forcing(h);
  if (rc) return rc;
  Dev &D = h->D;
  auto in = [&](const double *dst, const double *src) { if (!rc) rc = copy_in(h, (double *)dst, src, n2); };
  in(D.taux, f->taux); in(D.tauy, f->tauy); in(D.bnd_t, f->t); in(D.bnd_s, f->s); in(D.bnd_pa, f->pa);
  return rc;
}

int pcom_gpu_set_forcing_async(pcom_handle *h, const pcom_forcing *f) {
  if (!h || !f) return fail(PCOM_ERR_ARG, "null argument");
  const double *src[5] = {f->taux, f->tauy, f->t, f->s, f->pa};
  for (const double *p : src)
    if (!p) return fail(PCOM_ERR_ARG, "pcom_gpu_set_forcing_async needs taux, tauy, t, s and pa");
  const long long n2 = h->n2;
  if (!h->frc_buf[1][0]) {
    Dev &D = h->D;
    double *cur[5] = {const_cast<double *>(D.taux), const_cast<double *>(D.tauy), const_cast<double *>(D.bnd_t),
                      const_cast<double *>(D.bnd_s), const_cast<double *>(D.bnd_pa)};
    for (int k = 0; k < 5; ++k) {
      h->frc_buf[0][k] = cur[k];
      int rc = h->alloc(&h->frc_buf[1][k], (size_t)n2);
      if (rc) return rc;
    }
    // the upload stream writes the new set only after its zero-fill
    CK(cudaEventRecord(h->ev_frc_free[1], h->stream));
  }
  // the set not in use (or the one already staged); wait until the steps
  // that read it have run
  const int tgt = h->frc_pending >= 0 ? h->frc_pending : (h->frc_cur ^ 1);
  CK(cudaStreamWaitEvent(h->copy, h->ev_frc_free[tgt], 0));
  for (int k = 0; k < 5; ++k)
    CK(cudaMemcpyAsync(h->frc_buf[tgt][k], src[k], n2 * sizeof(double), cudaMemcpyHostToDevice, h->copy));
  CK(cudaEventRecord(h->ev_frc, h->copy));
  h->frc_pending = tgt;
  return PCOM_OK;
}

int pcom_gpu_get_state_async(pcom_handle *h, pcom_state *s) {
  if (!h || !s) return fail(PCOM_ERR_ARG, "null argument");
  struct Out { double *dst; const char *name; };
  const Out outs[] = {{s->tc, "tc"}, {s->sc, "sc"}, {s->tp, "tp"}, {s->sp, "sp"}, {s->uc, "uc"}, {s->vc, "vc"},
                      {s->up, "up"}, {s->vp, "vp"}, {s->auc, "auc"}, {s->aup, "aup"}, {s->aupp, "aupp"},
                      {s->avc, "avc"}, {s->avp, "avp"}, {s->avpp, "avpp"}, {s->ubc, "ubc"}, {s->vbc, "vbc"},
                      {s->ubp, "ubp"}, {s->vbp, "vbp"}, {s->chc, "chc"}, {s->chp, "chp"}, {s->mch, "mch"},
                      {s->mch2, "mch2"}, {s->am, "am"}, {s->prho, "prho"}, {s->alpha, "alpha"}, {s->adp, "adp"},
                      {s->wm, "wm"}};
  // the snapshots are rewritten only after the previous call's host copies
  CK(cudaStreamWaitEvent(h->stream, h->ev_d2h, 0));
  std::vector<std::pair<double *, std::pair<const double *, long long>>> jobs;
  for (const Out &o : outs) {
    if (!o.dst) continue;
    Named f = lookup(h, o.name);
    if (!f.p && !f.pf) return fail(PCOM_ERR_ARG, "unknown field '%s'", o.name);
    double *&buf = h->snap[o.name];
    if (!buf) {
      int rc = h->alloc(&buf, (size_t)f.n);
      if (rc) return rc;
    }
    if (f.p) {
      CK(cudaMemcpyAsync(buf, f.p, f.n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    } else {
      const Profile pr = profile_of(h->D);
      k_to_f64<<<592, 256, 0, h->stream>>>(f.pf, buf, f.n, h->n2, f.per, f.kind, pr);
      CK(cudaGetLastError());
      h->launches++;
    }
    jobs.push_back({o.dst, {buf, f.n}});
  }
  CK(cudaEventRecord(h->ev_snap, h->stream));
  CK(cudaStreamWaitEvent(h->copy_out, h->ev_snap, 0));
  for (auto &j : jobs)
    CK(cudaMemcpyAsync(j.first, j.second.first, j.second.second * sizeof(double), cudaMemcpyDeviceToHost,
                       h->copy_out));
  CK(cudaEventRecord(h->ev_d2h, h->copy_out));
  return PCOM_OK;
}

int pcom_gpu_get_accum(pcom_handle *h, pcom_accum *a) {
  if (!h || !a) return fail(PCOM_ERR_ARG, "null argument");
  int rc = 0;
  auto out = [&](double *dst, const char *name) { if (!rc) rc = fetch(h, name, dst); };
  out(a->act, "act"); out(a->acs, "acs"); out(a->acr, "acr");
  out(a->acu, "acu"); out(a->acv, "acv"); out(a->acw, "acw");
  out(a->acch, "acch"); out(a->acssh, "acssh");
  a->n_ts = h->n_ts; a->n_uv = h->n_uv; a->n_w = h->n_w; a->n_ch = h->n_ch; a->n_ssh = h->n_ssh;
  if (rc) return rc;
  return sync_check(h);
}

int pcom_gpu_reset_accum(pcom_handle *h) {
  if (!h) return fail(PCOM_ERR_ARG, "null handle");
  Dev &D = h->D;
  if (h->mixed) {
    for (float *p : {h->DM.act, h->DM.acs, h->DM.acr, h->DM.acu, h->DM.acv, h->DM.acw})
      CK(cudaMemsetAsync(p, 0, h->n3 * sizeof(float), h->stream));
  } else {
    for (double *p : {D.act, D.acs, D.acr, D.acu, D.acv, D.acw})
      CK(cudaMemsetAsync(p, 0, h->n3 * sizeof(double), h->stream));
  }
  for (double *p : {D.acch, D.acssh}) CK(cudaMemsetAsync(p, 0, h->n2 * sizeof(double), h->stream));
  h->n_ts = h->n_uv = h->n_w = h->n_ch = h->n_ssh = 0;
  return sync_check(h);
}

int pcom_gpu_den_prho(pcom_handle *h) {
  if (!h) return fail(PCOM_ERR_ARG, "null handle");
  if (!h->static_ok) return fail(PCOM_ERR_STATE, "den_prho before pcom_gpu_upload_static");
  {
    Prof p(h, "den_prho");
    if (h->mixed) launch_den_prho(h->DM, h->stream);
    else launch_den_prho(h->D, h->stream);
  }
  return sync_check(h);
}

int pcom_gpu_step_async(pcom_handle *h, int64_t tctr_i) { return enqueue_step(h, tctr_i); }

int pcom_gpu_step(pcom_handle *h, int64_t tctr_i) {
  int rc = enqueue_step(h, tctr_i);
  if (rc) return rc;
  return sync_check(h);
}

int pcom_gpu_phase(pcom_handle *h, int32_t phase, int64_t tctr_i) {
  if (!h) return fail(PCOM_ERR_ARG, "null handle");
  if (!h->static_ok) return fail(PCOM_ERR_STATE, "phase before pcom_gpu_upload_static");
  if (int rc = apply_staged_forcing(h)) return rc;
  int rc = run_phase(h, phase, tctr_i);
  if (rc) return rc;
  return sync_check(h);
}

int64_t pcom_gpu_field_size(pcom_handle *h, const char *name) {
  if (!h || !name) return 0;
  return lookup(h, name).n;
}

int pcom_gpu_get_field(pcom_handle *h, const char *name, double *host, int64_t n) {
  if (!h || !name || !host) return fail(PCOM_ERR_ARG, "null argument");
  Named f = lookup(h, name);
  if (!f.p && !f.pf) return fail(PCOM_ERR_ARG, "unknown field '%s'", name);
  if (n < f.n) return fail(PCOM_ERR_ARG, "buffer for '%s' holds %lld < %lld doubles", name, (long long)n, f.n);
  int rc = fetch(h, name, host);
  if (rc) return rc;
  return sync_check(h);
}

int pcom_gpu_set_rows(pcom_handle *h, int32_t j_lo, int32_t j_hi) {
  if (!h) return fail(PCOM_ERR_ARG, "null handle");
  if (j_lo < 1 || j_hi > h->nj || j_lo > j_hi)
    return fail(PCOM_ERR_ARG, "rows %d..%d are not a range within 1..%d", j_lo, j_hi, h->nj);
  CK(cudaStreamSynchronize(h->stream));
  h->D.j_lo = j_lo;
  h->D.j_hi = j_hi;
  sync_common(h);
  return PCOM_OK;
}

int pcom_gpu_field_ptr(pcom_handle *h, const char *name, void **dev, int64_t *count, int32_t *elem_bytes) {
  if (!h || !name || !dev || !count || !elem_bytes) return fail(PCOM_ERR_ARG, "null argument");
  Named f = lookup(h, name);
  if (!f.p && !f.pf) return fail(PCOM_ERR_ARG, "unknown field '%s'", name);
  *dev = f.p ? (void *)f.p : (void *)f.pf;
  *count = f.n;
  *elem_bytes = f.p ? 8 : 4;
  return PCOM_OK;
}

int pcom_gpu_check_finite(pcom_handle *h) {
  if (!h) return fail(PCOM_ERR_ARG, "null handle");
  Dev &D = h->D;
  CK(cudaMemsetAsync(h->d_count, 0, sizeof(unsigned long long), h->stream));
  if (h->mixed) {
    const DevM &M = h->DM;
    struct F { const float *p; const int *lev; } fs[] = {{M.tc, D.lev_t}, {M.sc, D.lev_t}, {M.uc, D.lev_u}, {M.vc, D.lev_u}};
    for (auto &f : fs) {
      Prof p(h, "watchdog");
      k_nonfinite<float><<<592, 256, 0, h->stream>>>(f.p, f.lev, h->nk, h->n2, h->nk, h->d_count);
    }
  } else {
    struct F { const double *p; const int *lev; } fs[] = {{D.tc, D.lev_t}, {D.sc, D.lev_t}, {D.uc, D.lev_u}, {D.vc, D.lev_u}};
    for (auto &f : fs) {
      Prof p(h, "watchdog");
      launch_nonfinite(f.p, f.lev, h->nk, h->n2, h->nk, h->d_count, h->stream);
    }
  }
  struct G { const double *p; const int *lev; } gs[] = {{D.chc, D.lev_t}, {D.ubc, D.lev_u}, {D.vbc, D.lev_u}};
  for (auto &f : gs) {
    Prof p(h, "watchdog");
    launch_nonfinite(f.p, f.lev, h->nk, h->n2, 1, h->d_count, h->stream);
  }
  unsigned long long c = 0;
  CK(cudaMemcpyAsync(&c, h->d_count, sizeof c, cudaMemcpyDeviceToHost, h->stream));
  int rc = sync_check(h);
  if (rc) return rc;
  if (c) return fail(PCOM_ERR_NUMERIC, "%llu non-finite wet values in the prognostic fields", c);
  return PCOM_OK;
}

int pcom_gpu_global_sums(pcom_handle *h, double *out3) {
  if (!h || !out3) return fail(PCOM_ERR_ARG, "null argument");
  if (!h->static_ok) return fail(PCOM_ERR_STATE, "global sums before pcom_gpu_upload_static");
  const int nb = 1024;
  if (h->mixed) k_sums<float><<<nb, 256, 0, h->stream>>>(h->DM, h->d_sums);
  else k_sums<double><<<nb, 256, 0, h->stream>>>(h->D, h->d_sums);
  k_sums_final<<<1, 32, 0, h->stream>>>(h->d_sums, nb, h->d_sums + 3 * nb);
  CK(cudaGetLastError());
  h->launches += 2;
  CK(cudaMemcpyAsync(out3, h->d_sums + 3 * nb, 3 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  return sync_check(h);
}

namespace {
CnnStatsDev stats_dev(const pcom_cnn_stats *s) {
  CnnStatsDev d{};
  memcpy(d.in_mean, s->in_mean, sizeof d.in_mean);
  memcpy(d.in_std, s->in_std, sizeof d.in_std);
  memcpy(d.out_std, s->out_std, sizeof d.out_std);
  memcpy(d.out_gain, s->out_gain, sizeof d.out_gain);
  d.out_clip = s->out_clip;
  memcpy(d.alpha_ref, s->alpha_ref, sizeof d.alpha_ref);
  return d;
}
Grid2 grid2(const pcom_handle *h) { return Grid2{h->ni, h->dims.glo_ni, h->dims.glo_nj, h->nk, h->n2}; }
}  // namespace

int pcom_gpu_coarsen(pcom_handle *f, pcom_handle *c, int32_t factor) {
  if (!f || !c || factor < 1) return fail(PCOM_ERR_ARG, "null handle or factor < 1");
  if (f->mixed || c->mixed) return fail(PCOM_ERR_ARG, "coarsening runs on FP64 handles");
  if (!f->static_ok || !c->static_ok) return fail(PCOM_ERR_STATE, "static data missing");
  if (f->dims.glo_ni != factor * c->dims.glo_ni || f->dims.glo_nj != factor * c->dims.glo_nj || f->nk != c->nk)
    return fail(PCOM_ERR_ARG, "grids do not nest with factor %d", factor);
  CK(cudaStreamSynchronize(f->stream));
  const Grid2 F = grid2(f), Cg = grid2(c);
  Dev &A = f->D, &B = c->D;
  const int nk = c->nk;
  auto run = [&](const double *src, double *dst, const int *lev, const int *levc, int nlev, int plane) {
    k_coarsen<<<592, 256, 0, c->stream>>>(src, dst, lev, levc, F, Cg, nlev, factor, plane);
  };
  run(A.tc, B.tc, A.lev_t, nullptr, nk, 1);
  run(A.sc, B.sc, A.lev_t, nullptr, nk, 1);
  if (B.tp != B.tc) { run(A.tp, B.tp, A.lev_t, nullptr, nk, 1); run(A.sp, B.sp, A.lev_t, nullptr, nk, 1); }
  // velocities and their tendencies vanish at the coarse grid's land U points
  const double *fu[] = {A.uc, A.vc, A.up, A.vp, A.auc, A.aup, A.aupp, A.avc, A.avp, A.avpp};
  double *cu[] = {B.uc, B.vc, B.up, B.vp, B.auc, B.aup, B.aupp, B.avc, B.avp, B.avpp};
  for (int q = 0; q < 10; ++q) run(fu[q], cu[q], A.lev_u, B.lev_u, nk, 1);
  run(A.am, B.am, A.lev_u, nullptr, nk, 1);
  const double *ft[] = {A.chc, A.chp, A.mch, A.mch2};
  double *ct[] = {B.chc, B.chp, B.mch, B.mch2};
  for (int q = 0; q < 4; ++q) run(ft[q], ct[q], A.lev_t, nullptr, 1, 0);
  const double *fb[] = {A.ubc, A.vbc, A.ubp, A.vbp};
  double *cb[] = {B.ubc, B.vbc, B.ubp, B.vbp};
  for (int q = 0; q < 4; ++q) run(fb[q], cb[q], A.lev_u, B.lev_u, 1, 0);
  CK(cudaGetLastError());
  c->launches += 21;
  return sync_check(c);
}

int pcom_gpu_cnn_features(pcom_handle *h, void *x, const pcom_cnn_stats *st) {
  if (!h || !x || !st) return fail(PCOM_ERR_ARG, "null argument");
  if ((uintptr_t)x & 15u) return fail(PCOM_ERR_ARG, "x must be 16-byte aligned");
  const dim3 grid((unsigned)((h->dims.glo_ni + 127) / 128), (unsigned)h->dims.glo_nj, (unsigned)h->nk);
  if (h->mixed) k_cnn_features<float><<<grid, 128, 0, h->stream>>>(h->DM, (__nv_bfloat16 *)x, stats_dev(st));
  else k_cnn_features<double><<<grid, 128, 0, h->stream>>>(h->D, (__nv_bfloat16 *)x, stats_dev(st));
  CK(cudaGetLastError());
  h->launches++;
  return PCOM_OK;
}

int pcom_gpu_cnn_target(pcom_handle *pred, pcom_handle *truth, float *target, float *mask, const pcom_cnn_stats *st,
                        double dt) {
  if (!pred || !truth || !st || dt <= 0) return fail(PCOM_ERR_ARG, "bad argument");
  if (pred->mixed || truth->mixed) return fail(PCOM_ERR_ARG, "closure targets are built from FP64 handles");
  if (pred->n3 != truth->n3) return fail(PCOM_ERR_ARG, "handles differ in size");
  CK(cudaStreamSynchronize(truth->stream));
  k_cnn_target<<<592, 256, 0, pred->stream>>>(pred->D, truth->D, target, mask, stats_dev(st), 1.0 / dt);
  CK(cudaGetLastError());
  pred->launches++;
  return PCOM_OK;
}

int pcom_gpu_cnn_apply(pcom_handle *h, const float *y, const pcom_cnn_stats *st, double dt) {
  if (!h || !y || !st) return fail(PCOM_ERR_ARG, "null argument");
  if ((uintptr_t)y & 15u) return fail(PCOM_ERR_ARG, "y must be 16-byte aligned");
  const dim3 grid((unsigned)((h->dims.glo_ni + 127) / 128), (unsigned)h->dims.glo_nj, (unsigned)h->nk);
  if (h->mixed)
    k_cnn_apply<float><<<grid, 128, 0, h->stream>>>(h->DM, y, stats_dev(st), dt, h->DM.tp != h->DM.tc ? 1 : 0);
  else
    k_cnn_apply<double><<<grid, 128, 0, h->stream>>>(h->D, y, stats_dev(st), dt, h->D.tp != h->D.tc ? 1 : 0);
  CK(cudaGetLastError());
  h->launches++;
  return PCOM_OK;
}

int pcom_gpu_set_forcing_months(pcom_handle *h, const pcom_forcing *months) {
  if (!h || !months) return fail(PCOM_ERR_ARG, "null argument");
  const long long n2 = h->n2;
  if (!h->frc_months) {
    int rc = h->alloc(&h->frc_months, (size_t)(5 * 12 * n2));
    if (rc) return rc;
  }
  const double *src[5] = {months->taux, months->tauy, months->t, months->s, months->pa};
  for (int q = 0; q < 5; ++q) {
    if (!src[q]) return fail(PCOM_ERR_ARG, "monthly forcing field %d missing", q);
    CK(cudaMemcpyAsync(h->frc_months + (long long)q * 12 * n2, src[q], 12 * n2 * sizeof(double),
                       cudaMemcpyHostToDevice, h->stream));
  }
  return sync_check(h);
}

int pcom_gpu_int_bnd(pcom_handle *h, int32_t m1, int32_t m2, double f) {
  if (!h) return fail(PCOM_ERR_ARG, "null handle");
  if (!h->frc_months) return fail(PCOM_ERR_STATE, "pcom_gpu_int_bnd before pcom_gpu_set_forcing_months");
  if (m1 < 1 || m1 > 12 || m2 < 1 || m2 > 12) return fail(PCOM_ERR_ARG, "months must be 1..12");
  if (int rc = apply_staged_forcing(h)) return rc;
  Dev &D = h->D;
  k_int_bnd<<<256, 256, 0, h->stream>>>(h->frc_months, (double *)D.taux, (double *)D.tauy, (double *)D.bnd_t,
                                        (double *)D.bnd_s, (double *)D.bnd_pa, h->n2, m1, m2, f);
  CK(cudaGetLastError());
  h->launches++;
  return PCOM_OK;
}

int pcom_gpu_set_trop_kernel(pcom_handle *h, int32_t which) {
  if (!h || which < 0 || which > 3) return fail(PCOM_ERR_ARG, "which must be 0..3");
  CK(cudaStreamSynchronize(h->stream));
  h->trop_force = which;
  h->trop_blocks = 0;  // re-pick at the next step
  return PCOM_OK;
}

int pcom_gpu_set_wait_limit(pcom_handle *h, double seconds) {
  if (!h) return fail(PCOM_ERR_ARG, "null handle");
  if (!(seconds >= 0.0) || seconds > 1.0e6) return fail(PCOM_ERR_ARG, "wait limit must be in [0, 1e6] s");
  CK(cudaStreamSynchronize(h->stream));
  h->D.wait_ns = (unsigned long long)(seconds * 1.0e9);
  sync_common(h);
  return PCOM_OK;
}

int pcom_gpu_set_overlap(pcom_handle *h, int32_t enable) {
  if (!h) return fail(PCOM_ERR_ARG, "null handle");
  CK(cudaStreamSynchronize(h->stream));
  h->overlap = enable != 0;
  return PCOM_OK;
}

int pcom_gpu_set_stream(pcom_handle *h, void *stream) {
  if (!h) return fail(PCOM_ERR_ARG, "null handle");
  CK(cudaStreamSynchronize(h->stream));
  if (h->own_stream) cudaStreamDestroy(h->stream);
  h->stream = (cudaStream_t)stream;
  h->own_stream = false;
  return PCOM_OK;
}

int pcom_gpu_sync(pcom_handle *h) {
  if (!h) return fail(PCOM_ERR_ARG, "null handle");
  return sync_check(h);
}

int pcom_gpu_trop_floor(pcom_handle *h, double *ms) {
  if (!h || !ms) return fail(PCOM_ERR_ARG, "null argument");
  if (!h->static_ok) return fail(PCOM_ERR_STATE, "latency floor before pcom_gpu_upload_static");
  if (h->trop_blocks <= 0) {
    int rc = pick_trop_config(h);
    if (rc) return rc;
  }
  if (!h->trop_resident || h->mixed)
    return fail(PCOM_ERR_STATE, "the latency floor is measured for the resident FP64 barotropic kernel");
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, h->stream));
  cudaError_t e = launch_trop_floor(h->D, h->trop_tx, h->trop_ty, h->trop_epoch, h->stream);
  if (e == cudaSuccess) h->trop_epoch += (unsigned long long)h->D.nstep * (unsigned long long)h->trop_blocks;
  CK(cudaEventRecord(e1, h->stream));
  int rc = sync_check(h);
  float t = 0.f;
  if (rc == PCOM_OK && e == cudaSuccess) cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return fail(PCOM_ERR_CUDA, "latency-floor kernel launch: %s", cudaGetErrorString(e));
  if (rc) return rc;
  *ms = t;
  return PCOM_OK;
}

int pcom_gpu_profile(pcom_handle *h, int32_t enable) {
  if (!h) return fail(PCOM_ERR_ARG, "null handle");
  CK(cudaStreamSynchronize(h->stream));
  for (auto &kv : h->prof_tab)
    for (auto &pe : kv.second.pending) { cudaEventDestroy(pe.first); cudaEventDestroy(pe.second); }
  h->prof_tab.clear();
  h->prof = enable != 0;
  return PCOM_OK;
}

int pcom_gpu_profile_read(pcom_handle *h, char *names, int64_t *launches, double *ms, int32_t cap) {
  if (!h) return fail(PCOM_ERR_ARG, "null handle");
  CK(cudaStreamSynchronize(h->stream));
  int n = 0;
  for (auto &kv : h->prof_tab) {
    ProfEntry &e = kv.second;
    for (auto &pe : e.pending) {
      float t = 0.f;
      cudaEventElapsedTime(&t, pe.first, pe.second);
      e.ms += t;
      cudaEventDestroy(pe.first);
      cudaEventDestroy(pe.second);
    }
    e.pending.clear();
    if (n < cap) {
      if (names) { strncpy(names + 64 * n, kv.first.c_str(), 63); names[64 * n + 63] = 0; }
      if (launches) launches[n] = e.launches;
      if (ms) ms[n] = e.ms;
    }
    ++n;
  }
  return n;
}

int64_t pcom_gpu_launch_count(pcom_handle *h) { return h ? h->launches : 0; }

}  // extern "C"

// constants of a handle, for entry points that build their own device view
void pcom_dev_consts(bool r8, DevConsts &c) { make_consts(r8, c); }

// record a failure for pcom_gpu_last_error from another translation unit
int pcom_set_error(int code, const char *msg) { return fail(code, "%s", msg); }

// =============================================================== batches
// Ensemble members and basins of uneven size stepped together: every kernel
// of the step runs once for all members (grid z = member, Dev per member in
// device memory) and the barotropic subcycle of all members is one
// persistent cooperative launch over the work list of their tiles.  The
// whole step can be captured into CUDA graphs (one per ring-buffer phase).
struct pcom_batch {
  std::vector<pcom_handle *> hs;
  // the batch's own stream (capturable), joined by events to the members'
  // streams before and after its work
  cudaStream_t stream = nullptr;
  cudaEvent_t ev = nullptr;
  std::vector<cudaStream_t> member_streams;
  BatchShape shape{};
  int nstep = 0;
  // barotropic work: members packed into groups whose tiles are co-resident
  // (one tile per CTA, the fast kernel over a tile list); members too large
  // to be resident go to one group of the multi-tile kernel
  struct TropGroup {
    TileRef *d;
    int ntiles, nblocks;
    bool resident;
  };
  std::vector<TropGroup> groups;
  int TX = 24, TY = 18;
  int max_resident = 0;  // > 0: cap on the tiles of one resident group
  int64_t launches = 0;  // kernels this batch launched
  unsigned long long *cnt = nullptr;
  int *err = nullptr;
  // per-phase device copies of the members' Dev (phase = ring indices)
  struct DevArray {
    Dev *d;
    std::vector<Dev> host;
  };
  std::map<int, DevArray> dev_arrays;
  std::map<int, cudaGraphExec_t> graphs;
  bool use_graphs = true;
  std::vector<void *> allocs;
  ~pcom_batch() {
    for (auto &kv : graphs) cudaGraphExecDestroy(kv.second);
    for (void *p : allocs) cudaFree(p);
    if (ev) cudaEventDestroy(ev);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

void member_tiles(const pcom_handle *h, int m, int TX, int TY, std::vector<TileRef> &t) {
  const int G = h->dims.glo_ni, nj = h->nj;
  for (int j0 = 1; j0 <= nj; j0 += TY)
    for (int r0 = 0; r0 < G; r0 += TX) t.push_back({m, r0, j0, std::min(TX, G - r0), std::min(TY, nj - j0 + 1)});
}

// plan the barotropic launches for tile shape TX x TY: first-fit decreasing
// packing of the members' tile lists into groups of at most `cap` tiles
int batch_tiles(pcom_batch *b, int TX, int TY) {
  for (pcom_batch::TropGroup &g : b->groups) {
    cudaFree(g.d);
    b->allocs.erase(std::find(b->allocs.begin(), b->allocs.end(), (void *)g.d));
  }
  b->groups.clear();
  for (auto &kv : b->graphs) cudaGraphExecDestroy(kv.second);
  b->graphs.clear();
  int cap = trop_group_max_blocks(TX, TY);
  if (b->max_resident > 0) cap = std::min(cap, b->max_resident);
  const int n = (int)b->hs.size();
  std::vector<std::vector<TileRef>> mt(n);
  for (int m = 0; m < n; ++m) member_tiles(b->hs[m], m, TX, TY, mt[m]);
  std::vector<int> order(n);
  for (int m = 0; m < n; ++m) order[m] = m;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return mt[x].size() > mt[y].size(); });
  std::vector<std::vector<TileRef>> res;  // resident groups
  std::vector<TileRef> big;               // members that cannot be resident
  for (int m : order) {
    const int nt = (int)mt[m].size();
    if (nt > cap) {
      big.insert(big.end(), mt[m].begin(), mt[m].end());
      continue;
    }
    bool placed = false;
    for (auto &g : res)
      if ((int)(g.size() + nt) <= cap) {
        g.insert(g.end(), mt[m].begin(), mt[m].end());
        placed = true;
        break;
      }
    if (!placed) res.push_back(mt[m]);
  }
  auto add = [&](const std::vector<TileRef> &t, bool resident) -> int {
    pcom_batch::TropGroup g{nullptr, (int)t.size(), 0, resident};
    CK(cudaMalloc(&g.d, t.size() * sizeof(TileRef)));
    b->allocs.push_back(g.d);
    CK(cudaMemcpy(g.d, t.data(), t.size() * sizeof(TileRef), cudaMemcpyHostToDevice));
    if (resident) {
      g.nblocks = g.ntiles;
    } else {
      const int mb = trop_batch_max_blocks(TX, TY);
      if (mb <= 0) return fail(PCOM_ERR_ARG, "tile %dx%d does not fit the multi-tile barotropic kernel", TX, TY);
      g.nblocks = std::min(g.ntiles, mb);
    }
    b->groups.push_back(g);
    return PCOM_OK;
  };
  for (auto &g : res) {
    int rc = add(g, true);
    if (rc) return rc;
  }
  if (!big.empty()) {
    int rc = add(big, false);
    if (rc) return rc;
  }
  b->TX = TX;
  b->TY = TY;
  return PCOM_OK;
}

// the barotropic subcycles of all members
cudaError_t batch_trop(pcom_batch *b, const Dev *dP) {
  for (const pcom_batch::TropGroup &g : b->groups) {
    cudaError_t e = g.resident ? launch_trop_group(dP, g.d, g.ntiles, b->TX, b->TY, b->cnt, b->err, b->stream)
                               : launch_trop_batch(dP, g.d, g.ntiles, b->TX, b->TY, g.nblocks, b->cnt, b->err, b->stream);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// order the batch's stream after the work enqueued on the members' streams
int batch_join_in(pcom_batch *b) {
  for (cudaStream_t s : b->member_streams) {
    CK(cudaEventRecord(b->ev, s));
    CK(cudaStreamWaitEvent(b->stream, b->ev, 0));
  }
  return PCOM_OK;
}
// and the members' streams after the batch's work
int batch_join_out(pcom_batch *b) {
  CK(cudaEventRecord(b->ev, b->stream));
  for (cudaStream_t s : b->member_streams) CK(cudaStreamWaitEvent(s, b->ev, 0));
  return PCOM_OK;
}

// the ring phase of a member: AB3 ring indices and the tracer buffers in use
int phase_key(const pcom_handle *h) { return h->ic * 100 + h->ip * 10 + h->ipp + 1000 * (h->itc * 4 + h->itp); }

// the device copy of the members' Dev for ring phase `key`, refreshed when a
// member's Dev changed since it was uploaded (the array keeps its address, so
// graphs captured with it stay valid)
int batch_dev_array(pcom_batch *b, int key, Dev **out) {
  std::vector<Dev> v;
  for (pcom_handle *h : b->hs) v.push_back(h->D);
  auto it = b->dev_arrays.find(key);
  if (it == b->dev_arrays.end()) {
    Dev *d = nullptr;
    CK(cudaMalloc(&d, v.size() * sizeof(Dev)));
    b->allocs.push_back(d);
    it = b->dev_arrays.emplace(key, pcom_batch::DevArray{d, {}}).first;
  }
  pcom_batch::DevArray &a = it->second;
  if (a.host.size() != v.size() || memcmp(a.host.data(), v.data(), v.size() * sizeof(Dev)) != 0) {
    a.host = v;
    CK(cudaMemcpyAsync(a.d, a.host.data(), v.size() * sizeof(Dev), cudaMemcpyHostToDevice, b->stream));
  }
  *out = a.d;
  return PCOM_OK;
}

// enqueue the kernels of one step for all members with Dev array dP
int batch_enqueue(pcom_batch *b, Dev *dP) {
  const BatchShape &s = b->shape;
  cudaStream_t st = b->stream;
  launch_batch(BK_ALPHA_TOBOT, dP, s, 0, st);
  launch_batch(BK_PGRA2D, dP, s, 0, st);
  launch_batch(BK_UV2D, dP, s, 0, st);
  launch_batch(BK_UPWELLING, dP, s, 0, st);
  launch_batch(BK_READYC3D, dP, s, 0, st);
  cudaError_t e = batch_trop(b, dP);
  if (e != cudaSuccess) return fail(PCOM_ERR_CUDA, "batched barotropic launch: %s", cudaGetErrorString(e));
  launch_batch(BK_UV2D, dP, s, 2, st);
  launch_batch(BK_CLIN, dP, s, 0, st);
  launch_batch(BK_SMAG, dP, s, 0, st);
  launch_batch(BK_SSH, dP, s, 0, st);
  launch_batch(BK_UV2D, dP, s, 1, st);
  launch_batch(BK_UPWELLING, dP, s, 1, st);
  launch_batch(BK_TS, dP, s, 0, st);
  CK(cudaGetLastError());
  return PCOM_OK;
}

int batch_sync(pcom_batch *b) {
  CK(cudaStreamSynchronize(b->stream));
  CK(cudaGetLastError());
  int err = 0;
  CK(cudaMemcpy(&err, b->err, sizeof err, cudaMemcpyDeviceToHost));
  if (err) {
    cudaMemsetAsync(b->err, 0, sizeof(int), b->stream);
    cudaStreamSynchronize(b->stream);
    return fail(PCOM_ERR_TIMEOUT, "a device-side grid barrier of the batch gave up waiting (bounded spin)");
  }
  return PCOM_OK;
}

}  // namespace

extern "C" {

int pcom_gpu_batch_create(pcom_handle *const *hs, int32_t n, pcom_batch **out) {
  if (!hs || n <= 0 || !out) return fail(PCOM_ERR_ARG, "null argument or empty batch");
  pcom_batch *b = new pcom_batch();
  for (int m = 0; m < n; ++m) {
    pcom_handle *h = hs[m];
    if (!h || !h->static_ok) { delete b; return fail(PCOM_ERR_STATE, "batch member %d has no static data", m); }
    if (!h->D.separable) { delete b; return fail(PCOM_ERR_ARG, "batch member %d: batches need lat-lon (separable) metrics", m); }
    if (h->mixed) { delete b; return fail(PCOM_ERR_ARG, "batch member %d: batches run the FP64 path only", m); }
    if (h->D.bt != hs[0]->D.bt || h->D.bc != hs[0]->D.bc) { delete b; return fail(PCOM_ERR_ARG, "batch members must share dtbt and dtbc"); }
    if (h->device != hs[0]->device) { delete b; return fail(PCOM_ERR_ARG, "batch members must live on one device"); }
    b->hs.push_back(h);
    b->shape.glo_ni = std::max(b->shape.glo_ni, h->dims.glo_ni);
    b->shape.ni = std::max(b->shape.ni, h->ni);
    b->shape.nj = std::max(b->shape.nj, h->nj);
    b->shape.nk = std::max(b->shape.nk, h->nk);
    cudaStreamSynchronize(h->stream);
  }
  b->shape.n = n;
  b->nstep = hs[0]->D.nstep;
  for (pcom_handle *h : b->hs)
    if (std::find(b->member_streams.begin(), b->member_streams.end(), h->stream) == b->member_streams.end())
      b->member_streams.push_back(h->stream);
  cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMalloc(&b->cnt, sizeof(unsigned long long));
  if (e == cudaSuccess) { b->allocs.push_back(b->cnt); e = cudaMalloc(&b->err, sizeof(int)); }
  if (e == cudaSuccess) { b->allocs.push_back(b->err); e = cudaMemsetAsync(b->err, 0, sizeof(int), b->stream); }
  if (e != cudaSuccess) { delete b; return fail(PCOM_ERR_CUDA, "batch scratch: %s", cudaGetErrorString(e)); }
  int rc = batch_tiles(b, 24, 18);
  if (rc) { delete b; return rc; }
  *out = b;
  return PCOM_OK;
}

int pcom_gpu_batch_destroy(pcom_batch *b) {
  if (!b) return PCOM_OK;
  cudaStreamSynchronize(b->stream);
  delete b;
  return PCOM_OK;
}

int pcom_gpu_batch_use_graphs(pcom_batch *b, int32_t enable) {
  if (!b) return fail(PCOM_ERR_ARG, "null batch");
  b->use_graphs = enable != 0;
  return PCOM_OK;
}

int pcom_gpu_batch_den_prho(pcom_batch *b) {
  if (!b) return fail(PCOM_ERR_ARG, "null batch");
  int rc = batch_join_in(b);
  if (rc) return rc;
  Dev *dP = nullptr;
  rc = batch_dev_array(b, phase_key(b->hs[0]), &dP);
  if (rc) return rc;
  b->launches++;
  launch_batch(BK_DEN_PRHO, dP, b->shape, 0, b->stream);
  rc = batch_join_out(b);
  if (rc) return rc;
  return batch_sync(b);
}

int pcom_gpu_batch_step_async(pcom_batch *b, int64_t tctr_i) {
  if (!b) return fail(PCOM_ERR_ARG, "null batch");
  if (tctr_i < 1) return fail(PCOM_ERR_ARG, "tctr_i must be >= 1");
  for (pcom_handle *h : b->hs)
    if (int rc = apply_staged_forcing(h)) return rc;
  // AB3 ring rotation of every member (mod_int.f90:115-118), in lock step
  const int key0 = phase_key(b->hs[0]);
  for (pcom_handle *h : b->hs) {
    if (phase_key(h) != key0) return fail(PCOM_ERR_STATE, "batch members are not in the same ring phase");
    int old_pp = h->ipp;
    h->ipp = h->ip;
    h->ip = h->ic;
    h->ic = old_pp;
    bind_rotating(h);
    const bool fresh = h->dims.rst != 1;
    h->D.ab3_mode = (fresh && tctr_i == 1) ? 1 : 0;
  }
  const bool startup = tctr_i <= 2;
  int rc0 = batch_join_in(b);
  if (rc0) return rc0;
  for (pcom_handle *h : b->hs)
    if (h->dims.rst != 1 && tctr_i == 2) {
      CK(cudaMemcpyAsync(h->D.aupp, h->D.aup, h->n3 * sizeof(double), cudaMemcpyDeviceToDevice, b->stream));
      CK(cudaMemcpyAsync(h->D.avpp, h->D.avp, h->n3 * sizeof(double), cudaMemcpyDeviceToDevice, b->stream));
    }
  const int key = phase_key(b->hs[0]);
  Dev *dP = nullptr;
  int rc = batch_dev_array(b, key, &dP);
  if (rc) return rc;
  if (startup || !b->use_graphs) {
    // the start-up steps (ab3_mode, aupp = aup) run kernel by kernel
    rc = batch_enqueue(b, dP);
  } else {
    auto it = b->graphs.find(key);
    if (it == b->graphs.end()) {
      cudaGraph_t g = nullptr;
      cudaGraphExec_t ge = nullptr;
      CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      rc = batch_enqueue(b, dP);
      cudaError_t e = cudaStreamEndCapture(b->stream, &g);
      if (rc) { if (g) cudaGraphDestroy(g); return rc; }
      if (e != cudaSuccess) return fail(PCOM_ERR_CUDA, "graph capture of the batched step: %s", cudaGetErrorString(e));
      e = cudaGraphInstantiate(&ge, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return fail(PCOM_ERR_CUDA, "graph instantiation: %s", cudaGetErrorString(e));
      it = b->graphs.emplace(key, ge).first;
    }
    CK(cudaGraphLaunch(it->second, b->stream));
  }
  if (rc) return rc;
  rc = batch_join_out(b);
  if (rc) return rc;
  b->launches += 13 + (int64_t)b->groups.size();  // kernels of one batched step
  for (pcom_handle *h : b->hs) {
    h->D.ab3_mode = 0;
    h->n_ch++; h->n_uv++; h->n_ssh++; h->n_w++; h->n_ts++;
    // tc = tp = the buffer int_ts wrote (mod_int.f90:496-497)
    int fr = 0;
    while (fr == h->itc || fr == h->itp) ++fr;
    h->itc = h->itp = fr;
    bind_rotating(h);
  }
  return PCOM_OK;
}

int pcom_gpu_batch_set_tiles(pcom_batch *b, int32_t tx, int32_t ty, int32_t max_resident) {
  if (!b) return fail(PCOM_ERR_ARG, "null batch");
  if (tx < 1 || ty < 1 || (tx + 4) * (ty + 4) > 640)
    return fail(PCOM_ERR_ARG, "tile %dx%d: need tx, ty >= 1 and (tx+4)*(ty+4) <= 640", tx, ty);
  CK(cudaStreamSynchronize(b->stream));
  b->max_resident = max_resident > 0 ? max_resident : 0;
  return batch_tiles(b, tx, ty);
}

int64_t pcom_gpu_batch_launch_count(pcom_batch *b) { return b ? b->launches : 0; }

int pcom_gpu_batch_sync(pcom_batch *b) {
  if (!b) return fail(PCOM_ERR_ARG, "null batch");
  return batch_sync(b);
}

int pcom_gpu_batch_step(pcom_batch *b, int64_t tctr_i) {
  int rc = pcom_gpu_batch_step_async(b, tctr_i);
  if (rc) return rc;
  return batch_sync(b);
}

// Autotuner: time the barotropic launches of the whole batch for candidate
// tile shapes on the members' current state (the 2-D fields they change are
// saved and restored around every trial) and keep the fastest.  The choice
// is cached per set of member grid sizes, so later batches of the same
// shapes skip the trials.
int pcom_gpu_batch_autotune(pcom_batch *b, char *report, int32_t len) {
  if (!b) return fail(PCOM_ERR_ARG, "null batch");
  static std::mutex cache_mu;
  static std::map<std::string, std::pair<int, int>> cache;
  std::vector<std::string> dims;
  for (pcom_handle *h : b->hs) dims.push_back(std::to_string(h->dims.glo_ni) + "x" + std::to_string(h->dims.glo_nj));
  std::sort(dims.begin(), dims.end());
  std::string sig;
  for (auto &d : dims) sig += d + ",";
  {
    std::lock_guard<std::mutex> lk(cache_mu);
    auto it = cache.find(sig);
    if (it != cache.end()) {
      int rc = batch_tiles(b, it->second.first, it->second.second);
      if (rc) return rc;
      std::string rep = "cached -> " + std::to_string(b->TX) + "x" + std::to_string(b->TY);
      if (report && len > 0) { strncpy(report, rep.c_str(), (size_t)len - 1); report[len - 1] = 0; }
      return PCOM_OK;
    }
  }
  static const int cand[][2] = {{12, 12}, {16, 8},  {16, 12}, {16, 16}, {24, 12}, {20, 16},
                                {24, 18}, {32, 8},  {32, 12}, {28, 16}, {48, 8},  {64, 6}};
  for (cudaStream_t s : b->member_streams) CK(cudaStreamSynchronize(s));
  CK(cudaStreamSynchronize(b->stream));
  // save the 2-D fields the subcycle writes
  std::vector<double *> saved;
  auto fields = [](pcom_handle *h) {
    return std::vector<double *>{h->D.chc, h->D.chp, h->D.mch, h->D.mch2, h->D.ubc, h->D.vbc, h->D.ubp, h->D.vbp, h->D.acch};
  };
  int rc = 0;
  for (pcom_handle *h : b->hs)
    for (double *f : fields(h)) {
      double *c = nullptr;
      if (!rc && cudaMalloc(&c, h->n2 * sizeof(double)) != cudaSuccess) rc = fail(PCOM_ERR_CUDA, "autotune scratch");
      if (!rc && cudaMemcpy(c, f, h->n2 * sizeof(double), cudaMemcpyDeviceToDevice) != cudaSuccess)
        rc = fail(PCOM_ERR_CUDA, "autotune save");
      saved.push_back(c);
    }
  auto restore = [&]() -> int {
    size_t q = 0;
    for (pcom_handle *h : b->hs)
      for (double *f : fields(h)) { CK(cudaMemcpy(f, saved[q], h->n2 * sizeof(double), cudaMemcpyDeviceToDevice)); ++q; }
    return PCOM_OK;
  };
  Dev *dP = nullptr;
  if (!rc) rc = batch_dev_array(b, phase_key(b->hs[0]), &dP);
  double best = 1e30;
  int bx = b->TX, by = b->TY;
  std::string rep;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (auto &c : cand) {
    if (rc) break;
    if (trop_group_max_blocks(c[0], c[1]) <= 0) continue;
    rc = batch_tiles(b, c[0], c[1]);
    if (rc) break;
    float ms = 0.f, tot = 0.f;
    for (int rep_i = 0; rep_i < 3 && !rc; ++rep_i) {
      cudaEventRecord(e0, b->stream);
      cudaError_t e = batch_trop(b, dP);
      cudaEventRecord(e1, b->stream);
      if (e != cudaSuccess) rc = fail(PCOM_ERR_CUDA, "autotune launch: %s", cudaGetErrorString(e));
      if (!rc) rc = batch_sync(b);
      cudaEventElapsedTime(&ms, e0, e1);
      if (rep_i > 0) tot += ms;
      if (!rc) rc = restore();
    }
    const double t = tot / 2.0;
    int res = 0, tiles = 0;
    for (auto &g : b->groups) { res += g.resident; tiles += g.ntiles; }
    char line[128];
    snprintf(line, sizeof line, "%dx%d:%.3fms(%d tiles,%d launches,%d resident) ", c[0], c[1], t, tiles,
             (int)b->groups.size(), res);
    rep += line;
    if (!rc && t < best) { best = t; bx = c[0]; by = c[1]; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  for (double *c : saved) cudaFree(c);
  if (rc) return rc;
  rc = batch_tiles(b, bx, by);
  if (rc) return rc;
  {
    std::lock_guard<std::mutex> lk(cache_mu);
    cache[sig] = {bx, by};
  }
  char line[96];
  snprintf(line, sizeof line, "-> %dx%d", bx, by);
  rep += line;
  if (report && len > 0) { strncpy(report, rep.c_str(), (size_t)len - 1); report[len - 1] = 0; }
  return PCOM_OK;
}

}  // extern "C"
