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
__global__ void k_nonfinite(const double *f, const int *lev, int nk, long long n2, int planes,
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

struct ProfEntry {
  long long launches = 0;
  double ms = 0.0;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending;
};

}  // namespace

void launch_nonfinite(const double *f, const int *lev, int nk, long long n2, int planes, unsigned long long *count,
                      cudaStream_t s) {
  k_nonfinite<<<592, 256, 0, s>>>(f, lev, nk, n2, planes, count);
}

struct pcom_handle {
  pcom_dims dims{};
  int ni = 0, nj = 0, nk = 0, nkp = 0;
  long long n2 = 0, n3 = 0, n3p = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int device = 0;
  Dev D{};
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
  unsigned long long trop_epoch = 0;  // barrier arrivals of the barotropic kernel so far
  bool prof = false;
  std::map<std::string, ProfEntry> prof_tab;
  long long launches = 0;
  unsigned long long *d_count = nullptr;

  template <class T>
  int alloc(T **p, size_t n) {
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, n * sizeof(T));
    if (e != cudaSuccess) return fail(PCOM_ERR_CUDA, "cudaMalloc(%zu bytes): %s", n * sizeof(T), cudaGetErrorString(e));
    cudaMemset(q, 0, n * sizeof(T));
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
  cudaEvent_t a = nullptr, b = nullptr;
  Prof(pcom_handle *h_, const char *n) : h(h_), name(n) {
    h->launches++;
    if (h->prof) {
      cudaEventCreate(&a);
      cudaEventCreate(&b);
      cudaEventRecord(a, h->stream);
    }
  }
  ~Prof() {
    if (h->prof) {
      cudaEventRecord(b, h->stream);
      ProfEntry &e = h->prof_tab[name];
      e.launches++;
      e.pending.emplace_back(a, b);
    }
  }
};

int sync_check(pcom_handle *h) {
  CK(cudaStreamSynchronize(h->stream));
  CK(cudaGetLastError());
  int err[2] = {0, 0};
  CK(cudaMemcpy(err, h->D.err, sizeof err, cudaMemcpyDeviceToHost));
  if (err[0]) {
    cudaMemset(h->D.err, 0, sizeof err);
    cudaMemset(h->D.bar, 0, 2 * sizeof(unsigned));
    cudaMemset(h->D.tile_flag, 0, sizeof(unsigned long long));
    h->trop_epoch = 0;
    return fail(PCOM_ERR_TIMEOUT, "a device-side grid barrier gave up waiting (bounded spin)");
  }
  return PCOM_OK;
}

void bind_rotating(pcom_handle *h) {
  Dev &D = h->D;
  D.auc = h->ab_u[h->ic]; D.aup = h->ab_u[h->ip]; D.aupp = h->ab_u[h->ipp];
  D.avc = h->ab_v[h->ic]; D.avp = h->ab_v[h->ip]; D.avpp = h->ab_v[h->ipp];
  D.tc = h->t_pool[h->itc]; D.tp = h->t_pool[h->itp];
  D.sc = h->s_pool[h->itc]; D.sp = h->s_pool[h->itp];
  int fr = 0;
  while (fr == h->itc || fr == h->itp) ++fr;
  D.tn_ = h->t_pool[fr];
  D.sn_ = h->s_pool[fr];
}

int pick_trop_config(pcom_handle *h) {
  // resident kernel: one tile per CTA, one region point per thread; pick the
  // tiling with the fewest tiles (fewest CTAs at the grid barrier)
  h->trop_resident = false;
  if (h->D.separable) {
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

// ---- the pieces of the step
int do_den_alpha(pcom_handle *h) {
  Prof p(h, "den_alpha+int_tobot");
  launch_alpha_tobot(h->D, h->stream);
  return PCOM_OK;
}
int do_pgra(pcom_handle *h) {
  Prof p(h, "int_pgra");
  launch_pgra2d(h->D, h->stream);
  return PCOM_OK;
}
int do_readyc(pcom_handle *h, int64_t iter) {
  {
    Prof p(h, "readyc_2d");
    launch_uv2d(h->D, 0, h->stream);
  }
  {
    Prof p(h, "upwelling");
    launch_upwelling(h->D, 0, h->stream);
  }
  // AB3 history: aupp <- aup <- auc (mod_int.f90:115-118) by rotation
  int old_pp = h->ipp;
  h->ipp = h->ip;
  h->ip = h->ic;
  h->ic = old_pp;
  bind_rotating(h);
  const bool fresh = h->dims.rst != 1;
  h->D.ab3_mode = (fresh && iter == 1) ? 1 : 0;
  if (fresh && iter == 2) {
    // aupp = aup (mod_int.f90:128-130)
    CK(cudaMemcpyAsync(h->D.aupp, h->D.aup, h->n3 * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(h->D.avpp, h->D.avp, h->n3 * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  }
  {
    Prof p(h, "readyc_3d");
    launch_readyc3d(h->D, h->stream);
  }
  h->D.ab3_mode = 0;
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
    e = launch_trop_fast(h->D, h->trop_tx, h->trop_ty, h->trop_epoch, h->stream);
    h->trop_epoch += (unsigned long long)h->D.nstep * (unsigned long long)h->trop_blocks;
  } else {
    e = launch_trop(h->D, h->trop_tx, h->trop_ty, h->trop_blocks, h->stream);
  }
  if (e != cudaSuccess) return fail(PCOM_ERR_CUDA, "barotropic kernel launch: %s", cudaGetErrorString(e));
  h->n_ch++;
  return PCOM_OK;
}
int do_clin(pcom_handle *h) {
  {
    Prof p(h, "clin_2d");
    launch_uv2d(h->D, 2, h->stream);
  }
  {
    Prof p(h, "int_clin");
    launch_clin(h->D, h->stream);
  }
  {
    Prof p(h, "smag");
    launch_smag(h->D, h->stream);
  }
  h->n_uv++;
  return PCOM_OK;
}
int do_ssh(pcom_handle *h) {
  Prof p(h, "int_ssh");
  launch_ssh(h->D, h->stream);
  h->n_ssh++;
  return PCOM_OK;
}
int do_ts(pcom_handle *h) {
  {
    Prof p(h, "ts_2d");
    launch_uv2d(h->D, 1, h->stream);
  }
  {
    Prof p(h, "upwelling+acw");
    launch_upwelling(h->D, 1, h->stream);
  }
  h->n_w++;
  {
    Prof p(h, "int_ts");
    launch_ts(h->D, h->stream);
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
  case 2: return do_readyc(h, iter);
  case 3: return do_trop(h);
  case 4: return do_clin(h);
  case 5: return do_ssh(h);
  case 6: return do_ts(h);
  default: return fail(PCOM_ERR_ARG, "unknown phase %d", phase);
  }
}

int enqueue_step(pcom_handle *h, int64_t iter) {
  if (!h) return fail(PCOM_ERR_ARG, "null handle");
  if (!h->static_ok) return fail(PCOM_ERR_STATE, "step before pcom_gpu_upload_static");
  if (iter < 1) return fail(PCOM_ERR_ARG, "tctr_i must be >= 1");
  for (int ph = 0; ph <= 6; ++ph) {
    int rc = run_phase(h, ph, iter);
    if (rc) return rc;
  }
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

struct Named {
  const double *p;
  long long n;
};

Named lookup(pcom_handle *h, const std::string &s) {
  Dev &D = h->D;
  const long long n2 = h->n2, n3 = h->n3, n3p = h->n3p;
  static const char *b4[4] = {"xn", "xs", "ye", "yw"};
  for (int q = 0; q < 4; ++q) {
    if (s == std::string("bphi_") + b4[q]) return {D.bphi[q], n2};
    if (s == std::string("bgraphi_") + b4[q]) return {D.bgra[q], n2};
  }
  const std::map<std::string, Named> m = {
      {"tc", {D.tc, n3}},     {"sc", {D.sc, n3}},       {"tp", {D.tp, n3}},     {"sp", {D.sp, n3}},
      {"uc", {D.uc, n3}},     {"vc", {D.vc, n3}},       {"up", {D.up, n3}},     {"vp", {D.vp, n3}},
      {"auc", {D.auc, n3}},   {"aup", {D.aup, n3}},     {"aupp", {D.aupp, n3}}, {"avc", {D.avc, n3}},
      {"avp", {D.avp, n3}},   {"avpp", {D.avpp, n3}},   {"ubc", {D.ubc, n2}},   {"vbc", {D.vbc, n2}},
      {"ubp", {D.ubp, n2}},   {"vbp", {D.vbp, n2}},     {"chc", {D.chc, n2}},   {"chp", {D.chp, n2}},
      {"mch", {D.mch, n2}},   {"mch2", {D.mch2, n2}},   {"am", {D.am, n3}},     {"alpha", {D.alpha, n3}},
      {"adp", {D.adp, n3}},   {"wm", {D.wm, n3p}},      {"prho", {(const double *)D.prho, 2 * n3}},
      {"fx", {D.fx, n3}},     {"fy", {D.fy, n3}},       {"pax", {D.pax, n2}},   {"pay", {D.pay, n2}},
      {"ut", {D.ut, n2}},     {"vt", {D.vt, n2}},       {"act", {D.act, n3}},   {"acs", {D.acs, n3}},
      {"acr", {D.acr, n3}},   {"acu", {D.acu, n3}},     {"acv", {D.acv, n3}},   {"acw", {D.acw, n3}},
      {"acch", {D.acch, n2}}, {"acssh", {D.acssh, n2}}, {"km", {D.km, n3p}},    {"kh", {D.kh, n3p}},
      {"cor", {D.cor, n2}},   {"cv1", {D.cv1, n2}},     {"cv2", {D.cv2, n2}},   {"graphihx", {D.graphihx, n2}},
      {"graphihy", {D.graphihy, n2}}, {"sch_r", {D.sch_r, n2}}, {"sch_w", {D.sch_w, n2}},
      {"bnd_taux", {D.taux, n2}}, {"bnd_tauy", {D.tauy, n2}}, {"bnd_t", {D.bnd_t, n2}}, {"bnd_s", {D.bnd_s, n2}},
      {"bnd_pa", {D.bnd_pa, n2}}, {"uu", {D.uu, n3}}, {"vv", {D.vv, n3}}};
  auto it = m.find(s);
  if (it == m.end()) return {nullptr, 0};
  return it->second;
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
  if ((d.flags & PCOM_PREC_MIXED) != 0) return fail(PCOM_ERR_ARG, "mixed precision is not built into this handle type");
  pcom_handle *h = new pcom_handle();
  h->dims = d;
  h->ni = d.ni; h->nj = d.nj; h->nk = d.nk; h->nkp = d.nk + 1;
  h->n2 = (long long)d.ni * d.nj;
  h->n3 = h->n2 * d.nk;
  h->n3p = h->n2 * (d.nk + 1);
  cudaGetDevice(&h->device);
  cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { delete h; return fail(PCOM_ERR_CUDA, "stream: %s", cudaGetErrorString(e)); }
  h->own_stream = true;
  Dev &D = h->D;
  D.ni = d.ni; D.nj = d.nj; D.nk = d.nk; D.nkp = d.nk + 1; D.nim = d.ni - 1; D.njm = d.nj - 1;
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
  A(&p, n3p); D.km = p; A(&p, n3p); D.kh = p;
  A(&p, n2); D.taux = p; A(&p, n2); D.tauy = p; A(&p, n2); D.bnd_t = p; A(&p, n2); D.bnd_s = p; A(&p, n2); D.bnd_pa = p;
  for (int q = 0; q < 3; ++q) { A(&h->t_pool[q], n3); A(&h->s_pool[q], n3); A(&h->ab_u[q], n3); A(&h->ab_v[q], n3); }
  A(&D.uc, n3); A(&D.vc, n3); A(&D.up, n3); A(&D.vp, n3);
  A(&D.ubc, n2); A(&D.vbc, n2); A(&D.ubp, n2); A(&D.vbp, n2);
  A(&D.chc, n2); A(&D.chp, n2); A(&D.mch, n2); A(&D.mch2, n2);
  A(&D.am, n3); A(&D.alpha, n3); A(&D.adp, n3); A(&D.wm, n3p);
  {
    double2 *pr = nullptr;
    if (!rc) rc = h->alloc(&pr, (size_t)n3);
    D.prho = pr;
  }
  A(&D.fx, n3); A(&D.fy, n3); A(&D.pax, n2); A(&D.pay, n2); A(&D.ut, n2); A(&D.vt, n2);
  for (int q = 0; q < 4; ++q) { A(&D.bphi[q], n2); A(&D.bgra[q], n2); }
  A(&D.sch_r, n2); A(&D.sch_w, n2); A(&D.uu, n3); A(&D.vv, n3);
  A(&D.act, n3); A(&D.acs, n3); A(&D.acr, n3); A(&D.acu, n3); A(&D.acv, n3); A(&D.acw, n3);
  A(&D.acch, n2); A(&D.acssh, n2);
  for (int q = 0; q < 2; ++q) { A(&D.tr_ch[q], n2); A(&D.tr_ub[q], n2); A(&D.tr_vb[q], n2); }
  for (int q = 0; q < 6; ++q) A(&D.tr_acc[q], n2);
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
    cudaMemcpy(D.alpha, v.data(), n3 * sizeof(double), cudaMemcpyHostToDevice);
    std::fill(v.begin(), v.end(), LIT(1.0e3));
    cudaMemcpy(D.am, v.data(), n3 * sizeof(double), cudaMemcpyHostToDevice);
    std::vector<double> one((size_t)n2, 1.0);
    for (double *c : {D.chc, D.chp, D.mch, D.mch2}) cudaMemcpy(c, one.data(), n2 * sizeof(double), cudaMemcpyHostToDevice);
  }
  h->itc = h->itp = 0;
  h->ic = 0; h->ip = 1; h->ipp = 2;
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
  CK(cudaMemcpy((void *)D.km, s->km, h->n3p * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy((void *)D.kh, s->kh, h->n3p * sizeof(double), cudaMemcpyHostToDevice));
  if (!s->pr2 || !s->dpr2 || !s->dz1) return fail(PCOM_ERR_ARG, "vertical grid missing");
  for (int k = 1; k <= nk; ++k) { D.pr2[k] = s->pr2[k - 1]; D.dpr2[k] = s->dpr2[k - 1]; D.rdpr2[k] = 1.0 / s->dpr2[k - 1]; }
  for (int k = 1; k <= nkp; ++k) { D.dz1[k] = s->dz1[k - 1]; D.rdz1[k] = 1.0 / s->dz1[k - 1]; }
  (void)ni; (void)nj;
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
      CK(cudaMemcpyAsync(h->t_pool[fr], h->t_pool[h->itc], n3 * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
      CK(cudaMemcpyAsync(h->s_pool[fr], h->s_pool[h->itc], n3 * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
      h->itp = fr;
      bind_rotating(h);
    }
  }
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
  const long long n2 = h->n2, n3 = h->n3;
  Dev &D = h->D;
  int rc = 0;
  auto out = [&](double *dst, const double *src, long long n) { if (!rc) rc = copy_out(h, dst, src, n); };
  out(s->tc, D.tc, n3); out(s->sc, D.sc, n3); out(s->tp, D.tp, n3); out(s->sp, D.sp, n3);
  out(s->uc, D.uc, n3); out(s->vc, D.vc, n3); out(s->up, D.up, n3); out(s->vp, D.vp, n3);
  out(s->auc, D.auc, n3); out(s->aup, D.aup, n3); out(s->aupp, D.aupp, n3);
  out(s->avc, D.avc, n3); out(s->avp, D.avp, n3); out(s->avpp, D.avpp, n3);
  out(s->ubc, D.ubc, n2); out(s->vbc, D.vbc, n2); out(s->ubp, D.ubp, n2); out(s->vbp, D.vbp, n2);
  out(s->chc, D.chc, n2); out(s->chp, D.chp, n2); out(s->mch, D.mch, n2); out(s->mch2, D.mch2, n2);
  out(s->am, D.am, n3); out(s->prho, (const double *)D.prho, 2 * n3);
  out(s->alpha, D.alpha, n3); out(s->adp, D.adp, n3); out(s->wm, D.wm, h->n3p);
  if (rc) return rc;
  return sync_check(h);
}

int pcom_gpu_set_forcing(pcom_handle *h, const pcom_forcing *f) {
  if (!h || !f) return fail(PCOM_ERR_ARG, "null argument");
  const long long n2 = h->n2;
  Dev &D = h->D;
  int rc = 0;
  auto in = [&](const double *dst, const double *src) { if (!rc) rc = copy_in(h, (double *)dst, src, n2); };
  in(D.taux, f->taux); in(D.tauy, f->tauy); in(D.bnd_t, f->t); in(D.bnd_s, f->s); in(D.bnd_pa, f->pa);
  return rc;
}

int pcom_gpu_get_accum(pcom_handle *h, pcom_accum *a) {
  if (!h || !a) return fail(PCOM_ERR_ARG, "null argument");
  const long long n2 = h->n2, n3 = h->n3;
  Dev &D = h->D;
  int rc = 0;
  auto out = [&](double *dst, const double *src, long long n) { if (!rc) rc = copy_out(h, dst, src, n); };
  out(a->act, D.act, n3); out(a->acs, D.acs, n3); out(a->acr, D.acr, n3);
  out(a->acu, D.acu, n3); out(a->acv, D.acv, n3); out(a->acw, D.acw, n3);
  out(a->acch, D.acch, n2); out(a->acssh, D.acssh, n2);
  a->n_ts = h->n_ts; a->n_uv = h->n_uv; a->n_w = h->n_w; a->n_ch = h->n_ch; a->n_ssh = h->n_ssh;
  if (rc) return rc;
  return sync_check(h);
}

int pcom_gpu_reset_accum(pcom_handle *h) {
  if (!h) return fail(PCOM_ERR_ARG, "null handle");
  Dev &D = h->D;
  for (double *p : {D.act, D.acs, D.acr, D.acu, D.acv, D.acw})
    CK(cudaMemsetAsync(p, 0, h->n3 * sizeof(double), h->stream));
  for (double *p : {D.acch, D.acssh}) CK(cudaMemsetAsync(p, 0, h->n2 * sizeof(double), h->stream));
  h->n_ts = h->n_uv = h->n_w = h->n_ch = h->n_ssh = 0;
  return sync_check(h);
}

int pcom_gpu_den_prho(pcom_handle *h) {
  if (!h) return fail(PCOM_ERR_ARG, "null handle");
  if (!h->static_ok) return fail(PCOM_ERR_STATE, "den_prho before pcom_gpu_upload_static");
  {
    Prof p(h, "den_prho");
    launch_den_prho(h->D, h->stream);
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
  if (!f.p) return fail(PCOM_ERR_ARG, "unknown field '%s'", name);
  if (n < f.n) return fail(PCOM_ERR_ARG, "buffer for '%s' holds %lld < %lld doubles", name, (long long)n, f.n);
  CK(cudaMemcpyAsync(host, f.p, f.n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  return sync_check(h);
}

int pcom_gpu_check_finite(pcom_handle *h) {
  if (!h) return fail(PCOM_ERR_ARG, "null handle");
  Dev &D = h->D;
  CK(cudaMemsetAsync(h->d_count, 0, sizeof(unsigned long long), h->stream));
  struct F { const double *p; const int *lev; int planes; } fs[] = {
      {D.tc, D.lev_t, h->nk}, {D.sc, D.lev_t, h->nk}, {D.uc, D.lev_u, h->nk}, {D.vc, D.lev_u, h->nk},
      {D.chc, D.lev_t, 1},    {D.ubc, D.lev_u, 1},    {D.vbc, D.lev_u, 1}};
  for (auto &f : fs) {
    Prof p(h, "watchdog");
    launch_nonfinite(f.p, f.lev, h->nk, h->n2, f.planes, h->d_count, h->stream);
  }
  unsigned long long c = 0;
  CK(cudaMemcpyAsync(&c, h->d_count, sizeof c, cudaMemcpyDeviceToHost, h->stream));
  int rc = sync_check(h);
  if (rc) return rc;
  if (c) return fail(PCOM_ERR_NUMERIC, "%llu non-finite wet values in the prognostic fields", c);
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
    cudaMemset(b->err, 0, sizeof(int));
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
  if (e == cudaSuccess) { b->allocs.push_back(b->err); e = cudaMemset(b->err, 0, sizeof(int)); }
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
  b->launches += 12 + (int64_t)b->groups.size();  // kernels of one batched step
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
