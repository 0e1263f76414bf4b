// k_trop_mixed.cu -- the barotropic subcycle of int_trop (mod_int.f90:153-296)
// for the mixed-precision path: the resident kernel of k_trop.cu (one tile
// per CTA, one region point per thread, coefficients in registers, grid
// barrier between substeps) with FP32 arithmetic wherever it does not decide
// the bottom pressure:
//
//   FP64: ch, the predictor ch, their 4-point means, every difference of
//         them (the bottom-pressure gradient), ter(ch) x bgraphi + graphih
//         (two large terms that nearly cancel), the ch update, and the
//         ch / mch / mch2 / ub / vb accumulators;
//   FP32: ub, vb and the volume fluxes, divergence, viscosity, Coriolis
//         adjustment, sqrt(ter(ch)), divisions (by FP32 reciprocals).
//
// The 2-D buffers it shares with the FP64 path stay FP64 in memory.
#include <cuda/atomic>

#include "pcom_dev.cuh"
#include "pcom_kernels.h"

namespace {

constexpr int kThreads = 640;

enum { D_CH, D_PRED, D_CN, D_CE, D_COUNT };  // FP64 region fields
enum {                                       // FP32 region fields
  F_UB, F_VB, F_S1, F_X2, F_SCHE, F_A1U, F_A1V, F_GY, F_A2U, F_A2V, F_GX, F_UBC, F_VBC,
  F_COUNT
};
constexpr int kVx = 8, kVy = 19;  // FP32 metric vectors over lx and ly

}  // namespace

// CTX, CTY > 0: compiled for one tile shape (constant region strides, as in
// k_trop_fast); CTX = CTY = 0: any shape
template <int CTX = 0, int CTY = 0>
__global__ void __launch_bounds__(kThreads, 1)
    k_trop_mixed(const __grid_constant__ Dev P, int TX, int TY, int ntx, unsigned long long epoch) {
  if (CTX > 0) { TX = CTX; TY = CTY; }
  extern __shared__ double smd[];
  __shared__ int s_stop;
  const int nj = P.nj, njm = P.njm, ni = P.ni, G = P.glo_ni;
  const int W = TX + 4, H = TY + 4, RS = W * H;
  float *smf = reinterpret_cast<float *>(smd + D_COUNT * RS);
  float *vx = smf + F_COUNT * RS;
  float *vy = vx + kVx * W;
  const float a = (float)P.c.a, ra = (float)P.ra, bt = (float)P.bt, gamma_b = (float)P.c.gamma_b;
  const double btd = (double)P.bt;
  const int nstep = P.nstep;
  const int tid = threadIdx.x;
  const int tx = blockIdx.x % ntx, ty = blockIdx.x / ntx;
  const int R0 = tx * TX, J0 = ty * TY + 1;
  const int tw = min(TX, G - R0), th = min(TY, nj - J0 + 1);
  const int rr0 = R0 - 2, jj0 = J0 - 2;
  auto ring_i = [&](int r) { r %= G; if (r < 0) r += G; return r + 2; };
  auto SD = [&](int f, int p) -> double & { return smd[f * RS + p]; };
  auto SF = [&](int f, int p) -> float & { return smf[f * RS + p]; };

  for (int l = tid; l < W; l += blockDim.x) {
    const int i = ring_i(rr0 + l);
    for (int g = 1; g <= 4; ++g) {
      vx[(g - 1) * W + l] = (float)ld(P.dxx1d[g], i - 1);
      vx[(4 + g - 1) * W + l] = (float)ld(P.rdxx1d[g], i - 1);
    }
  }
  for (int l = tid; l < H; l += blockDim.x) {
    const int j = jj0 + l;
    if (j < 1 || j > nj) continue;
    for (int g = 1; g <= 4; ++g) {
      vy[(g - 1) * H + l] = (float)ld(P.dxy1d[g], j - 1);
      vy[(4 + g - 1) * H + l] = (float)ld(P.rdxy1d[g], j - 1);
      vy[(8 + g - 1) * H + l] = (float)ld(P.rh1d[g], j - 1);
    }
    vy[12 * H + l] = (float)ld(P.arh1d[1], j - 1);
    vy[13 * H + l] = (float)ld(P.rarh1d[1], j - 1);
    vy[14 * H + l] = (float)ld(P.arh1d[2], j - 1);
    vy[15 * H + l] = (float)ld(P.rarh1d[2], j - 1);
    vy[16 * H + l] = (float)ld(P.rrh1d[4], j - 1);
    vy[17 * H + l] = (float)ld(P.aarh3, j - 1);
    vy[18 * H + l] = (float)ld(P.raarh3, j - 1);
  }
  auto RDXX = [&](int g, int lx) { return vx[(4 + g - 1) * W + lx]; };
  auto RDXY = [&](int g, int ly) { return vy[(4 + g - 1) * H + ly]; };
  auto RH = [&](int g, int ly) { return vy[(8 + g - 1) * H + ly]; };

  const int p = tid;
  const int lx = p % W, ly = p / W;
  const int j = jj0 + ly;
  const bool active = p < RS && j >= 1 && j <= nj;
  const int i = active ? ring_i(rr0 + lx) : 2;
  const long long q = active ? I2(P, i, j) : 0;
  const bool nrow = j <= njm, srow = j >= 2;
  const bool inS2 = active && lx < tw + 3 && ly < th + 3;
  const bool inS4 = active && lx >= 1 && lx < tw + 3 && ly >= 1 && ly < th + 3;
  const bool inS6 = active && lx >= 1 && lx < tw + 2 && ly >= 1 && ly < th + 2;
  const bool inN = active && lx >= 1 && lx < tw + 3 && ly >= 1 && ly < th + 2;
  const bool inE = active && lx >= 1 && lx < tw + 2 && ly >= 1 && ly < th + 3;
  const bool inS8 = active && lx >= 2 && lx < tw + 2 && ly >= 2 && ly < th + 2;
  const int levu = active ? __ldg(P.lev_u + q) : 0, levt = active ? __ldg(P.lev_t + q) : 0;
  const float seau = (float)(levu >= 1), mskt1 = (float)(levt >= 1);
  const float prh_u = active ? (float)ld(P.prh_u, q) : 1.f;
  const float rprh_t = active ? (float)ld(P.rprh_t, q) : 1.f;
  const float rden = active ? (float)ld(P.rwt, q) : 1.f;
  float sam1 = 0, bxn = 0, bxs = 0, bye = 0, byw = 0, cor = 0, ut = 0, vt = 0;
  double gxn = 0, gxs = 0, gye = 0, gyw = 0, ghx = 0, ghy = 0;
  if (inS6) {
    sam1 = seau * (float)ld(P.am, q);
    bxn = (float)ld(P.bphi[0], q); bye = (float)ld(P.bphi[2], q); byw = (float)ld(P.bphi[3], q + 1);
    gxn = ld(P.bgra[0], q); gye = ld(P.bgra[2], q); gyw = ld(P.bgra[3], q + 1);
    if (nrow) { bxs = (float)ld(P.bphi[1], q + ni); gxs = ld(P.bgra[1], q + ni); }
    ghx = ld(P.graphihx, q); ghy = ld(P.graphihy, q);
    cor = (float)ld(P.cor, q); ut = (float)ld(P.ut, q); vt = (float)ld(P.vt, q);
  }
  float vs0u = 0.f, vs0v = 0.f;
  double acc_m = 0, acc_m2 = 0, acc_u = 0, acc_v = 0;
  if (inS8) {
    acc_m = P.chc[q]; acc_m2 = acc_m;
    acc_u = P.ubc[q]; acc_v = P.vbc[q];
  }
  const double land_ch0 = inS4 ? P.chc[q] : 0.0;
  __syncthreads();

  for (int nt = 1; nt <= nstep; ++nt) {
    const int d = (nt - 1) & 1;
    const double *src_ch = (nt == 1) ? P.chp : P.tr_ch[1 - d];
    const double *src_ub = (nt == 1) ? P.ubp : P.tr_ub[1 - d];
    const double *src_vb = (nt == 1) ? P.vbp : P.tr_vb[1 - d];
    // S1: previous state (the tile's own points carry it in shared memory)
    if (active && (nt == 1 || !inS8)) {
      SD(D_CH, p) = __ldcg(src_ch + q);
      if (inS2) { SF(F_UB, p) = (float)__ldcg(src_ub + q); SF(F_VB, p) = (float)__ldcg(src_vb + q); }
    }
    __syncthreads();
    // S2: fluxes prh_u sqrt(ter(ch)) (ub, vb rh3)
    if (inS2) {
      float sch = 1.f;
      if (levu > 0) {
        const double w = nrow ? (SD(D_CH, p) + SD(D_CH, p + W) + SD(D_CH, p + 1) + SD(D_CH, p + W + 1)) * 0.25 : 0.0;
        sch = sqrtf((float)w);
      }
      const float ps = prh_u * sch;
      SF(F_S1, p) = ps * SF(F_UB, p);
      SF(F_X2, p) = ps * SF(F_VB, p) * RH(3, ly);
    }
    __syncthreads();
    // S4: predictor ch
    if (inS4) {
      const float tEc = srow ? 0.5f * (SF(F_S1, p - W) + SF(F_S1, p)) : 0.f;
      const float tEw = srow ? 0.5f * (SF(F_S1, p - W - 1) + SF(F_S1, p - 1)) : 0.f;
      const float A = (tEc - tEw) * RDXX(1, lx);
      float B = 0.f;
      if (srow) {
        const float tNc = 0.5f * (SF(F_X2, p - 1) + SF(F_X2, p));
        const float tNs = 0.5f * (SF(F_X2, p - W - 1) + SF(F_X2, p - W));
        B = (tNc - tNs) * RDXY(1, ly);
      }
      const float div = (A + B) * vy[13 * H + ly];
      double pred;
      if (levt > 0) pred = SD(D_CH, p) - (double)(div * bt * gamma_b * rprh_t);
      else pred = (nt == 1) ? land_ch0 : SD(D_CH, p);
      SD(D_PRED, p) = pred;
    }
    __syncthreads();
    // S5: sqrt(ter(pred)) on U; N- and E-grid intermediates
    if (inS6) {
      float sch = 1.f;
      if (levu > 0) {
        const double w = nrow ? (SD(D_PRED, p) + SD(D_PRED, p + W) + SD(D_PRED, p + 1) + SD(D_PRED, p + W + 1)) * 0.25 : 0.0;
        sch = sqrtf((float)w);
      }
      SF(F_SCHE, p) = sch;
    }
    if (inN) {
      const float rdx4 = RDXX(4, lx), rrh4 = vy[16 * H + ly];
      SF(F_A1U, p) = (SF(F_UB, p) - SF(F_UB, p - 1)) * rdx4 * rrh4;
      SF(F_A1V, p) = (SF(F_VB, p) - SF(F_VB, p - 1)) * rdx4 * rrh4;
      if (nrow) {
        SF(F_GY, p) = (float)(SD(D_PRED, p + W) - SD(D_PRED, p)) * RDXY(4, ly) * ra;
        SD(D_CN, p) = 0.5 * (SD(D_PRED, p) + SD(D_PRED, p + W));
      } else {
        SF(F_GY, p) = 0.f;
        SD(D_CN, p) = 0.0;
      }
    }
    if (inE) {
      const float rh2 = RH(2, ly);
      if (srow) {
        const float rdy2 = RDXY(2, ly);
        SF(F_A2U, p) = (SF(F_UB, p) - SF(F_UB, p - W)) * rdy2 * rh2;
        SF(F_A2V, p) = (SF(F_VB, p) - SF(F_VB, p - W)) * rdy2 * rh2;
      } else {
        SF(F_A2U, p) = 0.f;
        SF(F_A2V, p) = 0.f;
      }
      SF(F_GX, p) = (float)(SD(D_PRED, p + 1) - SD(D_PRED, p)) * RDXX(2, lx) * vy[15 * H + ly];
      SD(D_CE, p) = 0.5 * (SD(D_PRED, p) + SD(D_PRED, p + 1));
    }
    __syncthreads();
    // S6: corrector velocity
    if (inS6) {
      const float rh3 = RH(3, ly), rdx3 = RDXX(3, lx), rdy3 = RDXY(3, ly), raarh = vy[18 * H + ly];
      const float L1u = (SF(F_A1U, p + 1) - SF(F_A1U, p)) * rdx3;
      const float L1v = (SF(F_A1V, p + 1) - SF(F_A1V, p)) * rdx3;
      const float L2u = nrow ? (SF(F_A2U, p + W) - SF(F_A2U, p)) * rdy3 : 0.f;
      const float L2v = nrow ? (SF(F_A2V, p + W) - SF(F_A2V, p)) * rdy3 : 0.f;
      const float vsu = sam1 * ((L1u + L2u) * raarh);
      const float vsv = sam1 * ((L1v + L2v) * raarh);
      if (nt == 1) { vs0u = vsu; vs0v = vsv; }
      const float dvu = vsu - vs0u, dvv = vsv - vs0v;
      float gi1 = 0.f;
      double cg1 = 0.0;
      if (nrow) {
        gi1 = 0.5f * (SF(F_GX, p) * bxn + SF(F_GX, p + W) * bxs);
        cg1 = 0.5 * (SD(D_CE, p) * gxn + SD(D_CE, p + W) * gxs);
      }
      const float gi2 = 0.5f * (SF(F_GY, p) * bye + SF(F_GY, p + 1) * byw);
      const double cg2 = 0.5 * (SD(D_CN, p) * gye + SD(D_CN, p + 1) * gyw);
      const float sch = SF(F_SCHE, p);
      const float pg1 = (float)((double)gi1 + cg1 + ghx) * seau * sch;
      const float pg2 = (float)((double)gi2 + cg2 + ghy) * seau * sch;
      const float ubp = SF(F_UB, p), vbp = SF(F_VB, p);
      float p1 = seau * (dvu + ut - pg1 + 0.5f * cor * vbp);
      float p2 = seau * (dvv + vt - pg2 - 0.5f * cor * ubp);
      const float w1 = p1 * bt + ubp, w2 = p2 * bt + vbp;
      float u1 = (w1 + 0.5f * cor * bt * w2) * rden;
      float v1 = (w2 - 0.5f * cor * bt * w1) * rden;
      u1 = 0.5f * (u1 + ubp);
      v1 = 0.5f * (v1 + vbp);
      p1 = seau * (dvu - pg1 + ut + cor * v1);
      p2 = seau * (dvv - pg2 + vt - cor * u1);
      const float ubc = p1 * bt + ubp, vbc = p2 * bt + vbp;
      SF(F_UBC, p) = ubc;
      SF(F_VBC, p) = vbc;
      const float ps = prh_u * sch;
      SF(F_S1, p) = ps * ubc;
      SF(F_X2, p) = ps * vbc * rh3;
    }
    __syncthreads();
    // S8: corrector ch, store, accumulate
    if (inS8) {
      const float tEc = srow ? 0.5f * (SF(F_S1, p - W) + SF(F_S1, p)) : 0.f;
      const float tEw = srow ? 0.5f * (SF(F_S1, p - W - 1) + SF(F_S1, p - 1)) : 0.f;
      const float A = (tEc - tEw) * RDXX(1, lx);
      float B = 0.f;
      if (srow) {
        const float tNc = 0.5f * (SF(F_X2, p - 1) + SF(F_X2, p));
        const float tNs = 0.5f * (SF(F_X2, p - W - 1) + SF(F_X2, p - W));
        B = (tNc - tNs) * RDXY(1, ly);
      }
      const float div = (A + B) * vy[13 * H + ly];
      const double chn = SD(D_CH, p) - (double)(mskt1 * div * bt * rprh_t);
      const float ubc = SF(F_UBC, p), vbc = SF(F_VBC, p);
      st2(P.tr_ch[d], P, i, q, chn);
      st2(P.tr_ub[d], P, i, q, (double)ubc);
      st2(P.tr_vb[d], P, i, q, (double)vbc);
      SD(D_CH, p) = chn;
      SF(F_UB, p) = ubc;
      SF(F_VB, p) = vbc;
      if (nt <= nstep / 2) acc_m = acc_m + chn;
      acc_m2 = acc_m2 + chn;
      acc_u = acc_u + (double)ubc;
      acc_v = acc_v + (double)vbc;
    }
    // grid barrier (as in k_trop_fast): release-ordered arrival, bounded
    // acquire wait, outcome through shared memory
    __syncthreads();
    if (tid == 0) {
      cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> c(*P.tile_flag);
      c.fetch_add(1ULL, cuda::memory_order_release);
      const unsigned long long want = epoch + (unsigned long long)nt * gridDim.x;
      s_stop = wait_count(P.tile_flag, want, P.err, P.wait_ns) ? 0 : 1;
    }
    __syncthreads();
    if (s_stop) return;
  }
  if (inS8) {
    const double ub = acc_u / (nstep + 1), vb = acc_v / (nstep + 1);
    const double mch = acc_m / (nstep / 2 + 1), mch2 = acc_m2 / (nstep + 1);
    st2(P.ubc, P, i, q, ub);
    st2(P.vbc, P, i, q, vb);
    st2(P.ubp, P, i, q, ub);
    st2(P.vbp, P, i, q, vb);
    st2(P.mch, P, i, q, mch);
    st2(P.mch2, P, i, q, mch2);
    st2(P.chc, P, i, q, mch2);
    st2(P.chp, P, i, q, mch2);
    st2(P.acch, P, i, q, P.acch[q] + mch2);
  }
  (void)a;
  (void)btd;
}

namespace {
// the fixed-shape form for the 24 x 18 tiles of the 1-degree 360 x 160 domain
const void *mixed_kernel(int TX, int TY) {
  if (TX == 24 && TY == 18) return (const void *)k_trop_mixed<24, 18>;
  return (const void *)k_trop_mixed<>;
}
}  // namespace

size_t trop_mixed_smem_bytes(int TX, int TY) {
  const size_t rs = (size_t)(TX + 4) * (TY + 4);
  return D_COUNT * rs * sizeof(double) + (F_COUNT * rs + kVx * (TX + 4) + kVy * (TY + 4)) * sizeof(float);
}

int trop_mixed_max_blocks(int TX, int TY) {
  int dev = 0, nsm = 0, per = 0;
  if ((TX + 4) * (TY + 4) > kThreads) return 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const size_t smem = trop_mixed_smem_bytes(TX, TY);
  const void *fn = mixed_kernel(TX, TY);
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
  const int nthreads = ((TX + 4) * (TY + 4) + 31) / 32 * 32;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, nthreads, smem) != cudaSuccess) return 0;
  return per * nsm;
}

cudaError_t launch_trop_mixed(const Dev &P, int TX, int TY, unsigned long long epoch, cudaStream_t s) {
  const int ntx = (P.glo_ni + TX - 1) / TX, nty = (P.nj + TY - 1) / TY;
  const size_t smem = trop_mixed_smem_bytes(TX, TY);
  const void *fn = mixed_kernel(TX, TY);
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int nthreads = ((TX + 4) * (TY + 4) + 31) / 32 * 32;
  void *args[] = {(void *)&P, (void *)&TX, (void *)&TY, (void *)&ntx, (void *)&epoch};
  return cudaLaunchCooperativeKernel(fn, dim3(ntx * nty), dim3(nthreads), args, smem, s);
}
