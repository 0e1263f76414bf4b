// k_trop_multi_mixed.cu -- the barotropic subcycle of int_trop
// (mod_int.f90:153-296) for mixed-precision handles whose domain is too
// large for the resident kernel (one tile per CTA): the multi-tile kernel's
// structure (several tiles per CTA, each tile's (TX+4) x (TY+4) region
// staged per substep, one grid barrier per substep) with the precision of
// the resident mixed kernel (k_trop_mixed.cu):
//
//   FP64: ch, the predictor, their means and differences (the bottom-
//         pressure gradient), ter(ch) x bgraphi + graphih, the ch update and
//         the ch / mch / mch2 / ub / vb accumulators;
//   FP32: ub, vb and the volume fluxes, divergence, viscosity, Coriolis
//         adjustment, sqrt(ter(ch)), divisions by FP32 reciprocals.
//
// The multi-tile kernel re-reads its coefficients from L2 or HBM every
// substep (a 0.25-degree domain's working set is larger than L2), so the
// bytes per substep set its pace.  Here, once per step, k_mm_prep writes the
// coefficients the FP32 arithmetic uses as FP32 copies (bphi with the
// reference's neighbour shifts applied, am x mask, cor, ut, vt, prh_u,
// 1/prh_t, the Coriolis denominator's reciprocal) and the two masks as one
// byte, and the velocities move between substeps as FP32: about a third
// fewer bytes per point and substep than the FP64 kernel.  The arithmetic
// per point follows k_trop_mixed operation by operation.
#include <cuda/atomic>

#include "pcom_dev.cuh"
#include "pcom_kernels.h"

namespace {

constexpr int kThreads = 512;
enum { D_CH, D_PRED, D_CN, D_CE, D_COUNT };  // FP64 region fields
enum {                                       // FP32 region fields
  F_UB, F_VB, F_S1, F_X2, F_SCHE, F_A1U, F_A1V, F_GY, F_A2U, F_A2V, F_GX, F_UBC, F_VBC,
  F_COUNT
};

__device__ __forceinline__ void prefetch_l2(const void *a) { asm volatile("prefetch.global.L2 [%0];" ::"l"(a)); }

__device__ bool grid_barrier(unsigned long long *cnt, unsigned long long want, int *err, unsigned long long limit_ns) {
  __syncthreads();
  __shared__ int s_fail;
  if (threadIdx.x == 0) {
    cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> c(*cnt);
    c.fetch_add(1ULL, cuda::memory_order_release);
    s_fail = wait_count(cnt, want, err, limit_ns) ? 0 : 1;
  }
  __syncthreads();
  return s_fail == 0;
}

// per-step FP32 coefficients and masks of every interior point
__global__ void k_mm_prep(const __grid_constant__ Dev P, MultiMixed M) {
  const long long n2 = P.n2;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n2; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % P.ni) + 1, j = (int)(q / P.ni) + 1;
    if (i < 2 || i > P.ni - 1) continue;
    const int levu = P.lev_u[q], levt = P.lev_t[q];
    const float seau = (float)(levu >= 1);
    const bool nrow = j <= P.njm;
    float *cf = M.cf;
    cf[MC_BXN * n2 + q] = (float)ld(P.bphi[0], q);
    cf[MC_BXS * n2 + q] = nrow ? (float)ld(P.bphi[1], q + P.ni) : 0.f;
    cf[MC_BYE * n2 + q] = (float)ld(P.bphi[2], q);
    cf[MC_BYW * n2 + q] = (float)ld(P.bphi[3], q + 1);
    cf[MC_SAM * n2 + q] = seau * (float)ld(P.am, q);
    cf[MC_COR * n2 + q] = (float)ld(P.cor, q);
    cf[MC_UT * n2 + q] = (float)ld(P.ut, q);
    cf[MC_VT * n2 + q] = (float)ld(P.vt, q);
    cf[MC_PRHU * n2 + q] = (float)ld(P.prh_u, q);
    cf[MC_RPRHT * n2 + q] = (float)ld(P.rprh_t, q);
    cf[MC_RDEN * n2 + q] = (float)ld(P.rwt, q);
    M.fl[q] = (unsigned char)((levu >= 1 ? 1 : 0) | (levt >= 1 ? 2 : 0));
  }
}

}  // namespace

template <int CTX = 0, int CTY = 0>
__global__ void __launch_bounds__(kThreads) k_trop_multi_mixed(const __grid_constant__ Dev P, const MultiMixed M,
                                                               const TileRef *__restrict__ tiles, int ntiles, int TX,
                                                               int TY, unsigned long long *cnt, int *err) {
  if (CTX > 0) { TX = CTX; TY = CTY; }
  extern __shared__ double smd[];
  const int W = TX + 4, RS = W * (TY + 4);
  float *smf = reinterpret_cast<float *>(smd + D_COUNT * RS);
  const int tid = threadIdx.x, nth = blockDim.x;
  const int nstep = P.nstep;
  const int G = P.glo_ni, nj = P.nj, njm = P.njm, ni = P.ni;
  const long long n2 = P.n2;
  const float ra = (float)P.ra, bt = (float)P.bt, gamma_b = (float)P.c.gamma_b;
  auto SD = [&](int f, int p) -> double & { return smd[f * RS + p]; };
  auto SF = [&](int f, int p) -> float & { return smf[f * RS + p]; };
  auto CF = [&](int f, long long q) { return __ldg(M.cf + f * n2 + q); };
  auto RDXX = [&](int g, int i) { return (float)ld(P.rdxx1d[g], i - 1); };
  auto RDXY = [&](int g, int j) { return (float)ld(P.rdxy1d[g], j - 1); };
  auto RH = [&](int g, int j) { return (float)ld(P.rh1d[g], j - 1); };

  // accumulators of owned points (mod_int.f90:176-180)
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const TileRef T = tiles[t];
    for (int p = tid; p < T.tw * T.th; p += nth) {
      const int i = T.r0 + p % T.tw + 2, j = T.j0 + p / T.tw;
      const long long q = I2(P, i, j);
      P.tr_acc[0][q] = P.chc[q];
      P.tr_acc[1][q] = P.chc[q];
      P.tr_acc[2][q] = P.ubc[q];
      P.tr_acc[3][q] = P.vbc[q];
    }
  }

  for (int nt = 1; nt <= nstep; ++nt) {
    const int d = (nt - 1) & 1;
    const double *src_ch = (nt == 1) ? P.chp : P.tr_ch[1 - d];
    // the velocity ping-pong, selected without indexing the parameter array
    const float *src_ub = d ? M.ub[0] : M.ub[1], *src_vb = d ? M.vb[0] : M.vb[1];
    float *dst_ub = d ? M.ub[1] : M.ub[0], *dst_vb = d ? M.vb[1] : M.vb[0];
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
      const TileRef T = tiles[t];
      const int tw = T.tw, th = T.th, rr0 = T.r0 - 2, jj0 = T.j0 - 2;
      auto ring_i = [&](int r) { r %= G; if (r < 0) r += G; return r + 2; };
#define STAGE(e) for (int pp = tid; pp < (TX + (e)) * (TY + (e)); pp += nth)
#define PT(e, lo_x, lo_y)                                                   \
  const int lx = (lo_x) + pp % (TX + (e)), ly = (lo_y) + pp / (TX + (e));   \
  if (lx >= (lo_x) + tw + (e) || ly >= (lo_y) + th + (e)) continue;         \
  const int j = jj0 + ly;                                                   \
  if (j < 1 || j > nj) continue;                                            \
  const int i = ring_i(rr0 + lx);                                           \
  const long long q = I2(P, i, j);                                          \
  const int p = ly * W + lx;                                                \
  (void)i;
      // S1: previous state; the coefficients the later stages read at this
      // point are prefetched into L2
      STAGE(4) {
        PT(4, 0, 0)
        SD(D_CH, p) = __ldcg(src_ch + q);
        if (lx < tw + 3 && ly < th + 3) {
          SF(F_UB, p) = nt == 1 ? (float)__ldcg(P.ubp + q) : __ldcg(src_ub + q);
          SF(F_VB, p) = nt == 1 ? (float)__ldcg(P.vbp + q) : __ldcg(src_vb + q);
        }
        if ((lx & 15) == 0) {
          for (int f = 0; f < MC_COUNT; ++f) prefetch_l2(M.cf + f * n2 + q);
          for (int f = 0; f < 4; ++f) prefetch_l2(P.bgra[f] + q);
          prefetch_l2(P.graphihx + q); prefetch_l2(P.graphihy + q);
          for (int f = 0; f < 4; ++f) prefetch_l2(P.tr_acc[f] + q);
        }
      }
      __syncthreads();
      // S2: fluxes prh_u sqrt(ter(ch)) (ub, vb rh3)
      STAGE(3) {
        PT(3, 0, 0)
        float sch = 1.f;
        if (__ldg(M.fl + q) & 1) {
          const double w = (j <= njm) ? (SD(D_CH, p) + SD(D_CH, p + W) + SD(D_CH, p + 1) + SD(D_CH, p + W + 1)) * 0.25 : 0.0;
          sch = sqrtf((float)w);
        }
        const float ps = CF(MC_PRHU, q) * sch;
        SF(F_S1, p) = ps * SF(F_UB, p);
        SF(F_X2, p) = ps * SF(F_VB, p) * RH(3, j);
      }
      __syncthreads();
      // S4: predictor ch
      STAGE(2) {
        PT(2, 1, 1)
        const bool srow = j >= 2;
        const float tEc = srow ? 0.5f * (SF(F_S1, p - W) + SF(F_S1, p)) : 0.f;
        const float tEw = srow ? 0.5f * (SF(F_S1, p - W - 1) + SF(F_S1, p - 1)) : 0.f;
        const float A = (tEc - tEw) * RDXX(1, i);
        float B = 0.f;
        if (srow) {
          const float tNc = 0.5f * (SF(F_X2, p - 1) + SF(F_X2, p));
          const float tNs = 0.5f * (SF(F_X2, p - W - 1) + SF(F_X2, p - W));
          B = (tNc - tNs) * RDXY(1, j);
        }
        const float div = (A + B) * (float)ld(P.rarh1d[1], j - 1);
        double pred;
        if (__ldg(M.fl + q) & 2) pred = SD(D_CH, p) - (double)(div * bt * gamma_b * CF(MC_RPRHT, q));
        else pred = (nt == 1) ? P.chc[q] : SD(D_CH, p);
        SD(D_PRED, p) = pred;
      }
      __syncthreads();
      // S5: sqrt(ter(pred)) on U; N- and E-grid intermediates
      STAGE(2) {
        PT(2, 1, 1)
        const bool nrow = j <= njm, srow = j >= 2;
        const bool inU = lx < tw + 2 && ly < th + 2, inN = ly < th + 2, inE = lx < tw + 2;
        if (inU) {
          float sch = 1.f;
          if (__ldg(M.fl + q) & 1) {
            const double w = nrow ? (SD(D_PRED, p) + SD(D_PRED, p + W) + SD(D_PRED, p + 1) + SD(D_PRED, p + W + 1)) * 0.25 : 0.0;
            sch = sqrtf((float)w);
          }
          SF(F_SCHE, p) = sch;
        }
        if (inN) {
          const float rdx4 = RDXX(4, i), rrh4 = (float)ld(P.rrh1d[4], j - 1);
          SF(F_A1U, p) = (SF(F_UB, p) - SF(F_UB, p - 1)) * rdx4 * rrh4;
          SF(F_A1V, p) = (SF(F_VB, p) - SF(F_VB, p - 1)) * rdx4 * rrh4;
          if (nrow) {
            SF(F_GY, p) = (float)(SD(D_PRED, p + W) - SD(D_PRED, p)) * RDXY(4, j) * ra;
            SD(D_CN, p) = 0.5 * (SD(D_PRED, p) + SD(D_PRED, p + W));
          } else {
            SF(F_GY, p) = 0.f;
            SD(D_CN, p) = 0.0;
          }
        }
        if (inE) {
          const float rh2 = RH(2, j);
          if (srow) {
            const float rdy2 = RDXY(2, j);
            SF(F_A2U, p) = (SF(F_UB, p) - SF(F_UB, p - W)) * rdy2 * rh2;
            SF(F_A2V, p) = (SF(F_VB, p) - SF(F_VB, p - W)) * rdy2 * rh2;
          } else {
            SF(F_A2U, p) = 0.f;
            SF(F_A2V, p) = 0.f;
          }
          SF(F_GX, p) = (float)(SD(D_PRED, p + 1) - SD(D_PRED, p)) * RDXX(2, i) * (float)ld(P.rarh1d[2], j - 1);
          SD(D_CE, p) = 0.5 * (SD(D_PRED, p) + SD(D_PRED, p + 1));
        }
      }
      __syncthreads();
      // S6: corrector velocity
      STAGE(1) {
        PT(1, 1, 1)
        const bool nrow = j <= njm;
        const float seau = (float)(__ldg(M.fl + q) & 1);
        const float rh3 = RH(3, j), rdx3 = RDXX(3, i), rdy3 = RDXY(3, j), raarh = (float)ld(P.raarh3, j - 1);
        const float L1u = (SF(F_A1U, p + 1) - SF(F_A1U, p)) * rdx3;
        const float L1v = (SF(F_A1V, p + 1) - SF(F_A1V, p)) * rdx3;
        const float L2u = nrow ? (SF(F_A2U, p + W) - SF(F_A2U, p)) * rdy3 : 0.f;
        const float L2v = nrow ? (SF(F_A2V, p + W) - SF(F_A2V, p)) * rdy3 : 0.f;
        const float sam1 = CF(MC_SAM, q);
        const float vsu = sam1 * ((L1u + L2u) * raarh);
        const float vsv = sam1 * ((L1v + L2v) * raarh);
        float dvu, dvv;
        if (nt == 1) {
          dvu = vsu - vsu;
          dvv = vsv - vsv;
          if (lx >= 2 && ly >= 2) { M.vs0[0][q] = vsu; M.vs0[1][q] = vsv; }
        } else {
          dvu = vsu - __ldcg(M.vs0[0] + q);
          dvv = vsv - __ldcg(M.vs0[1] + q);
        }
        float gi1 = 0.f;
        double cg1 = 0.0;
        if (nrow) {
          gi1 = 0.5f * (SF(F_GX, p) * CF(MC_BXN, q) + SF(F_GX, p + W) * CF(MC_BXS, q));
          cg1 = 0.5 * (SD(D_CE, p) * ld(P.bgra[0], q) + SD(D_CE, p + W) * ld(P.bgra[1], q + ni));
        }
        const float gi2 = 0.5f * (SF(F_GY, p) * CF(MC_BYE, q) + SF(F_GY, p + 1) * CF(MC_BYW, q));
        const double cg2 = 0.5 * (SD(D_CN, p) * ld(P.bgra[2], q) + SD(D_CN, p + 1) * ld(P.bgra[3], q + 1));
        const float sch = SF(F_SCHE, p);
        const float pg1 = (float)((double)gi1 + cg1 + ld(P.graphihx, q)) * seau * sch;
        const float pg2 = (float)((double)gi2 + cg2 + ld(P.graphihy, q)) * seau * sch;
        const float cor = CF(MC_COR, q), ut = CF(MC_UT, q), vt = CF(MC_VT, q), rden = CF(MC_RDEN, q);
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
        const float ps = CF(MC_PRHU, q) * sch;
        SF(F_S1, p) = ps * ubc;
        SF(F_X2, p) = ps * vbc * rh3;
      }
      __syncthreads();
      // S8: corrector ch on the tile, store, accumulate
      STAGE(0) {
        PT(0, 2, 2)
        const bool srow = j >= 2;
        const float tEc = srow ? 0.5f * (SF(F_S1, p - W) + SF(F_S1, p)) : 0.f;
        const float tEw = srow ? 0.5f * (SF(F_S1, p - W - 1) + SF(F_S1, p - 1)) : 0.f;
        const float A = (tEc - tEw) * RDXX(1, i);
        float B = 0.f;
        if (srow) {
          const float tNc = 0.5f * (SF(F_X2, p - 1) + SF(F_X2, p));
          const float tNs = 0.5f * (SF(F_X2, p - W - 1) + SF(F_X2, p - W));
          B = (tNc - tNs) * RDXY(1, j);
        }
        const float div = (A + B) * (float)ld(P.rarh1d[1], j - 1);
        const float mskt1 = (float)((__ldg(M.fl + q) >> 1) & 1);
        const double chn = SD(D_CH, p) - (double)(mskt1 * div * bt * CF(MC_RPRHT, q));
        const float ubc = SF(F_UBC, p), vbc = SF(F_VBC, p);
        st2(P.tr_ch[d], P, i, q, chn);
        dst_ub[q] = ubc;
        dst_vb[q] = vbc;
        if (nt <= nstep / 2) P.tr_acc[0][q] = P.tr_acc[0][q] + chn;
        P.tr_acc[1][q] = P.tr_acc[1][q] + chn;
        P.tr_acc[2][q] = P.tr_acc[2][q] + (double)ubc;
        P.tr_acc[3][q] = P.tr_acc[3][q] + (double)vbc;
      }
#undef PT
#undef STAGE
      __syncthreads();
    }
    if (!grid_barrier(cnt, (unsigned long long)nt * gridDim.x, err, P.wait_ns)) return;
  }

  // averages (mod_int.f90:276-288)
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const TileRef T = tiles[t];
    for (int p = tid; p < T.tw * T.th; p += nth) {
      const int i = T.r0 + p % T.tw + 2, j = T.j0 + p / T.tw;
      const long long q = I2(P, i, j);
      const double ub = P.tr_acc[2][q] / (nstep + 1), vb = P.tr_acc[3][q] / (nstep + 1);
      const double mch = P.tr_acc[0][q] / (nstep / 2 + 1), mch2 = P.tr_acc[1][q] / (nstep + 1);
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
  }
}

namespace {
// the fixed-shape form for the 32 x 10 tiles the single-domain multi-tile
// path uses
const void *mm_kernel(int TX, int TY) {
  if (TX == 32 && TY == 10) return (const void *)k_trop_multi_mixed<32, 10>;
  return (const void *)k_trop_multi_mixed<>;
}
}  // namespace

size_t trop_multi_mixed_smem(int TX, int TY) {
  const size_t rs = (size_t)(TX + 4) * (TY + 4);
  return D_COUNT * rs * sizeof(double) + F_COUNT * rs * sizeof(float);
}

size_t trop_multi_mixed_scratch_bytes(long long n2) {
  return (size_t)n2 * ((MC_COUNT + 4 + 2) * sizeof(float) + 1);
}

void trop_multi_mixed_bind(MultiMixed &M, void *scratch, long long n2) {
  float *f = (float *)scratch;
  M.cf = f;
  f += MC_COUNT * n2;
  for (int q = 0; q < 2; ++q) {
    M.ub[q] = f; f += n2;
    M.vb[q] = f; f += n2;
  }
  M.vs0[0] = f; f += n2;
  M.vs0[1] = f; f += n2;
  M.fl = (unsigned char *)f;
}

int trop_multi_mixed_max_blocks(int TX, int TY) {
  int dev = 0, nsm = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const size_t smem = trop_multi_mixed_smem(TX, TY);
  const void *fn = mm_kernel(TX, TY);
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, kThreads, smem) != cudaSuccess) return 0;
  return per * nsm;
}

cudaError_t launch_trop_multi_mixed(const Dev &P, const MultiMixed &M, const TileRef *dtiles, int ntiles, int TX,
                                    int TY, int nblocks, unsigned long long *cnt, int *err, cudaStream_t s) {
  k_mm_prep<<<592, 256, 0, s>>>(P, M);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const size_t smem = trop_multi_mixed_smem(TX, TY);
  const void *fn = mm_kernel(TX, TY);
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  // the barrier counter starts from zero in every launch
  e = cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  void *args[] = {(void *)&P, (void *)&M, (void *)&dtiles, (void *)&ntiles, (void *)&TX, (void *)&TY, (void *)&cnt,
                  (void *)&err};
  return cudaLaunchCooperativeKernel(fn, dim3(nblocks), dim3(kThreads), args, smem, s);
}
