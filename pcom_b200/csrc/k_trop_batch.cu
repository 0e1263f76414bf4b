// k_trop_batch.cu -- the barotropic subcycle of int_trop (mod_int.f90:153-296)
// for a batch of domains (ensemble members and basins of uneven size) in ONE
// persistent cooperative launch.
//
// The tiles of every member form one work list; each CTA owns tiles of any
// member (possibly several) and, per substep, stages each tile's
// (TX+4) x (TY+4) region in shared memory and evaluates the same predictor /
// viscosity / pressure-gradient / Coriolis / corrector sequence as the
// single-domain kernel (same operation order, divisions by reciprocals), then
// all CTAs meet at one grid barrier.  Static coefficients are read per point
// from the member's arrays (L2-resident); accumulators and the first
// substep's viscosity live in the member's 2-D scratch.  All members share
// dtbt and dtbc, so they take the same number of substeps.
#include <cuda/atomic>

#include "pcom_dev.cuh"
#include "pcom_kernels.h"

namespace {


enum {
  B_CH, B_UB, B_VB, B_S1, B_X2, B_PRED, B_SCHE,
  B_A1U, B_A1V, B_GY, B_CN, B_A2U, B_A2V, B_GX, B_CE,
  B_UBC, B_VBC,
  B_COUNT
};

__device__ __forceinline__ void prefetch_l2(const void *a) { asm volatile("prefetch.global.L2 [%0];" ::"l"(a)); }

__device__ bool batch_barrier(unsigned long long *cnt, unsigned long long want, int *err, unsigned long long limit_ns) {
  __syncthreads();
  __shared__ int s_fail;
  if (threadIdx.x == 0) {
    // release: cumulative over the CTA's writes ordered before it by bar.sync
    cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> c(*cnt);
    c.fetch_add(1ULL, cuda::memory_order_release);
    s_fail = wait_count(cnt, want, err, limit_ns) ? 0 : 1;
  }
  __syncthreads();
  return s_fail == 0;
}

}  // namespace

// SINGLE: every tile belongs to one domain, passed by value (P0, read through
// the constant cache); otherwise each tile's domain is Ps[tile.m].
// CTX, CTY > 0: compiled for one tile shape, so the region strides and the
// stage loops' point -> (lx, ly) divisions are constants; each stage walks
// the rectangle a full tile would cover and skips points outside its part
// of a partial tile.
// Threads per CTA: 512 for one domain (about 40 registers: a region point
// per thread for 32 x 10 tiles), 256 for a batch (more registers per thread).
template <bool SINGLE>
constexpr int batch_threads() { return SINGLE ? 512 : 256; }

template <bool SINGLE, int CTX = 0, int CTY = 0>
__global__ void __launch_bounds__(batch_threads<SINGLE>()) k_trop_batch(const __grid_constant__ Dev P0, const Dev *__restrict__ Ps,
                                                    const TileRef *__restrict__ tiles, int ntiles, int TX, int TY,
                                                    unsigned long long *cnt, int *err) {
  if (CTX > 0) { TX = CTX; TY = CTY; }
  extern __shared__ double sm[];
  const int W = TX + 4, RS = W * (TY + 4);
  const int tid = threadIdx.x, nth = blockDim.x;
  const int nstep = SINGLE ? P0.nstep : Ps[0].nstep;
  const unsigned long long wait_ns = SINGLE ? P0.wait_ns : Ps[0].wait_ns;
  auto S = [&](int f, int p) -> double & { return sm[f * RS + p]; };

  // accumulators of owned points (mod_int.f90:176-180)
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const TileRef T = tiles[t];
    const Dev &P = SINGLE ? P0 : Ps[T.m];
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
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
      const TileRef T = tiles[t];
      const Dev &P = SINGLE ? P0 : Ps[T.m];
      const int G = P.glo_ni, nj = P.nj, njm = P.njm, ni = P.ni;
      const int tw = T.tw, th = T.th, rr0 = T.r0 - 2, jj0 = T.j0 - 2;
      const double a = P.c.a, ra = P.ra, bt = (double)P.bt, gamma_b = P.c.gamma_b;
      const double *src_ch = (nt == 1) ? P.chp : P.tr_ch[1 - d];
      const double *src_ub = (nt == 1) ? P.ubp : P.tr_ub[1 - d];
      const double *src_vb = (nt == 1) ? P.vbp : P.tr_vb[1 - d];
      auto ring_i = [&](int r) { r %= G; if (r < 0) r += G; return r + 2; };
      // stage loop over the (TX + e) x (TY + e) rectangle from (lo_x, lo_y)
      // that a full tile's stage covers; region point -> (lx, ly, i, j, q),
      // points outside this tile's (tw + e) x (th + e) part and invalid rows
      // skipped
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
      // S1: previous state (L2 loads: written by other CTAs).  The 2-D
      // fields the later stages read at this point are prefetched into L2
      // (the substep's working set is larger than L2, so they would otherwise
      // come from HBM one stage at a time)
      STAGE(4) {
        PT(4, 0, 0)
        S(B_CH, p) = __ldcg(src_ch + q);
        if (lx < tw + 3 && ly < th + 3) { S(B_UB, p) = __ldcg(src_ub + q); S(B_VB, p) = __ldcg(src_vb + q); }
        prefetch_l2(P.lev_u + q); prefetch_l2(P.lev_t + q);
        prefetch_l2(P.prh_u + q); prefetch_l2(P.prh_t + q); prefetch_l2(P.rprh_t + q);
        prefetch_l2(P.am + q); prefetch_l2(P.rwt + q); prefetch_l2(P.cor + q);
        prefetch_l2(P.ut + q); prefetch_l2(P.vt + q); prefetch_l2(P.graphihx + q); prefetch_l2(P.graphihy + q);
        for (int f = 0; f < 4; ++f) { prefetch_l2(P.bphi[f] + q); prefetch_l2(P.bgra[f] + q); }
        for (int f = 0; f < 6; ++f) prefetch_l2(P.tr_acc[f] + q);
      }
      __syncthreads();
      // S2: sch = sqrt(ter(ch)) on U, supb
      STAGE(3) {
        PT(3, 0, 0)
        double sch = 1.0;
        if (__ldg(P.lev_u + q) > 0) {
          const double w = (j <= njm) ? (S(B_CH, p) + S(B_CH, p + W) + S(B_CH, p + 1) + S(B_CH, p + W + 1)) * 0.25 : 0.0;
          sch = sqrt(w);
        }
        const double ps = ld(P.prh_u, q) * sch;
        S(B_S1, p) = ps * S(B_UB, p);
        S(B_X2, p) = ps * S(B_VB, p) * __ldg(P.rh1d[3] + j - 1);
      }
      __syncthreads();
      // S4: predictor ch
      STAGE(2) {
        PT(2, 1, 1)
        const bool srow = j >= 2;
        const double tEc = srow ? 0.5 * (S(B_S1, p - W) + S(B_S1, p)) : 0.0;
        const double tEw = srow ? 0.5 * (S(B_S1, p - W - 1) + S(B_S1, p - 1)) : 0.0;
        const double A = dvr(tEc - tEw, __ldg(P.dxx1d[1] + i - 1), __ldg(P.rdxx1d[1] + i - 1));
        double B = 0.0;
        if (srow) {
          const double tNc = 0.5 * (S(B_X2, p - 1) + S(B_X2, p));
          const double tNs = 0.5 * (S(B_X2, p - W - 1) + S(B_X2, p - W));
          B = dvr(tNc - tNs, __ldg(P.dxy1d[1] + j - 1), __ldg(P.rdxy1d[1] + j - 1));
        }
        const double div = dvr(A + B, __ldg(P.arh1d[1] + j - 1), __ldg(P.rarh1d[1] + j - 1));
        double pred;
        if (__ldg(P.lev_t + q) > 0) pred = S(B_CH, p) - dvr(div * bt * gamma_b, ld(P.prh_t, q), ld(P.rprh_t, q));
        else pred = (nt == 1) ? P.chc[q] : S(B_CH, p);
        S(B_PRED, p) = pred;
      }
      __syncthreads();
      // S5: sch on U, N- and E-grid intermediates
      STAGE(2) {
        PT(2, 1, 1)
        const bool nrow = j <= njm, srow = j >= 2;
        const bool inU = lx < tw + 2 && ly < th + 2, inN = ly < th + 2, inE = lx < tw + 2;
        if (inU) {
          double sch = 1.0;
          if (__ldg(P.lev_u + q) > 0) {
            const double w = nrow ? (S(B_PRED, p) + S(B_PRED, p + W) + S(B_PRED, p + 1) + S(B_PRED, p + W + 1)) * 0.25 : 0.0;
            sch = sqrt(w);
          }
          S(B_SCHE, p) = sch;
        }
        if (inN) {
          const double dx4 = __ldg(P.dxx1d[4] + i - 1), rdx4 = __ldg(P.rdxx1d[4] + i - 1);
          const double rh4 = __ldg(P.rh1d[4] + j - 1), rrh4 = __ldg(P.rrh1d[4] + j - 1);
          S(B_A1U, p) = dvr(dvr(S(B_UB, p) - S(B_UB, p - 1), dx4, rdx4), rh4, rrh4);
          S(B_A1V, p) = dvr(dvr(S(B_VB, p) - S(B_VB, p - 1), dx4, rdx4), rh4, rrh4);
          if (nrow) {
            S(B_GY, p) = dvr(dvr(S(B_PRED, p + W) - S(B_PRED, p), __ldg(P.dxy1d[4] + j - 1), __ldg(P.rdxy1d[4] + j - 1)), a, ra);
            S(B_CN, p) = 0.5 * (S(B_PRED, p) + S(B_PRED, p + W));
          } else {
            S(B_GY, p) = 0.0;
            S(B_CN, p) = 0.0;
          }
        }
        if (inE) {
          const double rh2 = __ldg(P.rh1d[2] + j - 1);
          if (srow) {
            const double dy2 = __ldg(P.dxy1d[2] + j - 1), rdy2 = __ldg(P.rdxy1d[2] + j - 1);
            S(B_A2U, p) = dvr(S(B_UB, p) - S(B_UB, p - W), dy2, rdy2) * rh2;
            S(B_A2V, p) = dvr(S(B_VB, p) - S(B_VB, p - W), dy2, rdy2) * rh2;
          } else {
            S(B_A2U, p) = 0.0;
            S(B_A2V, p) = 0.0;
          }
          S(B_GX, p) = dvr(dvr(S(B_PRED, p + 1) - S(B_PRED, p), __ldg(P.dxx1d[2] + i - 1), __ldg(P.rdxx1d[2] + i - 1)),
                           __ldg(P.arh1d[2] + j - 1), __ldg(P.rarh1d[2] + j - 1));
          S(B_CE, p) = 0.5 * (S(B_PRED, p) + S(B_PRED, p + 1));
        }
      }
      __syncthreads();
      // S6: corrector velocity
      STAGE(1) {
        PT(1, 1, 1)
        const bool nrow = j <= njm;
        const double seau = (double)(__ldg(P.lev_u + q) >= 1);
        const double rh3 = __ldg(P.rh1d[3] + j - 1);
        const double dx3 = __ldg(P.dxx1d[3] + i - 1), rdx3 = __ldg(P.rdxx1d[3] + i - 1);
        const double dy3 = __ldg(P.dxy1d[3] + j - 1), rdy3 = __ldg(P.rdxy1d[3] + j - 1);
        const double aarh = __ldg(P.aarh3 + j - 1), raarh = __ldg(P.raarh3 + j - 1);
        const double L1u = dvr(S(B_A1U, p + 1) - S(B_A1U, p), dx3, rdx3);
        const double L1v = dvr(S(B_A1V, p + 1) - S(B_A1V, p), dx3, rdx3);
        const double L2u = nrow ? dvr(S(B_A2U, p + W) - S(B_A2U, p), dy3, rdy3) : 0.0;
        const double L2v = nrow ? dvr(S(B_A2V, p + W) - S(B_A2V, p), dy3, rdy3) : 0.0;
        const double sam1 = seau * ld(P.am, q);
        const double vsu = sam1 * dvr(L1u + L2u, aarh, raarh);
        const double vsv = sam1 * dvr(L1v + L2v, aarh, raarh);
        double dvu, dvv;
        if (nt == 1) {
          dvu = vsu - vsu;
          dvv = vsv - vsv;
          if (lx >= 2 && ly >= 2) { P.tr_acc[4][q] = vsu; P.tr_acc[5][q] = vsv; }
        } else {
          dvu = vsu - __ldcg(P.tr_acc[4] + q);
          dvv = vsv - __ldcg(P.tr_acc[5] + q);
        }
        double gi1 = 0.0, cg1 = 0.0;
        if (nrow) {
          gi1 = 0.5 * (S(B_GX, p) * ld(P.bphi[0], q) + S(B_GX, p + W) * ld(P.bphi[1], q + ni));
          cg1 = 0.5 * (S(B_CE, p) * ld(P.bgra[0], q) + S(B_CE, p + W) * ld(P.bgra[1], q + ni));
        }
        const double gi2 = 0.5 * (S(B_GY, p) * ld(P.bphi[2], q) + S(B_GY, p + 1) * ld(P.bphi[3], q + 1));
        const double cg2 = 0.5 * (S(B_CN, p) * ld(P.bgra[2], q) + S(B_CN, p + 1) * ld(P.bgra[3], q + 1));
        const double sch = S(B_SCHE, p);
        const double pg1 = (gi1 + cg1 + ld(P.graphihx, q)) * seau * sch;
        const double pg2 = (gi2 + cg2 + ld(P.graphihy, q)) * seau * sch;
        const double cor = ld(P.cor, q), ut = ld(P.ut, q), vt = ld(P.vt, q);
        const double ubp = S(B_UB, p), vbp = S(B_VB, p);
        double p1 = seau * (dvu + ut - pg1 + 0.5 * cor * vbp);
        double p2 = seau * (dvv + vt - pg2 - 0.5 * cor * ubp);
        const double w1 = p1 * bt + ubp, w2 = p2 * bt + vbp;
        const double cb = 0.5 * cor * bt;
        const double den = 1 + cb * cb, rden = ld(P.rwt, q);
        double u1 = dvr(w1 + 0.5 * cor * bt * w2, den, rden);
        double v1 = dvr(w2 - 0.5 * cor * bt * w1, den, rden);
        u1 = 0.5 * (u1 + ubp);
        v1 = 0.5 * (v1 + vbp);
        p1 = seau * (dvu - pg1 + ut + cor * v1);
        p2 = seau * (dvv - pg2 + vt - cor * u1);
        const double ubc = p1 * bt + ubp, vbc = p2 * bt + vbp;
        S(B_UBC, p) = ubc;
        S(B_VBC, p) = vbc;
        const double ps = ld(P.prh_u, q) * sch;
        S(B_S1, p) = ps * ubc;
        S(B_X2, p) = ps * vbc * rh3;
      }
      __syncthreads();
      // S8: corrector ch on the tile, store, accumulate
      STAGE(0) {
        PT(0, 2, 2)
        const bool srow = j >= 2;
        const double tEc = srow ? 0.5 * (S(B_S1, p - W) + S(B_S1, p)) : 0.0;
        const double tEw = srow ? 0.5 * (S(B_S1, p - W - 1) + S(B_S1, p - 1)) : 0.0;
        const double A = dvr(tEc - tEw, __ldg(P.dxx1d[1] + i - 1), __ldg(P.rdxx1d[1] + i - 1));
        double B = 0.0;
        if (srow) {
          const double tNc = 0.5 * (S(B_X2, p - 1) + S(B_X2, p));
          const double tNs = 0.5 * (S(B_X2, p - W - 1) + S(B_X2, p - W));
          B = dvr(tNc - tNs, __ldg(P.dxy1d[1] + j - 1), __ldg(P.rdxy1d[1] + j - 1));
        }
        const double div = dvr(A + B, __ldg(P.arh1d[1] + j - 1), __ldg(P.rarh1d[1] + j - 1));
        const double m1 = (double)(__ldg(P.lev_t + q) >= 1);
        const double chn = S(B_CH, p) - dvr(m1 * div * bt, ld(P.prh_t, q), ld(P.rprh_t, q));
        const double ubc = S(B_UBC, p), vbc = S(B_VBC, p);
        st2(P.tr_ch[d], P, i, q, chn);
        st2(P.tr_ub[d], P, i, q, ubc);
        st2(P.tr_vb[d], P, i, q, vbc);
        if (nt <= nstep / 2) P.tr_acc[0][q] = P.tr_acc[0][q] + chn;
        P.tr_acc[1][q] = P.tr_acc[1][q] + chn;
        P.tr_acc[2][q] = P.tr_acc[2][q] + ubc;
        P.tr_acc[3][q] = P.tr_acc[3][q] + vbc;
      }
#undef PT
#undef STAGE
      __syncthreads();
    }
    if (!batch_barrier(cnt, (unsigned long long)nt * gridDim.x, err, wait_ns)) return;
  }

  // averages (mod_int.f90:276-288)
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const TileRef T = tiles[t];
    const Dev &P = SINGLE ? P0 : Ps[T.m];
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
// the form for a tile shape: the fixed-shape one for the 32 x 10 tiles the
// single-domain selector uses (a 36 x 14 region: 504 of the 512 threads), the
// general one otherwise
template <bool SINGLE>
const void *batch_kernel(int TX, int TY) {
  if (SINGLE && TX == 32 && TY == 10) return (const void *)k_trop_batch<true, 32, 10>;
  return (const void *)k_trop_batch<SINGLE>;
}
}  // namespace

size_t trop_batch_smem(int TX, int TY) { return (size_t)B_COUNT * (TX + 4) * (TY + 4) * sizeof(double); }

// co-resident CTAs of the multi-tile kernel for a tile shape (the smaller of
// its single-domain and batched forms)
int trop_batch_max_blocks(int TX, int TY) {
  int dev = 0, nsm = 0, best = 1 << 30;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const size_t smem = trop_batch_smem(TX, TY);
  const void *fns[2] = {batch_kernel<true>(TX, TY), batch_kernel<false>(TX, TY)};
  const int nth[2] = {batch_threads<true>(), batch_threads<false>()};
  for (int f = 0; f < 2; ++f) {
    int per = 0;
    if (cudaFuncSetAttribute(fns[f], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fns[f], nth[f], smem) != cudaSuccess) return 0;
    best = per < best ? per : best;
  }
  return best * nsm;
}

namespace {
cudaError_t launch_batch_form(const void *fn, int nthreads, const Dev &P0, const Dev *dPs, const TileRef *dtiles,
                              int ntiles, int TX, int TY, int nblocks, unsigned long long *cnt, int *err,
                              cudaStream_t s) {
  const size_t smem = trop_batch_smem(TX, TY);
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  // the barrier counter starts from zero in every launch
  e = cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  void *args[] = {(void *)&P0, (void *)&dPs, (void *)&dtiles, (void *)&ntiles, (void *)&TX, (void *)&TY,
                  (void *)&cnt, (void *)&err};
  return cudaLaunchCooperativeKernel(fn, dim3(nblocks), dim3(nthreads), args, smem, s);
}
}  // namespace

cudaError_t launch_trop_batch(const Dev *dPs, const TileRef *dtiles, int ntiles, int TX, int TY, int nblocks,
                              unsigned long long *cnt, int *err, cudaStream_t s) {
  const Dev none{};
  return launch_batch_form(batch_kernel<false>(TX, TY), batch_threads<false>(), none, dPs, dtiles, ntiles, TX, TY,
                           nblocks, cnt, err, s);
}

cudaError_t launch_trop_multi(const Dev &P, const TileRef *dtiles, int ntiles, int TX, int TY, int nblocks,
                              unsigned long long *cnt, int *err, cudaStream_t s) {
  return launch_batch_form(batch_kernel<true>(TX, TY), batch_threads<true>(), P, nullptr, dtiles, ntiles, TX, TY,
                           nblocks, cnt, err, s);
}
