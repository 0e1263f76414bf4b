// k_trop.cu -- the barotropic predictor/corrector subcycle of int_trop
// (mod_int.f90:153-296) as ONE persistent cooperative kernel.
//
// The 2-D domain (interior columns x all rows) is cut into TX x TY tiles.
// Each CTA owns tiles; for every substep it stages a (TX+4) x (TY+4) region of
// the previous substep's (ch, ub, vb) in shared memory, evaluates the
// predictor ch, the viscosity, the bottom-pressure gradient forces, the
// Coriolis-adjusted corrector velocity and the corrector ch for its tile
// (recomputing the 1-2 cell halo of intermediates instead of exchanging
// them), writes (ch, ub, vb) for the tile to a ping-pong buffer in L2, and
// meets the other CTAs at one grid barrier per substep.  The 120 substeps of
// a 3600 s / 60 s step therefore cost 120 grid barriers and no launches.
//
// The grid barrier is a counter/generation pair with a bounded spin: if a
// wait exceeds its iteration limit the kernel records PCOM_ERR_TIMEOUT in
// err[0] and every CTA returns at its next barrier.  The launch is
// cooperative, so all CTAs are co-resident and the limit is never reached in
// normal operation.
#include <cuda/atomic>
#include "pcom_dev.cuh"
#include "pcom_kernels.h"

namespace {

constexpr long long kSpinLimit = 1LL << 26;  // ~seconds with the nanosleep below

__device__ bool grid_barrier(const Dev &P, unsigned nblocks) {
  __syncthreads();
  __shared__ int s_fail;
  if (threadIdx.x == 0) {
    cuda::atomic_ref<unsigned, cuda::thread_scope_device> cnt(P.bar[0]);
    cuda::atomic_ref<unsigned, cuda::thread_scope_device> gen(P.bar[1]);
    cuda::atomic_ref<int, cuda::thread_scope_device> err(P.err[0]);
    int fail = err.load(cuda::memory_order_relaxed) != 0;
    if (!fail) {
      const unsigned g = gen.load(cuda::memory_order_acquire);
      const unsigned arrived = cnt.fetch_add(1u, cuda::memory_order_acq_rel);
      if (arrived == nblocks - 1) {
        cnt.store(0u, cuda::memory_order_relaxed);
        gen.fetch_add(1u, cuda::memory_order_release);
      } else {
        const unsigned long long t0 = global_ns();
        long long it = 0;
        while (gen.load(cuda::memory_order_acquire) == g) {
          if (++it > kSpinLimit || err.load(cuda::memory_order_relaxed) != 0 || global_ns() - t0 > P.wait_ns) {
            err.store(1, cuda::memory_order_relaxed);
            fail = 1;
            break;
          }
          if (it > 64) __nanosleep(64);
        }
      }
    }
    s_fail = fail;
  }
  __syncthreads();
  return s_fail == 0;
}

// field slots in shared memory
enum {
  F_CH, F_UB, F_VB,          // previous substep state (T, U, U)
  F_S1, F_X2,                // supb1, supb2*rh3 (U)
  F_TE, F_TN,                // ter to E / N of the above
  F_PRED,                    // predictor ch (T)
  F_SCHE,                    // sqrt(ter(pred)) (U)
  F_A1U, F_A1V, F_GY, F_CN,  // N-grid intermediates
  F_A2U, F_A2V, F_GX, F_CE,  // E-grid intermediates
  F_UBC, F_VBC, F_S1N, F_X2N, F_TEN, F_TNN,
  F_COUNT
};

}  // namespace

__global__ void __launch_bounds__(256, 1) k_trop(const __grid_constant__ Dev P, int TX, int TY, int ntx, int nty) {
  extern __shared__ double smem[];
  const int ni = P.ni, nj = P.nj, njm = P.njm, G = P.glo_ni;
  const int W = TX + 4, H = TY + 4, RS = W * H;
  const double a = P.c.a, bt = (double)P.bt, gamma_b = P.c.gamma_b;
  const int nstep = P.nstep;
  const int ntiles = ntx * nty;
  const unsigned nblocks = gridDim.x;
  const int tid = threadIdx.x, nth = blockDim.x;
  // accumulators and the first substep's viscosity live in 2-D scratch (one per point)
  double *A_mch = P.tr_acc[0], *A_mch2 = P.tr_acc[1], *A_ua = P.tr_acc[2], *A_va = P.tr_acc[3];
  double *VS0U = P.tr_acc[4], *VS0V = P.tr_acc[5];

  auto S = [&](int f, int lx, int ly) -> double & { return smem[f * RS + ly * W + lx]; };
  auto ring_i = [&](int r) { r %= G; if (r < 0) r += G; return r + 2; };

  // initialise accumulators for owned points: mch = mch2 = chc, ua = ubc, va = vbc
  for (int t = blockIdx.x; t < ntiles; t += nblocks) {
    const int tx = t % ntx, ty = t / ntx;
    const int R0 = tx * TX, J0 = ty * TY + 1;
    const int tw = min(TX, G - R0), th = min(TY, nj - J0 + 1);
    for (int p = tid; p < tw * th; p += nth) {
      const int i = R0 + (p % tw) + 2, j = J0 + p / tw;
      const long long q = I2(P, i, j);
      A_mch[q] = P.chc[q];
      A_mch2[q] = P.chc[q];
      A_ua[q] = P.ubc[q];
      A_va[q] = P.vbc[q];
    }
  }
  // (no barrier needed: accumulators are point-private)

  for (int nt = 1; nt <= nstep; ++nt) {
    const int d = (nt - 1) & 1;
    const double *src_ch = (nt == 1) ? P.chp : P.tr_ch[1 - d];
    const double *src_ub = (nt == 1) ? P.ubp : P.tr_ub[1 - d];
    const double *src_vb = (nt == 1) ? P.vbp : P.tr_vb[1 - d];
    double *dst_ch = P.tr_ch[d], *dst_ub = P.tr_ub[d], *dst_vb = P.tr_vb[d];
    const double *land_ch = (nt == 1) ? P.chc : src_ch;  // chc before the predictor

    for (int t = blockIdx.x; t < ntiles; t += nblocks) {
      const int tx = t % ntx, ty = t / ntx;
      const int R0 = tx * TX, J0 = ty * TY + 1;
      const int tw = min(TX, G - R0), th = min(TY, nj - J0 + 1);
      const int rr0 = R0 - 2, jj0 = J0 - 2;  // region origin
      // --- S1: load ch (T, region [0, tw+4) x [0, th+4)) and ub, vb (U, [0, tw+3) x [0, th+3))
      {
        const int nx = tw + 4, ny = th + 4;
        for (int p = tid; p < nx * ny; p += nth) {
          const int lx = p % nx, ly = p / nx;
          const int j = jj0 + ly;
          if (j < 1 || j > nj) continue;
          const long long q = I2(P, ring_i(rr0 + lx), j);
          S(F_CH, lx, ly) = src_ch[q];
          if (lx < tw + 3 && ly < th + 3) {
            S(F_UB, lx, ly) = src_ub[q];
            S(F_VB, lx, ly) = src_vb[q];
          }
        }
      }
      __syncthreads();
      // --- S2: sch, supb on U [0, tw+3) x [0, th+3)
      {
        const int nx = tw + 3, ny = th + 3;
        for (int p = tid; p < nx * ny; p += nth) {
          const int lx = p % nx, ly = p / nx;
          const int j = jj0 + ly;
          if (j < 1 || j > nj) continue;
          const long long q = I2(P, ring_i(rr0 + lx), j);
          double sch = 1.0;
          if (__ldg(P.lev_u + q) > 0) {
            const double w = (j <= njm)
                                 ? (S(F_CH, lx, ly) + S(F_CH, lx, ly + 1) + S(F_CH, lx + 1, ly) + S(F_CH, lx + 1, ly + 1)) * 0.25
                                 : 0.0;
            sch = sqrt(w);
          }
          const double ps = ld(P.prh_u, q) * sch;
          S(F_S1, lx, ly) = ps * S(F_UB, lx, ly);
          S(F_X2, lx, ly) = ps * S(F_VB, lx, ly) * ld(P.rh[3], q);
        }
      }
      __syncthreads();
      // --- S3: tE on E [0, tw+3) x [1, th+3); tN on N [1, tw+3) x [0, th+3)
      {
        const int nx = tw + 3, ny = th + 3;
        for (int p = tid; p < nx * ny; p += nth) {
          const int lx = p % nx, ly = p / nx;
          const int j = jj0 + ly;
          if (j < 1 || j > nj) continue;
          if (ly >= 1) S(F_TE, lx, ly) = (j >= 2) ? 0.5 * (S(F_S1, lx, ly - 1) + S(F_S1, lx, ly)) : 0.0;
          if (lx >= 1) S(F_TN, lx, ly) = 0.5 * (S(F_X2, lx - 1, ly) + S(F_X2, lx, ly));
        }
      }
      __syncthreads();
      // --- S4: predictor ch on T [1, tw+3) x [1, th+3)
      {
        const int nx = tw + 2, ny = th + 2;
        for (int p = tid; p < nx * ny; p += nth) {
          const int lx = 1 + p % nx, ly = 1 + p / nx;
          const int j = jj0 + ly;
          if (j < 1 || j > nj) continue;
          const long long q = I2(P, ring_i(rr0 + lx), j);
          const double A = (S(F_TE, lx, ly) - S(F_TE, lx - 1, ly)) / ld(P.dxx[1], q);
          const double B = (j >= 2) ? (S(F_TN, lx, ly) - S(F_TN, lx, ly - 1)) / ld(P.dxy[1], q) : 0.0;
          const double div = (A + B) / (a * ld(P.rh[1], q));
          double pred;
          if (__ldg(P.lev_t + q) > 0) pred = S(F_CH, lx, ly) - div * bt * gamma_b / ld(P.prh_t, q);
          else pred = land_ch[q];
          S(F_PRED, lx, ly) = pred;
        }
      }
      __syncthreads();
      // --- S5: sch_e on U [1, tw+2) x [1, th+2); N-grid values on [1, tw+3) x [1, th+2);
      //         E-grid values on [1, tw+2) x [1, th+3)
      {
        const int nx = tw + 2, ny = th + 2;
        for (int p = tid; p < nx * ny; p += nth) {
          const int lx = 1 + p % nx, ly = 1 + p / nx;
          const int j = jj0 + ly;
          if (j < 1 || j > nj) continue;
          const long long q = I2(P, ring_i(rr0 + lx), j);
          const bool nrow = j <= njm, srow = j >= 2;
          // U: sch_e
          if (lx < tw + 2 && ly < th + 2) {
            double sch = 1.0;
            if (__ldg(P.lev_u + q) > 0) {
              const double w = nrow ? (S(F_PRED, lx, ly) + S(F_PRED, lx, ly + 1) + S(F_PRED, lx + 1, ly) +
                                       S(F_PRED, lx + 1, ly + 1)) * 0.25
                                    : 0.0;
              sch = sqrt(w);
            }
            S(F_SCHE, lx, ly) = sch;
          }
          // N grid (i, j): a1 = p1(ub)/rh4, gy = gra_y(pred), cN = ter_N(pred)
          if (ly < th + 2) {
            const double dx4 = ld(P.dxx[4], q), rh4 = ld(P.rh[4], q);
            S(F_A1U, lx, ly) = ((S(F_UB, lx, ly) - S(F_UB, lx - 1, ly)) / dx4) / rh4;
            S(F_A1V, lx, ly) = ((S(F_VB, lx, ly) - S(F_VB, lx - 1, ly)) / dx4) / rh4;
            if (nrow) {
              S(F_GY, lx, ly) = ((S(F_PRED, lx, ly + 1) - S(F_PRED, lx, ly)) / ld(P.dxy[4], q)) / a;
              S(F_CN, lx, ly) = 0.5 * (S(F_PRED, lx, ly) + S(F_PRED, lx, ly + 1));
            } else {
              S(F_GY, lx, ly) = 0.0;
              S(F_CN, lx, ly) = 0.0;
            }
          }
          // E grid (i, j): a2 = p2(ub)*rh2, gx = gra_x(pred), cE = ter_E(pred)
          if (lx < tw + 2) {
            const double rh2 = ld(P.rh[2], q);
            if (srow) {
              const double dy2 = ld(P.dxy[2], q);
              S(F_A2U, lx, ly) = ((S(F_UB, lx, ly) - S(F_UB, lx, ly - 1)) / dy2) * rh2;
              S(F_A2V, lx, ly) = ((S(F_VB, lx, ly) - S(F_VB, lx, ly - 1)) / dy2) * rh2;
            } else {
              S(F_A2U, lx, ly) = 0.0;
              S(F_A2V, lx, ly) = 0.0;
            }
            S(F_GX, lx, ly) = ((S(F_PRED, lx + 1, ly) - S(F_PRED, lx, ly)) / ld(P.dxx[2], q)) / (a * rh2);
            S(F_CE, lx, ly) = 0.5 * (S(F_PRED, lx, ly) + S(F_PRED, lx + 1, ly));
          }
        }
      }
      __syncthreads();
      // --- S6: corrector velocity on U [1, tw+2) x [1, th+2)
      {
        const int nx = tw + 1, ny = th + 1;
        for (int p = tid; p < nx * ny; p += nth) {
          const int lx = 1 + p % nx, ly = 1 + p / nx;
          const int j = jj0 + ly;
          if (j < 1 || j > nj) continue;
          const int i = ring_i(rr0 + lx);
          const long long q = I2(P, i, j);
          const bool nrow = j <= njm;
          const double seau = (double)(__ldg(P.lev_u + q) >= 1);
          const double rh3 = ld(P.rh[3], q), dx3 = ld(P.dxx[3], q), dy3 = ld(P.dxy[3], q);
          const double aarh = a * a * rh3;
          // op_lap (mod_op.f90:904-925)
          const double L1u = (S(F_A1U, lx + 1, ly) - S(F_A1U, lx, ly)) / dx3;
          const double L1v = (S(F_A1V, lx + 1, ly) - S(F_A1V, lx, ly)) / dx3;
          const double L2u = nrow ? (S(F_A2U, lx, ly + 1) - S(F_A2U, lx, ly)) / dy3 : 0.0;
          const double L2v = nrow ? (S(F_A2V, lx, ly + 1) - S(F_A2V, lx, ly)) / dy3 : 0.0;
          const double am1 = ld(P.am, q);
          const double vsu = seau * am1 * ((L1u + L2u) / aarh);
          const double vsv = seau * am1 * ((L1v + L2v) / aarh);
          double dvu, dvv;
          if (nt == 1) {
            dvu = vsu - vsu;
            dvv = vsv - vsv;
          } else {
            dvu = vsu - VS0U[q];
            dvv = vsv - VS0V[q];
          }
          // bottom-pressure gradient forces (mod_int.f90:211-233)
          double gi1 = 0.0, cg1 = 0.0;
          if (nrow) {
            gi1 = 0.5 * (S(F_GX, lx, ly) * ld(P.bphi[0], q) + S(F_GX, lx, ly + 1) * ld(P.bphi[1], q + ni));
            cg1 = 0.5 * (S(F_CE, lx, ly) * ld(P.bgra[0], q) + S(F_CE, lx, ly + 1) * ld(P.bgra[1], q + ni));
          }
          const double gi2 = 0.5 * (S(F_GY, lx, ly) * ld(P.bphi[2], q) + S(F_GY, lx + 1, ly) * ld(P.bphi[3], q + 1));
          const double cg2 = 0.5 * (S(F_CN, lx, ly) * ld(P.bgra[2], q) + S(F_CN, lx + 1, ly) * ld(P.bgra[3], q + 1));
          const double sch = S(F_SCHE, lx, ly);
          const double pg1 = (gi1 + cg1 + ld(P.graphihx, q)) * seau * sch;
          const double pg2 = (gi2 + cg2 + ld(P.graphihy, q)) * seau * sch;
          const double cor = ld(P.cor, q), ut = ld(P.ut, q), vt = ld(P.vt, q);
          const double ubp = S(F_UB, lx, ly), vbp = S(F_VB, lx, ly);
          double p1 = seau * (dvu + ut - pg1 + 0.5 * cor * vbp);
          double p2 = seau * (dvv + vt - pg2 - 0.5 * cor * ubp);
          const double w1 = p1 * bt + ubp, w2 = p2 * bt + vbp;
          const double cb = 0.5 * cor * bt;
          double u1 = (w1 + 0.5 * cor * bt * w2) / (1 + cb * cb);
          double v1 = (w2 - 0.5 * cor * bt * w1) / (1 + cb * cb);
          u1 = 0.5 * (u1 + ubp);
          v1 = 0.5 * (v1 + vbp);
          p1 = seau * (dvu - pg1 + ut + cor * v1);
          p2 = seau * (dvv - pg2 + vt - cor * u1);
          const double ubc = p1 * bt + ubp, vbc = p2 * bt + vbp;
          S(F_UBC, lx, ly) = ubc;
          S(F_VBC, lx, ly) = vbc;
          const double ps = ld(P.prh_u, q) * sch;
          S(F_S1N, lx, ly) = ps * ubc;
          S(F_X2N, lx, ly) = ps * vbc * rh3;
          // the first substep's viscosity is kept for the later ones (mod_int.f90:202-207)
          if (nt == 1 && lx >= 2 && ly >= 2) {
            VS0U[q] = vsu;
            VS0V[q] = vsv;
          }
        }
      }
      __syncthreads();
      // --- S7: ter to E on [1, tw+2) x [2, th+2), ter to N on [2, tw+2) x [1, th+2)
      {
        const int nx = tw + 1, ny = th + 1;
        for (int p = tid; p < nx * ny; p += nth) {
          const int lx = 1 + p % nx, ly = 1 + p / nx;
          const int j = jj0 + ly;
          if (j < 1 || j > nj) continue;
          if (ly >= 2) S(F_TEN, lx, ly) = (j >= 2) ? 0.5 * (S(F_S1N, lx, ly - 1) + S(F_S1N, lx, ly)) : 0.0;
          if (lx >= 2) S(F_TNN, lx, ly) = 0.5 * (S(F_X2N, lx - 1, ly) + S(F_X2N, lx, ly));
        }
      }
      __syncthreads();
      // --- S8: corrector ch on the tile, store, accumulate
      for (int p = tid; p < tw * th; p += nth) {
        const int lx = 2 + p % tw, ly = 2 + p / tw;
        const int j = jj0 + ly;
        const int i = ring_i(rr0 + lx);
        const long long q = I2(P, i, j);
        const double A = (S(F_TEN, lx, ly) - S(F_TEN, lx - 1, ly)) / ld(P.dxx[1], q);
        const double B = (j >= 2) ? (S(F_TNN, lx, ly) - S(F_TNN, lx, ly - 1)) / ld(P.dxy[1], q) : 0.0;
        const double div = (A + B) / (a * ld(P.rh[1], q));
        const double m1 = (double)(__ldg(P.lev_t + q) >= 1);
        const double chn = S(F_CH, lx, ly) - m1 * div * bt / ld(P.prh_t, q);
        const double ubc = S(F_UBC, lx, ly), vbc = S(F_VBC, lx, ly);
        st2(dst_ch, P, i, q, chn);
        st2(dst_ub, P, i, q, ubc);
        st2(dst_vb, P, i, q, vbc);
        if (nt <= nstep / 2) A_mch[q] = A_mch[q] + chn;
        A_mch2[q] = A_mch2[q] + chn;
        A_ua[q] = A_ua[q] + ubc;
        A_va[q] = A_va[q] + vbc;
      }
      __syncthreads();
    }
    if (!grid_barrier(P, nblocks)) return;
  }

  // averages (mod_int.f90:276-288)
  for (int t = blockIdx.x; t < ntiles; t += nblocks) {
    const int tx = t % ntx, ty = t / ntx;
    const int R0 = tx * TX, J0 = ty * TY + 1;
    const int tw = min(TX, G - R0), th = min(TY, nj - J0 + 1);
    for (int p = tid; p < tw * th; p += nth) {
      const int i = R0 + (p % tw) + 2, j = J0 + p / tw;
      const long long q = I2(P, i, j);
      const double ub = A_ua[q] / (nstep + 1), vb = A_va[q] / (nstep + 1);
      const double mch = A_mch[q] / (nstep / 2 + 1), mch2 = A_mch2[q] / (nstep + 1);
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

size_t trop_smem_bytes(int TX, int TY) { return (size_t)F_COUNT * (TX + 4) * (TY + 4) * sizeof(double); }

cudaError_t launch_trop(const Dev &P, int TX, int TY, int nblocks, cudaStream_t s) {
  const int ntx = (P.glo_ni + TX - 1) / TX, nty = (P.nj + TY - 1) / TY;
  const size_t smem = trop_smem_bytes(TX, TY);
  cudaError_t e = cudaFuncSetAttribute(k_trop, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  void *args[] = {(void *)&P, (void *)&TX, (void *)&TY, (void *)&ntx, (void *)&nty};
  return cudaLaunchCooperativeKernel((const void *)k_trop, dim3(nblocks), dim3(256), args, smem, s);
}

int trop_max_blocks(int TX, int TY) {
  int dev = 0, nsm = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const size_t smem = trop_smem_bytes(TX, TY);
  cudaFuncSetAttribute(k_trop, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_trop, 256, smem);
  return per * nsm;
}

// ============================================================================
// Resident variant: one tile per CTA and one region point per thread.
//
// Every thread owns one point of its CTA's (TX+4) x (TY+4) region for the
// whole subcycle, so each stage evaluates exactly one point per thread and
// every coefficient a point's formulas need (bottom pressures, the first
// substep's viscosity, the bphi/bgraphi integrals with the shifts the
// reference applies, Coriolis, the depth-mean tendency ...) is loaded into
// registers once and reused by all substeps.  The lat-lon metrics, which
// depend on i or on j only, are staged as 1-D vectors in shared memory.  Per
// substep the only global traffic is the (ch, ub, vb) halo exchange through
// L2 and the accumulators stay in registers.
namespace {
enum {
  R_CH, R_UB, R_VB,
  R_S1, R_X2,        // supb1, supb2*rh3 (reused for the corrector's supb)
  R_PRED, R_SCHE,
  R_A1U, R_A1V, R_GY, R_CN,
  R_A2U, R_A2V, R_GX, R_CE,
  R_UBC, R_VBC,
  R_COUNT
};
}  // namespace

constexpr int kResThreads = 640;

__global__ void __launch_bounds__(kResThreads, 1)
    k_trop_res(const __grid_constant__ Dev P, int TX, int TY, int ntx) {
  extern __shared__ double sm[];
  const int ni = P.ni, nj = P.nj, njm = P.njm, G = P.glo_ni;
  const int W = TX + 4, H = TY + 4, RS = W * H;
  double *vx = sm + R_COUNT * RS;  // dxx[1..4] over lx: 4*W
  double *vy = vx + 4 * W;         // dxy[1..4], rh[1..4] over ly: 8*H
  const double a = P.c.a, bt = (double)P.bt, gamma_b = P.c.gamma_b;
  const int nstep = P.nstep;
  const unsigned nblocks = gridDim.x;
  const int tid = threadIdx.x;
  const int tx = blockIdx.x % ntx, ty = blockIdx.x / ntx;
  const int R0 = tx * TX, J0 = ty * TY + 1;
  const int tw = min(TX, G - R0), th = min(TY, nj - J0 + 1);
  const int rr0 = R0 - 2, jj0 = J0 - 2;
  auto ring_i = [&](int r) { r %= G; if (r < 0) r += G; return r + 2; };

  // 1-D metrics
  for (int l = tid; l < W; l += blockDim.x) {
    const long long q = I2(P, ring_i(rr0 + l), J0);
    for (int g = 1; g <= 4; ++g) vx[(g - 1) * W + l] = ld(P.dxx[g], q);
  }
  for (int l = tid; l < H; l += blockDim.x) {
    const int j = jj0 + l;
    if (j < 1 || j > nj) continue;
    for (int g = 1; g <= 4; ++g) {
      vy[(g - 1) * H + l] = ld(P.dxy1d[g], j - 1);
      vy[(4 + g - 1) * H + l] = ld(P.rh1d[g], j - 1);
    }
  }
  auto DXX = [&](int g, int lx) { return vx[(g - 1) * W + lx]; };
  auto DXY = [&](int g, int ly) { return vy[(g - 1) * H + ly]; };
  auto RH = [&](int g, int ly) { return vy[(4 + g - 1) * H + ly]; };
  auto S = [&](int f, int p) -> double & { return sm[f * RS + p]; };

  // this thread's region point
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
  const double seau = (double)(levu >= 1), mskt1 = (double)(levt >= 1);
  const double prh_u = active ? ld(P.prh_u, q) : 1.0, prh_t = active ? ld(P.prh_t, q) : 1.0;
  // S6 coefficients (shifted where the reference's formulas shift them)
  double sam1 = 0, bxn = 0, bxs = 0, bye = 0, byw = 0, gxn = 0, gxs = 0, gye = 0, gyw = 0;
  double ghx = 0, ghy = 0, cor = 0, ut = 0, vt = 0;
  if (inS6) {
    sam1 = seau * ld(P.am, q);
    bxn = ld(P.bphi[0], q); bye = ld(P.bphi[2], q); byw = ld(P.bphi[3], q + 1);
    gxn = ld(P.bgra[0], q); gye = ld(P.bgra[2], q); gyw = ld(P.bgra[3], q + 1);
    if (nrow) { bxs = ld(P.bphi[1], q + ni); gxs = ld(P.bgra[1], q + ni); }
    ghx = ld(P.graphihx, q); ghy = ld(P.graphihy, q);
    cor = ld(P.cor, q); ut = ld(P.ut, q); vt = ld(P.vt, q);
  }
  double vs0u = 0.0, vs0v = 0.0;
  // accumulators (mod_int.f90:176-180)
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
    // S1: previous state
    if (active) {
      S(R_CH, p) = src_ch[q];
      if (inS2) { S(R_UB, p) = src_ub[q]; S(R_VB, p) = src_vb[q]; }
    }
    __syncthreads();
    // S2: sch = sqrt(ter(ch)) on U, supb
    if (inS2) {
      double sch = 1.0;
      if (levu > 0) {
        const double w = nrow ? (S(R_CH, p) + S(R_CH, p + W) + S(R_CH, p + 1) + S(R_CH, p + W + 1)) * 0.25 : 0.0;
        sch = sqrt(w);
      }
      const double ps = prh_u * sch;
      S(R_S1, p) = ps * S(R_UB, p);
      S(R_X2, p) = ps * S(R_VB, p) * RH(3, ly);
    }
    __syncthreads();
    // S4: predictor ch; the ter U->E (rows >= 2) and U->N means of supb are
    // formed here from the staged supb
    if (inS4) {
      // tE at (i, j) and (i-1, j): j >= 2 ? 0.5 (s1(j-1) + s1(j)) : 0
      const double tEc = srow ? 0.5 * (S(R_S1, p - W) + S(R_S1, p)) : 0.0;
      const double tEw = srow ? 0.5 * (S(R_S1, p - W - 1) + S(R_S1, p - 1)) : 0.0;
      const double A = (tEc - tEw) / DXX(1, lx);
      double B = 0.0;
      if (srow) {
        // tN at (i, j) and (i, j-1): 0.5 (x2(i-1) + x2(i))
        const double tNc = 0.5 * (S(R_X2, p - 1) + S(R_X2, p));
        const double tNs = 0.5 * (S(R_X2, p - W - 1) + S(R_X2, p - W));
        B = (tNc - tNs) / DXY(1, ly);
      }
      const double div = (A + B) / (a * RH(1, ly));
      double pred;
      if (levt > 0) pred = S(R_CH, p) - div * bt * gamma_b / prh_t;
      else pred = (nt == 1) ? land_ch0 : S(R_CH, p);
      S(R_PRED, p) = pred;
    }
    __syncthreads();
    // S5: sch on U; N- and E-grid intermediates
    if (inS6) {
      double sch = 1.0;
      if (levu > 0) {
        const double w = nrow ? (S(R_PRED, p) + S(R_PRED, p + W) + S(R_PRED, p + 1) + S(R_PRED, p + W + 1)) * 0.25 : 0.0;
        sch = sqrt(w);
      }
      S(R_SCHE, p) = sch;
    }
    if (inN) {
      const double dx4 = DXX(4, lx), rh4 = RH(4, ly);
      S(R_A1U, p) = ((S(R_UB, p) - S(R_UB, p - 1)) / dx4) / rh4;
      S(R_A1V, p) = ((S(R_VB, p) - S(R_VB, p - 1)) / dx4) / rh4;
      if (nrow) {
        S(R_GY, p) = ((S(R_PRED, p + W) - S(R_PRED, p)) / DXY(4, ly)) / a;
        S(R_CN, p) = 0.5 * (S(R_PRED, p) + S(R_PRED, p + W));
      } else {
        S(R_GY, p) = 0.0;
        S(R_CN, p) = 0.0;
      }
    }
    if (inE) {
      const double rh2 = RH(2, ly);
      if (srow) {
        const double dy2 = DXY(2, ly);
        S(R_A2U, p) = ((S(R_UB, p) - S(R_UB, p - W)) / dy2) * rh2;
        S(R_A2V, p) = ((S(R_VB, p) - S(R_VB, p - W)) / dy2) * rh2;
      } else {
        S(R_A2U, p) = 0.0;
        S(R_A2V, p) = 0.0;
      }
      S(R_GX, p) = ((S(R_PRED, p + 1) - S(R_PRED, p)) / DXX(2, lx)) / (a * rh2);
      S(R_CE, p) = 0.5 * (S(R_PRED, p) + S(R_PRED, p + 1));
    }
    __syncthreads();
    // S6: corrector velocity (viscosity, pressure gradient, Coriolis adjustment)
    if (inS6) {
      const double rh3 = RH(3, ly), dx3 = DXX(3, lx), dy3 = DXY(3, ly);
      const double aarh = a * a * rh3;
      const double L1u = (S(R_A1U, p + 1) - S(R_A1U, p)) / dx3;
      const double L1v = (S(R_A1V, p + 1) - S(R_A1V, p)) / dx3;
      const double L2u = nrow ? (S(R_A2U, p + W) - S(R_A2U, p)) / dy3 : 0.0;
      const double L2v = nrow ? (S(R_A2V, p + W) - S(R_A2V, p)) / dy3 : 0.0;
      const double vsu = sam1 * ((L1u + L2u) / aarh);
      const double vsv = sam1 * ((L1v + L2v) / aarh);
      if (nt == 1) { vs0u = vsu; vs0v = vsv; }
      const double dvu = vsu - vs0u, dvv = vsv - vs0v;
      double gi1 = 0.0, cg1 = 0.0;
      if (nrow) {
        gi1 = 0.5 * (S(R_GX, p) * bxn + S(R_GX, p + W) * bxs);
        cg1 = 0.5 * (S(R_CE, p) * gxn + S(R_CE, p + W) * gxs);
      }
      const double gi2 = 0.5 * (S(R_GY, p) * bye + S(R_GY, p + 1) * byw);
      const double cg2 = 0.5 * (S(R_CN, p) * gye + S(R_CN, p + 1) * gyw);
      const double sch = S(R_SCHE, p);
      const double pg1 = (gi1 + cg1 + ghx) * seau * sch;
      const double pg2 = (gi2 + cg2 + ghy) * seau * sch;
      const double ubp = S(R_UB, p), vbp = S(R_VB, p);
      double p1 = seau * (dvu + ut - pg1 + 0.5 * cor * vbp);
      double p2 = seau * (dvv + vt - pg2 - 0.5 * cor * ubp);
      const double w1 = p1 * bt + ubp, w2 = p2 * bt + vbp;
      const double cb = 0.5 * cor * bt;
      double u1 = (w1 + 0.5 * cor * bt * w2) / (1 + cb * cb);
      double v1 = (w2 - 0.5 * cor * bt * w1) / (1 + cb * cb);
      u1 = 0.5 * (u1 + ubp);
      v1 = 0.5 * (v1 + vbp);
      p1 = seau * (dvu - pg1 + ut + cor * v1);
      p2 = seau * (dvv - pg2 + vt - cor * u1);
      const double ubc = p1 * bt + ubp, vbc = p2 * bt + vbp;
      S(R_UBC, p) = ubc;
      S(R_VBC, p) = vbc;
      const double ps = prh_u * sch;
      S(R_S1, p) = ps * ubc;
      S(R_X2, p) = ps * vbc * rh3;
    }
    __syncthreads();
    // S8: corrector ch (with the ter means of the corrector's supb), store, accumulate
    if (inS8) {
      const double tEc = srow ? 0.5 * (S(R_S1, p - W) + S(R_S1, p)) : 0.0;
      const double tEw = srow ? 0.5 * (S(R_S1, p - W - 1) + S(R_S1, p - 1)) : 0.0;
      const double A = (tEc - tEw) / DXX(1, lx);
      double B = 0.0;
      if (srow) {
        const double tNc = 0.5 * (S(R_X2, p - 1) + S(R_X2, p));
        const double tNs = 0.5 * (S(R_X2, p - W - 1) + S(R_X2, p - W));
        B = (tNc - tNs) / DXY(1, ly);
      }
      const double div = (A + B) / (a * RH(1, ly));
      const double chn = S(R_CH, p) - mskt1 * div * bt / prh_t;
      const double ubc = S(R_UBC, p), vbc = S(R_VBC, p);
      const int d2 = d;
      st2(P.tr_ch[d2], P, i, q, chn);
      st2(P.tr_ub[d2], P, i, q, ubc);
      st2(P.tr_vb[d2], P, i, q, vbc);
      if (nt <= nstep / 2) acc_m = acc_m + chn;
      acc_m2 = acc_m2 + chn;
      acc_u = acc_u + ubc;
      acc_v = acc_v + vbc;
    }
    if (!grid_barrier(P, nblocks)) return;
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
}

size_t trop_res_smem_bytes(int TX, int TY) {
  return ((size_t)R_COUNT * (TX + 4) * (TY + 4) + 4 * (TX + 4) + 8 * (TY + 4)) * sizeof(double);
}

bool trop_res_fits(int TX, int TY) { return (TX + 4) * (TY + 4) <= kResThreads; }

cudaError_t launch_trop_res(const Dev &P, int TX, int TY, cudaStream_t s) {
  const int ntx = (P.glo_ni + TX - 1) / TX, nty = (P.nj + TY - 1) / TY;
  const size_t smem = trop_res_smem_bytes(TX, TY);
  cudaError_t e = cudaFuncSetAttribute(k_trop_res, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int nthreads = ((TX + 4) * (TY + 4) + 31) / 32 * 32;
  void *args[] = {(void *)&P, (void *)&TX, (void *)&TY, (void *)&ntx};
  return cudaLaunchCooperativeKernel((const void *)k_trop_res, dim3(ntx * nty), dim3(nthreads), args, smem, s);
}

int trop_res_max_blocks(int TX, int TY) {
  int dev = 0, nsm = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const size_t smem = trop_res_smem_bytes(TX, TY);
  if (cudaFuncSetAttribute(k_trop_res, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
  const int nthreads = ((TX + 4) * (TY + 4) + 31) / 32 * 32;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_trop_res, nthreads, smem) != cudaSuccess) return 0;
  return per * nsm;
}

// ============================================================================
// Fast variant of the resident kernel: the same arithmetic with every division
// by a static metric, bottom pressure or Coriolis denominator done with its
// correctly rounded reciprocal (dvr), which removes the per-division
// reciprocal-approximation instruction from the critical path.

//
// GROUP = true: the same kernel over a work list of tiles of several domains
// (ensemble members, basins), one tile per CTA; each CTA reads its domain's
// Dev from `Ps`, and the grid barrier counts on `gcnt` (zeroed before the
// launch) with timeouts flagged in `gerr`.
//
// CTX, CTY > 0: the same kernel compiled for one tile shape, so that the
// region's row length and plane size are constants and every shared-memory
// operand is a fixed offset from the thread's own point (fewer instructions
// and registers per substep than the general form, CTX = CTY = 0).
template <bool GROUP, int CTX = 0, int CTY = 0>
__global__ void __launch_bounds__(kResThreads, 1)
    k_trop_fast(const __grid_constant__ Dev P0, const Dev *__restrict__ Ps, const TileRef *__restrict__ tiles,
                int TX, int TY, int ntx, unsigned long long epoch, unsigned long long *gcnt, int *gerr) {
  if (CTX > 0) { TX = CTX; TY = CTY; }
  extern __shared__ double sm[];
  __shared__ int s_stop;
  const TileRef T = GROUP ? tiles[blockIdx.x] : TileRef{0, 0, 0, 0, 0};
  const Dev &P = GROUP ? Ps[T.m] : P0;
  unsigned long long *const bar_cnt = GROUP ? gcnt : P.tile_flag;
  int *const bar_err = GROUP ? gerr : P.err;
  const int ni = P.ni, nj = P.nj, njm = P.njm, G = P.glo_ni;
  const int W = TX + 4, H = TY + 4, RS = W * H;
  double *vx = sm + R_COUNT * RS;  // dxx[1..4], 1/dxx[1..4] over lx: 8*W
  double *vy = vx + 8 * W;         // kFastVy vectors over ly (see below)
  const double a = P.c.a, bt = (double)P.bt, gamma_b = P.c.gamma_b;
  const int nstep = P.nstep;
  const int tid = threadIdx.x;
  int R0, J0, tw, th;
  if (GROUP) {
    R0 = T.r0; J0 = T.j0; tw = T.tw; th = T.th;
  } else {
    const int tx = blockIdx.x % ntx, ty = blockIdx.x / ntx;
    R0 = tx * TX; J0 = ty * TY + 1;
    tw = min(TX, G - R0); th = min(TY, nj - J0 + 1);
  }
  const int rr0 = R0 - 2, jj0 = J0 - 2;
  auto ring_i = [&](int r) { r %= G; if (r < 0) r += G; return r + 2; };

  // 1-D metrics and the reciprocals of every divisor (dvr)
  for (int l = tid; l < W; l += blockDim.x) {
    const int i = ring_i(rr0 + l);
    for (int g = 1; g <= 4; ++g) {
      vx[(g - 1) * W + l] = ld(P.dxx1d[g], i - 1);
      vx[(4 + g - 1) * W + l] = ld(P.rdxx1d[g], i - 1);
    }
  }
  for (int l = tid; l < H; l += blockDim.x) {
    const int j = jj0 + l;
    if (j < 1 || j > nj) continue;
    for (int g = 1; g <= 4; ++g) {
      vy[(g - 1) * H + l] = ld(P.dxy1d[g], j - 1);
      vy[(4 + g - 1) * H + l] = ld(P.rdxy1d[g], j - 1);
      vy[(8 + g - 1) * H + l] = ld(P.rh1d[g], j - 1);
    }
    vy[12 * H + l] = ld(P.arh1d[1], j - 1);
    vy[13 * H + l] = ld(P.rarh1d[1], j - 1);
    vy[14 * H + l] = ld(P.arh1d[2], j - 1);
    vy[15 * H + l] = ld(P.rarh1d[2], j - 1);
    vy[16 * H + l] = ld(P.rrh1d[4], j - 1);
    vy[17 * H + l] = ld(P.aarh3, j - 1);
    vy[18 * H + l] = ld(P.raarh3, j - 1);
  }
  auto DXX = [&](int g, int lx) { return vx[(g - 1) * W + lx]; };
  auto RDXX = [&](int g, int lx) { return vx[(4 + g - 1) * W + lx]; };
  auto DXY = [&](int g, int ly) { return vy[(g - 1) * H + ly]; };
  auto RDXY = [&](int g, int ly) { return vy[(4 + g - 1) * H + ly]; };
  auto RH = [&](int g, int ly) { return vy[(8 + g - 1) * H + ly]; };
  const double ra = P.ra;
  auto S = [&](int f, int p) -> double & { return sm[f * RS + p]; };

  // this thread's region point
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
  const double seau = (double)(levu >= 1), mskt1 = (double)(levt >= 1);
  const double prh_u = active ? ld(P.prh_u, q) : 1.0, prh_t = active ? ld(P.prh_t, q) : 1.0;
  const double rprh_t = active ? ld(P.rprh_t, q) : 1.0;
  const double rden = active ? ld(P.rwt, q) : 1.0;  // 1 / (1 + (0.5 cor dtbt)^2)
  // S6 coefficients (shifted where the reference's formulas shift them)
  double sam1 = 0, bxn = 0, bxs = 0, bye = 0, byw = 0, gxn = 0, gxs = 0, gye = 0, gyw = 0;
  double ghx = 0, ghy = 0, cor = 0, ut = 0, vt = 0;
  if (inS6) {
    sam1 = seau * ld(P.am, q);
    bxn = ld(P.bphi[0], q); bye = ld(P.bphi[2], q); byw = ld(P.bphi[3], q + 1);
    gxn = ld(P.bgra[0], q); gye = ld(P.bgra[2], q); gyw = ld(P.bgra[3], q + 1);
    if (nrow) { bxs = ld(P.bphi[1], q + ni); gxs = ld(P.bgra[1], q + ni); }
    ghx = ld(P.graphihx, q); ghy = ld(P.graphihy, q);
    cor = ld(P.cor, q); ut = ld(P.ut, q); vt = ld(P.vt, q);
  }
  double vs0u = 0.0, vs0v = 0.0;
  // accumulators (mod_int.f90:176-180)
  double acc_m = 0, acc_m2 = 0, acc_u = 0, acc_v = 0;
  if (inS8) {
    acc_m = P.chc[q]; acc_m2 = acc_m;
    acc_u = P.ubc[q]; acc_v = P.vbc[q];
  }
  const double land_ch0 = inS4 ? P.chc[q] : 0.0;
  __syncthreads();

  // S2 at this thread's point: sch = sqrt(ter(ch)) on U and the fluxes
  // supb.  Points with lx in 2..tw and ly in 2..th read only the tile's own
  // state (ch at the point and its E, N, NE neighbours; ub, vb at the point)
  auto s2 = [&]() {
    double sch = 1.0;
    if (levu > 0) {
      const double w = nrow ? (S(R_CH, p) + S(R_CH, p + W) + S(R_CH, p + 1) + S(R_CH, p + W + 1)) * 0.25 : 0.0;
      sch = sqrt(w);
    }
    const double ps = prh_u * sch;
    S(R_S1, p) = ps * S(R_UB, p);
    S(R_X2, p) = ps * S(R_VB, p) * RH(3, ly);
  };
  const bool s2own = inS2 && lx >= 2 && lx <= tw && ly >= 2 && ly <= th;

  const unsigned long long base = epoch;  // arrivals counted before this launch
  for (int nt = 1; nt <= nstep; ++nt) {
    const int d = (nt - 1) & 1;
    const double *src_ch = (nt == 1) ? P.chp : P.tr_ch[1 - d];
    const double *src_ub = (nt == 1) ? P.ubp : P.tr_ub[1 - d];
    const double *src_vb = (nt == 1) ? P.vbp : P.tr_vb[1 - d];
    // S1: previous state.  After the first substep the tile's own points
    // already hold it (written in S8), so only the 2-cell ring comes from
    // L2 (.cg loads: written by other SMs)
    if (active && (nt == 1 || !inS8)) {
      S(R_CH, p) = __ldcg(src_ch + q);
      if (inS2) { S(R_UB, p) = __ldcg(src_ub + q); S(R_VB, p) = __ldcg(src_vb + q); }
    }
    __syncthreads();
    // S2: sch = sqrt(ter(ch)) on U, supb (after the first substep the
    // points whose inputs are all the tile's own were done while waiting at
    // the grid barrier)
    if (inS2 && (nt == 1 || !s2own)) s2();
    __syncthreads();
    // S4: predictor ch; the ter U->E (rows >= 2) and U->N means of supb are
    // formed here from the staged supb
    if (inS4) {
      // tE at (i, j) and (i-1, j): j >= 2 ? 0.5 (s1(j-1) + s1(j)) : 0
      const double tEc = srow ? 0.5 * (S(R_S1, p - W) + S(R_S1, p)) : 0.0;
      const double tEw = srow ? 0.5 * (S(R_S1, p - W - 1) + S(R_S1, p - 1)) : 0.0;
      const double A = dvr(tEc - tEw, DXX(1, lx), RDXX(1, lx));
      double B = 0.0;
      if (srow) {
        // tN at (i, j) and (i, j-1): 0.5 (x2(i-1) + x2(i))
        const double tNc = 0.5 * (S(R_X2, p - 1) + S(R_X2, p));
        const double tNs = 0.5 * (S(R_X2, p - W - 1) + S(R_X2, p - W));
        B = dvr(tNc - tNs, DXY(1, ly), RDXY(1, ly));
      }
      const double div = dvr(A + B, vy[12 * H + ly], vy[13 * H + ly]);
      double pred;
      if (levt > 0) pred = S(R_CH, p) - dvr(div * bt * gamma_b, prh_t, rprh_t);
      else pred = (nt == 1) ? land_ch0 : S(R_CH, p);
      S(R_PRED, p) = pred;
    }
    __syncthreads();
    // S5: sch on U; N- and E-grid intermediates
    if (inS6) {
      double sch = 1.0;
      if (levu > 0) {
        const double w = nrow ? (S(R_PRED, p) + S(R_PRED, p + W) + S(R_PRED, p + 1) + S(R_PRED, p + W + 1)) * 0.25 : 0.0;
        sch = sqrt(w);
      }
      S(R_SCHE, p) = sch;
    }
    if (inN) {
      const double dx4 = DXX(4, lx), rdx4 = RDXX(4, lx), rh4 = RH(4, ly), rrh4 = vy[16 * H + ly];
      S(R_A1U, p) = dvr(dvr(S(R_UB, p) - S(R_UB, p - 1), dx4, rdx4), rh4, rrh4);
      S(R_A1V, p) = dvr(dvr(S(R_VB, p) - S(R_VB, p - 1), dx4, rdx4), rh4, rrh4);
      if (nrow) {
        S(R_GY, p) = dvr(dvr(S(R_PRED, p + W) - S(R_PRED, p), DXY(4, ly), RDXY(4, ly)), a, ra);
        S(R_CN, p) = 0.5 * (S(R_PRED, p) + S(R_PRED, p + W));
      } else {
        S(R_GY, p) = 0.0;
        S(R_CN, p) = 0.0;
      }
    }
    if (inE) {
      const double rh2 = RH(2, ly);
      if (srow) {
        const double dy2 = DXY(2, ly), rdy2 = RDXY(2, ly);
        S(R_A2U, p) = dvr(S(R_UB, p) - S(R_UB, p - W), dy2, rdy2) * rh2;
        S(R_A2V, p) = dvr(S(R_VB, p) - S(R_VB, p - W), dy2, rdy2) * rh2;
      } else {
        S(R_A2U, p) = 0.0;
        S(R_A2V, p) = 0.0;
      }
      S(R_GX, p) = dvr(dvr(S(R_PRED, p + 1) - S(R_PRED, p), DXX(2, lx), RDXX(2, lx)), vy[14 * H + ly], vy[15 * H + ly]);
      S(R_CE, p) = 0.5 * (S(R_PRED, p) + S(R_PRED, p + 1));
    }
    __syncthreads();
    // S6: corrector velocity (viscosity, pressure gradient, Coriolis adjustment)
    if (inS6) {
      const double rh3 = RH(3, ly), dx3 = DXX(3, lx), rdx3 = RDXX(3, lx), dy3 = DXY(3, ly), rdy3 = RDXY(3, ly);
      const double aarh = vy[17 * H + ly], raarh = vy[18 * H + ly];
      const double L1u = dvr(S(R_A1U, p + 1) - S(R_A1U, p), dx3, rdx3);
      const double L1v = dvr(S(R_A1V, p + 1) - S(R_A1V, p), dx3, rdx3);
      const double L2u = nrow ? dvr(S(R_A2U, p + W) - S(R_A2U, p), dy3, rdy3) : 0.0;
      const double L2v = nrow ? dvr(S(R_A2V, p + W) - S(R_A2V, p), dy3, rdy3) : 0.0;
      const double vsu = sam1 * dvr(L1u + L2u, aarh, raarh);
      const double vsv = sam1 * dvr(L1v + L2v, aarh, raarh);
      if (nt == 1) { vs0u = vsu; vs0v = vsv; }
      const double dvu = vsu - vs0u, dvv = vsv - vs0v;
      double gi1 = 0.0, cg1 = 0.0;
      if (nrow) {
        gi1 = 0.5 * (S(R_GX, p) * bxn + S(R_GX, p + W) * bxs);
        cg1 = 0.5 * (S(R_CE, p) * gxn + S(R_CE, p + W) * gxs);
      }
      const double gi2 = 0.5 * (S(R_GY, p) * bye + S(R_GY, p + 1) * byw);
      const double cg2 = 0.5 * (S(R_CN, p) * gye + S(R_CN, p + 1) * gyw);
      const double sch = S(R_SCHE, p);
      const double pg1 = (gi1 + cg1 + ghx) * seau * sch;
      const double pg2 = (gi2 + cg2 + ghy) * seau * sch;
      const double ubp = S(R_UB, p), vbp = S(R_VB, p);
      double p1 = seau * (dvu + ut - pg1 + 0.5 * cor * vbp);
      double p2 = seau * (dvv + vt - pg2 - 0.5 * cor * ubp);
      const double w1 = p1 * bt + ubp, w2 = p2 * bt + vbp;
      const double cb = 0.5 * cor * bt;
      const double den = 1 + cb * cb;
      double u1 = dvr(w1 + 0.5 * cor * bt * w2, den, rden);
      double v1 = dvr(w2 - 0.5 * cor * bt * w1, den, rden);
      u1 = 0.5 * (u1 + ubp);
      v1 = 0.5 * (v1 + vbp);
      p1 = seau * (dvu - pg1 + ut + cor * v1);
      p2 = seau * (dvv - pg2 + vt - cor * u1);
      const double ubc = p1 * bt + ubp, vbc = p2 * bt + vbp;
      S(R_UBC, p) = ubc;
      S(R_VBC, p) = vbc;
      const double ps = prh_u * sch;
      S(R_S1, p) = ps * ubc;
      S(R_X2, p) = ps * vbc * rh3;
    }
    __syncthreads();
    // S8: corrector ch (with the ter means of the corrector's supb), store, accumulate
    if (inS8) {
      const double tEc = srow ? 0.5 * (S(R_S1, p - W) + S(R_S1, p)) : 0.0;
      const double tEw = srow ? 0.5 * (S(R_S1, p - W - 1) + S(R_S1, p - 1)) : 0.0;
      const double A = dvr(tEc - tEw, DXX(1, lx), RDXX(1, lx));
      double B = 0.0;
      if (srow) {
        const double tNc = 0.5 * (S(R_X2, p - 1) + S(R_X2, p));
        const double tNs = 0.5 * (S(R_X2, p - W - 1) + S(R_X2, p - W));
        B = dvr(tNc - tNs, DXY(1, ly), RDXY(1, ly));
      }
      const double div = dvr(A + B, vy[12 * H + ly], vy[13 * H + ly]);
      const double chn = S(R_CH, p) - dvr(mskt1 * div * bt, prh_t, rprh_t);
      const double ubc = S(R_UBC, p), vbc = S(R_VBC, p);
      const int d2 = d;
      st2(P.tr_ch[d2], P, i, q, chn);
      st2(P.tr_ub[d2], P, i, q, ubc);
      st2(P.tr_vb[d2], P, i, q, vbc);
      // the next substep's state at this point (during S8 only this thread
      // reads these three entries)
      S(R_CH, p) = chn;
      S(R_UB, p) = ubc;
      S(R_VB, p) = vbc;
      if (nt <= nstep / 2) acc_m = acc_m + chn;
      acc_m2 = acc_m2 + chn;
      acc_u = acc_u + ubc;
      acc_v = acc_v + vbc;
    }
    // grid barrier on a monotone arrival counter: after the CTA barrier,
    // thread 0 adds 1 with release semantics (cumulative over the CTA's
    // writes ordered before it by bar.sync), then waits (bounded, acquire)
    // for all arrivals of this substep; the counter is never reset, targets
    // grow per launch.  The outcome reaches the CTA through shared memory.
    // Between the arrival and the wait the CTA does the next substep's S2 on
    // the points that need no other tile's state (shared memory only: the
    // S8 reads of supb are behind the CTA barrier).
    __syncthreads();
    if (tid == 0) {
      cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> c(*bar_cnt);
      c.fetch_add(1ULL, cuda::memory_order_release);
    }
    if (nt < nstep && s2own) s2();
    if (tid == 0) {
      const unsigned long long want = base + (unsigned long long)nt * gridDim.x;
      s_stop = wait_count(bar_cnt, want, bar_err, P.wait_ns) ? 0 : 1;
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
}


// The resident kernel's synchronisation skeleton, its latency floor: the
// same grid, block and shared memory (so the same residency, one CTA per SM),
// and per substep the same ring reload of ch, ub, vb from L2, the same seven
// CTA barriers, the same interior stores and the same grid barrier on the
// monotone arrival counter, with none of the arithmetic.  It writes only the
// subcycle's ping-pong buffers, which every barotropic launch starts afresh
// from chp, ubp, vbp.  (The real kernel also does the next substep's S2 on
// its own points while it waits at the grid barrier.)
__global__ void __launch_bounds__(kResThreads, 1)
    k_trop_floor(const __grid_constant__ Dev P, int TX, int TY, int ntx, unsigned long long epoch) {
  extern __shared__ double sm[];
  __shared__ int s_stop;
  const int nj = P.nj, G = P.glo_ni;
  const int W = TX + 4, H = TY + 4, RS = W * H;
  const int tid = threadIdx.x;
  const int tx = blockIdx.x % ntx, ty = blockIdx.x / ntx;
  const int R0 = tx * TX, J0 = ty * TY + 1;
  const int tw = min(TX, G - R0), th = min(TY, nj - J0 + 1);
  const int rr0 = R0 - 2, jj0 = J0 - 2;
  auto ring_i = [&](int r) { r %= G; if (r < 0) r += G; return r + 2; };
  auto S = [&](int f, int p) -> double & { return sm[f * RS + p]; };
  const int p = tid;
  const int lx = p % W, ly = p / W;
  const int j = jj0 + ly;
  const bool active = p < RS && j >= 1 && j <= nj;
  const int i = active ? ring_i(rr0 + lx) : 2;
  const long long q = active ? I2(P, i, j) : 0;
  const bool inS2 = active && lx < tw + 3 && ly < th + 3;
  const bool inS8 = active && lx >= 2 && lx < tw + 2 && ly >= 2 && ly < th + 2;
  __syncthreads();
  for (int nt = 1; nt <= P.nstep; ++nt) {
    const int d = (nt - 1) & 1;
    const double *src_ch = (nt == 1) ? P.chp : P.tr_ch[1 - d];
    const double *src_ub = (nt == 1) ? P.ubp : P.tr_ub[1 - d];
    const double *src_vb = (nt == 1) ? P.vbp : P.tr_vb[1 - d];
    if (active && (nt == 1 || !inS8)) {
      S(R_CH, p) = __ldcg(src_ch + q);
      if (inS2) { S(R_UB, p) = __ldcg(src_ub + q); S(R_VB, p) = __ldcg(src_vb + q); }
    }
    #pragma unroll 1
    for (int b = 0; b < 5; ++b) __syncthreads();  // after S1, S2, S4, S5, S6
    if (inS8) {
      st2(P.tr_ch[d], P, i, q, S(R_CH, p));
      st2(P.tr_ub[d], P, i, q, S(R_UB, p));
      st2(P.tr_vb[d], P, i, q, S(R_VB, p));
    }
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
}

cudaError_t launch_trop_floor(const Dev &P, int TX, int TY, unsigned long long epoch, cudaStream_t s) {
  const int ntx = (P.glo_ni + TX - 1) / TX, nty = (P.nj + TY - 1) / TY;
  const size_t smem = trop_fast_smem_bytes(TX, TY);
  cudaError_t e = cudaFuncSetAttribute(k_trop_floor, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int nthreads = ((TX + 4) * (TY + 4) + 31) / 32 * 32;
  void *args[] = {(void *)&P, (void *)&TX, (void *)&TY, (void *)&ntx, (void *)&epoch};
  return cudaLaunchCooperativeKernel((const void *)k_trop_floor, dim3(ntx * nty), dim3(nthreads), args, smem, s);
}

size_t trop_fast_smem_bytes(int TX, int TY) {
  return ((size_t)R_COUNT * (TX + 4) * (TY + 4) + 8 * (TX + 4) + 19 * (TY + 4)) * sizeof(double);
}

namespace {
// the single-domain kernel for a tile shape: the fixed-shape form where one
// is compiled (the 24 x 18 tiles of the 1-degree 360 x 160 domain)
const void *fast_kernel(int TX, int TY) {
  if (TX == 24 && TY == 18) return (const void *)k_trop_fast<false, 24, 18>;
  return (const void *)k_trop_fast<false>;
}
// the group kernel for a tile shape: a fixed-shape form for each tile shape
// the batch autotuner tries (pcom_gpu_batch_autotune), the general one
// otherwise
const void *group_kernel(int TX, int TY) {
#define PCOM_GROUP_SHAPE(x, y) \
  if (TX == (x) && TY == (y)) return (const void *)k_trop_fast<true, (x), (y)>;
  PCOM_GROUP_SHAPE(12, 12) PCOM_GROUP_SHAPE(16, 8) PCOM_GROUP_SHAPE(16, 12) PCOM_GROUP_SHAPE(16, 16)
  PCOM_GROUP_SHAPE(24, 12) PCOM_GROUP_SHAPE(20, 16) PCOM_GROUP_SHAPE(24, 18) PCOM_GROUP_SHAPE(32, 8)
  PCOM_GROUP_SHAPE(32, 12) PCOM_GROUP_SHAPE(28, 16) PCOM_GROUP_SHAPE(48, 8) PCOM_GROUP_SHAPE(64, 6)
#undef PCOM_GROUP_SHAPE
  return (const void *)k_trop_fast<true>;
}
}  // namespace

cudaError_t launch_trop_fast(const Dev &P, int TX, int TY, unsigned long long epoch, cudaStream_t s) {
  const int ntx = (P.glo_ni + TX - 1) / TX, nty = (P.nj + TY - 1) / TY;
  const size_t smem = trop_fast_smem_bytes(TX, TY);
  const void *fn = fast_kernel(TX, TY);
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int nthreads = ((TX + 4) * (TY + 4) + 31) / 32 * 32;
  const Dev *nps = nullptr;
  const TileRef *nts = nullptr;
  unsigned long long *ncnt = nullptr;
  int *nerr = nullptr;
  void *args[] = {(void *)&P, (void *)&nps, (void *)&nts, (void *)&TX, (void *)&TY, (void *)&ntx, (void *)&epoch,
                  (void *)&ncnt, (void *)&nerr};
  return cudaLaunchCooperativeKernel(fn, dim3(ntx * nty), dim3(nthreads), args, smem, s);
}

namespace {
template <bool GROUP>
int fast_max_blocks(int TX, int TY) {
  int dev = 0, nsm = 0, per = 0;
  if ((TX + 4) * (TY + 4) > kResThreads) return 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const size_t smem = trop_fast_smem_bytes(TX, TY);
  const void *fn = GROUP ? group_kernel(TX, TY) : fast_kernel(TX, TY);
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
  const int nthreads = ((TX + 4) * (TY + 4) + 31) / 32 * 32;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, nthreads, smem) != cudaSuccess) return 0;
  return per * nsm;
}
}  // namespace

int trop_fast_max_blocks(int TX, int TY) { return fast_max_blocks<false>(TX, TY); }
int trop_group_max_blocks(int TX, int TY) { return fast_max_blocks<true>(TX, TY); }

cudaError_t launch_trop_group(const Dev *dPs, const TileRef *dtiles, int ntiles, int TX, int TY,
                              unsigned long long *cnt, int *err, cudaStream_t s) {
  const size_t smem = trop_fast_smem_bytes(TX, TY);
  const void *fn = group_kernel(TX, TY);
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  // the group's barrier counter starts from zero in every launch
  e = cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  const int nthreads = ((TX + 4) * (TY + 4) + 31) / 32 * 32;
  Dev none{};
  const int ntx = 0;
  const unsigned long long epoch = 0;
  void *args[] = {(void *)&none, (void *)&dPs, (void *)&dtiles, (void *)&TX, (void *)&TY, (void *)&ntx, (void *)&epoch,
                  (void *)&cnt, (void *)&err};
  return cudaLaunchCooperativeKernel(fn, dim3(ntiles), dim3(nthreads), args, smem, s);
}
