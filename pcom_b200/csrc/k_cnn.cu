// k_cnn.cu -- the learned subgrid closure: a 5-layer 3x3 convolutional
// network (input channels u, v, T, S and the specific-volume anomaly per
// model level; 64 hidden channels; outputs the du, dv, dT, dS tendency
// residuals), trained and evaluated with the kernels below.
//
// Every convolution is an implicit GEMM on the 5th-generation tensor cores:
// BF16 operands staged in shared memory in the UMMA "interleave" (no
// swizzle) canonical layout, one elected thread issuing tcgen05.mma
// (kind::f16, FP32 accumulation in tensor memory), completion tracked with
// tcgen05.commit on an mbarrier, and the epilogue reading the accumulator
// with tcgen05.ld.  Forward and data-gradient convolutions are K-major GEMMs
// (rows = pixels, K = tap x input channel, N = output channels); the weight
// gradient is an MN-major GEMM (rows = tap x input channel, N = output
// channels, K = pixels) split over CTAs with FP32 atomics.
//
// Activations are NHWC over images of H x W pixels (one image per model
// level), channels contiguous: 16 (the 5 inputs, zero-padded) or 64.
// Weights are [9 taps][N out][K in] (K contiguous).  Halo: zero padding in
// y and, when periodic_x, wrap-around in x (the zonally periodic grid).
//
// Every wait is bounded: a timed-out mbarrier wait sets the error flag,
// waits (bounded) once more for the MMAs in flight, frees tensor memory and
// returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include <cudaTypedefs.h>

#include "cnn_kernels.h"

namespace {

// polls of an mbarrier before a wait gives up: try_wait may suspend between
// polls (a system-dependent time), test_wait returns at once
constexpr long long kSpin = 1LL << 22, kSpinPoll = 1LL << 26;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// UMMA shared-memory matrix descriptor, no swizzle: start address, leading
// (K-direction core-matrix) byte offset, stride (M/N-direction 8-row group)
// byte offset, each without their 4 low bits; version 1 at bit 46.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// The same for the 128-byte swizzled K-major layout (rows of 128 bytes, the
// 16-byte chunks of row r at position c ^ (r % 8), 1024-byte atoms of 8
// rows): stride byte offset = 1024 (8-row groups), leading byte offset
// unused (1), layout type 2 at bit 61, base offset 0.  The swizzle follows
// the absolute shared-memory address, so an operand may start a whole
// number of rows into an atom with base offset 0 (checked against a CPU
// convolution on the B200; the start address's row phase in the base
// offset field gave wrong results).
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

// Instruction descriptor for kind::f16: D = F32 (bits 4-5 = 1), A = B = BF16
// (bits 7-9 = 1, 10-12 = 1), A/B major (bit 15/16: 0 = K, 1 = MN),
// N >> 3 at bits 17-22, M >> 4 at bits 24-28.
__host__ __device__ constexpr uint32_t umma_idesc(int M, int N, int a_mn, int b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count));
}

// bounded wait for phase `parity` of an mbarrier.  try_wait may suspend the
// thread until the phase completes, so waiting warps give their issue slots
// to the warps that work; mbar_spin polls with test_wait instead, for the
// one thread whose wake-up latency is on the critical path (the MMA issuer
// of the persistent convolution).
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (long long it = 0; it < kSpin; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
__device__ __forceinline__ bool mbar_spin(uint32_t mbar, uint32_t parity) {
  for (long long it = 0; it < kSpinPoll; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, bool valid) {
  const int n = valid ? 16 : 0;  // 0: zero-fill
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(ncols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

// 16 consecutive FP32 accumulator columns of this thread's lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
  for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

// the same, without waiting: issue several, then tmem_ld_wait()
__device__ __forceinline__ void tmem_ld16_nowait(uint32_t taddr, uint32_t *r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// source pixel of tap t (0..8, dy = t/3 - 1, dx = t%3 - 1) for pixel p; -1 if padding
__device__ __forceinline__ long long tap_src(long long p, int t, int H, int W, int periodic_x) {
  const long long hw = (long long)H * W;
  const long long img = p / hw;
  const int rem = (int)(p - img * hw);
  int y = rem / W + (t / 3 - 1), x = rem % W + (t % 3 - 1);
  if (y < 0 || y >= H) return -1;
  if (x < 0 || x >= W) {
    if (!periodic_x) return -1;
    x = (x + W) % W;
  }
  return img * hw + (long long)y * W + x;
}

constexpr int kThreads = 128;  // 4 warps: one TMEM lane quarter each
constexpr int kM = 128;        // pixels (fwd/dgrad) or tap x channel rows (wgrad) per tile

// ----------------------------------------------------------------------------
// Forward / data-gradient convolution: out[p][n] = sum_t sum_c in[src(p, t)][c] w[t][n][c]
// mode 0: + bias, ReLU, BF16 out (stride NOUT)
// mode 1: + bias, FP32 out, first nstore channels (stride nstore)
// mode 2: ReLU mask from aux (BF16, stride NOUT): out = acc * (aux > 0), BF16
template <int CIN, int NOUT>
__global__ void __launch_bounds__(kThreads) k_conv_tc(const __nv_bfloat16 *__restrict__ in,
                                                      const __nv_bfloat16 *__restrict__ w,
                                                      const float *__restrict__ bias, const __nv_bfloat16 *__restrict__ aux,
                                                      void *out, long long npix, int H, int W, int periodic_x, int mode,
                                                      int nstore, int *err) {
  constexpr int KC = CIN / 8;                 // 16-byte chunks per pixel per tap
  constexpr int A_BYTES = kM * CIN * 2;
  constexpr int B_BYTES = NOUT * CIN * 2;
  constexpr int STAGE = A_BYTES + B_BYTES;
  constexpr uint32_t NCOLS = NOUT < 32 ? 32 : NOUT;
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t tmem_slot;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const long long p0 = (long long)blockIdx.x * kM;

  if (warp == 0) tmem_alloc(smem_u32(&tmem_slot), NCOLS);
  if (tid == 0) {
    mbar_init(smem_u32(&mbar[0]), 1);
    mbar_init(smem_u32(&mbar[1]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  constexpr uint32_t idesc = umma_idesc(kM, NOUT, 0, 0);
  uint32_t phase[2] = {0, 0};
  bool ok = true;

  for (int t = 0; t < 9; ++t) {
    const int s = t & 1;
    uint8_t *A = smem + s * STAGE, *B = A + A_BYTES;
    if (t >= 2) {  // the MMAs of tap t-2 read this stage
      if (!mbar_wait(smem_u32(&mbar[s]), phase[s])) ok = false;
      phase[s] ^= 1;
    }
    // A: 128 pixels x KC chunks, core matrix (g, c) at ((g*KC + c) * 128) + (m%8)*16
    for (int q = tid; q < kM * KC; q += kThreads) {
      const int m = q / KC, c = q % KC;
      const long long p = p0 + m;
      long long src = p < npix ? tap_src(p, t, H, W, periodic_x) : -1;
      if (src >= npix) src = -1;  // a partial last image: missing pixels are zero
      const uint32_t dst = smem_u32(A) + (uint32_t)(((m / 8) * KC + c) * 128 + (m % 8) * 16);
      cp_async16(dst, src >= 0 ? (const void *)(in + src * CIN + c * 8) : (const void *)in, src >= 0);
    }
    // B: NOUT rows x KC chunks of tap t
    for (int q = tid; q < NOUT * KC; q += kThreads) {
      const int n = q / KC, c = q % KC;
      const uint32_t dst = smem_u32(B) + (uint32_t)(((n / 8) * KC + c) * 128 + (n % 8) * 16);
      cp_async16(dst, w + ((long long)t * NOUT + n) * CIN + c * 8, true);
    }
    cp_async_wait_all();
    fence_async_smem();
    __syncthreads();
    if (tid == 0 && ok) {
      tc_fence_after();
      #pragma unroll
      for (int j = 0; j < CIN / 16; ++j) {
        const uint64_t ad = umma_desc(smem_u32(A) + j * 256, 128, KC * 128);
        const uint64_t bd = umma_desc(smem_u32(B) + j * 256, 128, KC * 128);
        umma_bf16(tmem, ad, bd, idesc, (t > 0 || j > 0) ? 1u : 0u);
      }
      umma_commit(smem_u32(&mbar[s]));
    }
    __syncthreads();
  }
  // the last commit (tap 8, stage 0) covers every MMA issued before it
  if (!mbar_wait(smem_u32(&mbar[0]), phase[0])) ok = false;
  if (!mbar_wait(smem_u32(&mbar[1]), phase[1])) ok = false;
  tc_fence_after();
  if (!ok) {
    if (tid == 0) atomicExch(err, 1);
  } else {
    const int row = warp * 32 + lane;
    const long long p = p0 + row;
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
    #pragma unroll
    for (int c0 = 0; c0 < NOUT; c0 += 16) {
      float v[16];
      tmem_ld16(lane_addr + c0, v);
      if (p < npix) {
        if (mode == 0) {
          __nv_bfloat16 *o = (__nv_bfloat16 *)out + p * NOUT + c0;
          #pragma unroll
          for (int q = 0; q < 16; ++q) o[q] = __float2bfloat16(fmaxf(v[q] + bias[c0 + q], 0.f));
        } else if (mode == 1) {
          float *o = (float *)out + p * nstore;
          for (int q = 0; q < 16; ++q)
            if (c0 + q < nstore) o[c0 + q] = v[q] + bias[c0 + q];
        } else {
          __nv_bfloat16 *o = (__nv_bfloat16 *)out + p * NOUT + c0;
          const __nv_bfloat16 *a = aux + p * NOUT + c0;
          #pragma unroll
          for (int q = 0; q < 16; ++q) o[q] = __float2bfloat16(__bfloat162float(a[q]) > 0.f ? v[q] : 0.f);
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, NCOLS);
}

// Ring geometry of the persistent convolution below: a tile is 128
// consecutive pixels of one image row, its halo rows hold 130 pixels, stored
// "chunk-planar" (plane c holds channels 8c..8c+7, 16 bytes per pixel).
constexpr int kHaloW = kM + 2;               // halo columns
constexpr int kRowB = kHaloW * 16;           // one slot of one plane (2,080 bytes)

// ----------------------------------------------------------------------------
// Persistent convolution (the form every whole-image convolution takes).
// Each CTA walks a contiguous strip of tiles down the rows of one column of
// tiles, so consecutive tiles share two of their three halo rows: the rows
// live in a ring of slots, each tile loads one new row, and the A operand of
// tap (dy, dx) is the planes of the slot holding row y + dy read from pixel
// dx + 1 (leading byte offset = plane stride, stride byte offset = 128 bytes
// = 8 pixels).  Taps whose row falls outside the image are skipped.  All 9
// taps of the weights stay in shared memory.  Two accumulators in tensor
// memory let the MMAs of one tile run while the previous one is drained.
// Each role has its own warps and
// they hand work to one another through mbarriers instead of CTA barriers
// (six ring slots instead of four, so row loads run up to three tiles ahead):
//   warps 0-7  epilogue: warp w drains half the columns (w / 4) of lane
//              quarter w % 4 of an accumulator (tcgen05.ld, all issued
//              before one wait), frees it, applies bias + ReLU (or the ReLU
//              mask) and stores the tile; 64-channel BF16 tiles go through a
//              double-buffered staging tile in the 128-byte swizzled layout
//              and leave with one TMA tensor store (cp.async.bulk.tensor)
//   warps 8-11 loads: stream each new halo row into its ring slot with
//              cp.async, whose completion arrives on the slot's "full"
//              mbarrier; reuse a slot once the MMAs reading its old row have
//              completed ("empty" mbarrier, tcgen05.commit).  One warp's
//              cp.async stream delivered a 16.6 KB row per ~5,500 cycles,
//              slower than the tile's MMAs (clock64 timestamps per role);
//              four keep the MMA thread supplied
//   warp 12    MMA: one thread (the only one that polls: the others wait
//              suspended, which leaves it the issue slots; with every waiter
//              polling, it took ~95 cycles to issue each MMA) waits for the tile's rows and a free
//              accumulator, issues the 9 taps x CIN/16 MMAs and commits
//              "accumulator full" and the release of the rows the next tile
//              does not read.
// The plane stride of the ring is padded by 16 bytes so a load warp's eight
// 16-byte chunks of one pixel land in different banks.  Every wait is
// bounded: a wait that gives up sets the error flag and a shared stop flag,
// and every role leaves its loop; the MMA thread then waits (bounded) for its
// MMAs before tensor memory is freed.
constexpr int kLoadWarps = 4;    // one warp's cp.async stream cannot keep a row per tile in flight
constexpr int kWsThreads = (8 + kLoadWarps + 1) * 32;  // 8 epilogue warps, the load warps, 1 MMA warp
constexpr int kWsRing = 6;                     // halo row slots: loads run up to three tiles ahead
constexpr int kPlaneW = kWsRing * kRowB + 16;  // padded ring plane (12,496 bytes)
// 64-channel inputs: a slot is 130 pixel rows of 128 bytes in the 128-byte
// swizzled layout, 1024-byte aligned (17 KB), so a tap's one-pixel shift
// moves the A operand by whole 128-byte rows; in the plane layout the
// shifted operand started 16 or 32 bytes into its 128-byte core matrices
// and each MMA read took about twice as long
constexpr int kSlotSW = 17 * 1024;
template <int CIN>
__host__ __device__ constexpr bool ring_sw() { return CIN == 64; }
template <int CIN>
__host__ __device__ constexpr int ring_bytes() { return ring_sw<CIN>() ? kWsRing * kSlotSW : (CIN / 8) * kPlaneW; }

__device__ __forceinline__ void cp_async_arrive_noinc(uint32_t mbar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(mbar) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}
__device__ __forceinline__ void tma_store3(const CUtensorMap *map, uint32_t src, int c0, int c1, int c2) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(map),
               "r"(src), "r"(c0), "r"(c1), "r"(c2)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read1() { asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

template <int CIN, int NOUT>
__host__ __device__ constexpr bool ws_tma() { return NOUT == 64; }

template <int CIN, int NOUT>
__global__ void __launch_bounds__(kWsThreads) k_conv_ws(const __nv_bfloat16 *__restrict__ in,
                                                        const __nv_bfloat16 *__restrict__ w,
                                                        const float *__restrict__ bias,
                                                        const __nv_bfloat16 *__restrict__ aux, void *out, int nimg,
                                                        int H, int W, int periodic_x, int mode, int nstore, int *err,
                                                        const __grid_constant__ CUtensorMap tmap) {
  constexpr int KC = CIN / 8;
  constexpr int W_BYTES = 9 * NOUT * CIN * 2;
  constexpr int STG = kM * NOUT * 2;  // one staging tile
  constexpr uint32_t NCOLS = NOUT < 32 ? 32 : NOUT;
  constexpr int NSPLIT = NOUT >= 32 ? 2 : 1;  // epilogue warps per lane quarter
  constexpr int CPW = NOUT / NSPLIT;          // accumulator columns per epilogue warp
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ float s_bias[NOUT];
  __shared__ __align__(8) uint64_t full[kWsRing], empty[kWsRing], accf[2], acce[2], sfree[2], swritten[2], done;
  __shared__ uint32_t tmem_slot;
  __shared__ volatile int s_stop;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  // 1024-byte aligned base: the swizzled staging tiles need it
  const uint32_t base = (smem_u32(smem_raw) + 1023u) & ~1023u;
  uint8_t *const sbase = smem_raw + (base - smem_u32(smem_raw));
  const bool tma = ws_tma<CIN, NOUT>() && mode != 1;
  static_assert(!ring_sw<CIN>() || (W_BYTES % 1024 == 0 && STG % 1024 == 0), "swizzled ring slots need 1024-byte alignment");
  const uint32_t Stg = base, Wsm = base + (ws_tma<CIN, NOUT>() ? 2 * STG : 0), Ring = Wsm + W_BYTES;
  uint8_t *const stg_p = sbase;
  const int ntx = (W + kM - 1) / kM;
  const long long NR = (long long)nimg * H;
  const long long ntiles = NR * ntx;
  const long long chunk = (ntiles + gridDim.x - 1) / gridDim.x;
  const long long t0 = (long long)blockIdx.x * chunk;
  const long long t1 = t0 + chunk < ntiles ? t0 + chunk : ntiles;

  if (warp == 0) tmem_alloc(smem_u32(&tmem_slot), 2 * NCOLS);
  if (tid == 0) {
    for (int q = 0; q < kWsRing; ++q) {
      mbar_init(smem_u32(&full[q]), 32 * kLoadWarps);  // one arrival per load thread
      mbar_init(smem_u32(&empty[q]), 1);
    }
    for (int q = 0; q < 2; ++q) {
      mbar_init(smem_u32(&accf[q]), 1);
      mbar_init(smem_u32(&acce[q]), 4 * NSPLIT);      // one per epilogue warp
      mbar_init(smem_u32(&sfree[q]), 1);              // staging tile q read by its last store
      mbar_init(smem_u32(&swritten[q]), 4 * NSPLIT);  // staging tile q written (one arrival per epilogue warp)
    }
    mbar_init(smem_u32(&done), 1);
    s_stop = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // weights (all threads), resident for the kernel's lifetime
  for (int q = tid; q < 9 * NOUT * KC; q += kWsThreads) {
    const int t = q / (NOUT * KC), r = q % (NOUT * KC), n = r / KC, c = r % KC;
    cp_async16(Wsm + (uint32_t)(t * NOUT * CIN * 2 + ((n / 8) * KC + c) * 128 + (n % 8) * 16),
               w + ((long long)t * NOUT + n) * CIN + c * 8, true);
  }
  for (int q = tid; q < NOUT; q += kWsThreads) s_bias[q] = mode == 2 ? 0.f : bias[q];
  cp_async_wait_all();
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;

  struct Pos {
    int tx, gr, y;
  };
  auto advance = [&](Pos a) {
    ++a.gr;
    if (++a.y == H) a.y = 0;
    if (a.gr == (int)NR) {
      a.gr = 0;
      a.y = 0;
      ++a.tx;
    }
    return a;
  };
  auto row_used = [&](const Pos &a, int dy) { return a.y + dy >= 0 && a.y + dy < H; };
  Pos first{0, 0, 0};
  if (t0 < t1) {
    first.tx = (int)(t0 / NR);
    first.gr = (int)(t0 % NR);
    first.y = first.gr % H;
  }
  auto stop = [&]() {
    s_stop = 1;
    atomicExch(err, 1);
  };

  if (warp >= 8 && warp < 8 + kLoadWarps) {
    // ---------------------------------------------------------------- loads
    const int lt = tid - 8 * 32;  // load thread 0 .. 32 * kLoadWarps - 1
    int tag_row[kWsRing], tag_tx[kWsRing], nload[kWsRing];
    for (int q = 0; q < kWsRing; ++q) tag_row[q] = tag_tx[q] = -1, nload[q] = 0;
    Pos a = first;
    for (long long tile = t0; tile < t1 && !s_stop; ++tile, a = advance(a)) {
      for (int dy = -1; dy <= 1; ++dy) {
        if (!row_used(a, dy)) continue;
        const int r = a.gr + dy, s = r % kWsRing;
        if (tag_row[s] == r && tag_tx[s] == a.tx) continue;
        // the slot's previous row is free once the MMAs that read it are done
        if (nload[s] > 0 && !mbar_wait(smem_u32(&empty[s]), (uint32_t)((nload[s] - 1) & 1))) {
          stop();
          break;
        }
        const int x0 = a.tx * kM;
        for (int q = lt; q < kHaloW * KC; q += 32 * kLoadWarps) {
          const int u = q / KC, c = q % KC;
          int xx = x0 - 1 + u;
          bool ok = true;
          if (xx < 0 || xx >= W) {
            if (periodic_x) {
              if (xx < 0) xx += W;
              else if ((xx -= W) >= W) xx %= W;
            } else {
              ok = false;
            }
          }
          const uint32_t dst = ring_sw<CIN>() ? Ring + (uint32_t)(s * kSlotSW + u * 128 + ((c ^ (u & 7)) << 4))
                                              : Ring + (uint32_t)(c * kPlaneW + s * kRowB + u * 16);
          cp_async16(dst, ok ? (const void *)(in + ((long long)r * W + xx) * CIN + c * 8) : (const void *)in, ok);
        }
        cp_async_arrive_noinc(smem_u32(&full[s]));
        tag_row[s] = r;
        tag_tx[s] = a.tx;
        ++nload[s];
      }
    }
    cp_async_wait_all();
  } else if (warp == 8 + kLoadWarps) {
    // ------------------------------------------------------------------ MMA
    if (lane == 0) {
      constexpr uint32_t idesc = umma_idesc(kM, NOUT, 0, 0);
      const uint64_t adesc0 = umma_desc(Ring, kPlaneW, 128);
      const uint64_t bdesc0 = umma_desc(Wsm, 128, KC * 128);
      int tag_row[kWsRing], tag_tx[kWsRing], nload[kWsRing];
      for (int q = 0; q < kWsRing; ++q) tag_row[q] = tag_tx[q] = -1, nload[q] = 0;
      bool issued = false;
      Pos a = first;
      int it = 0;
      for (long long tile = t0; tile < t1 && !s_stop; ++tile, ++it, a = advance(a)) {
        const int b = it & 1;
        bool ok = true;
        for (int dy = -1; dy <= 1 && ok; ++dy) {
          if (!row_used(a, dy)) continue;
          const int r = a.gr + dy, s = r % kWsRing;
          if (tag_row[s] == r && tag_tx[s] == a.tx) continue;
          tag_row[s] = r;
          tag_tx[s] = a.tx;
          ++nload[s];
          ok = mbar_spin(smem_u32(&full[s]), (uint32_t)((nload[s] - 1) & 1));
        }
        // accumulator b was last drained for tile it - 2
        if (ok && it >= 2) ok = mbar_spin(smem_u32(&acce[b]), (uint32_t)(((it >> 1) - 1) & 1));
        if (!ok) {
          stop();
          break;
        }
        // the rows arrived through cp.async (generic proxy); the MMAs read
        // them through the async proxy
        fence_async_smem();
        tc_fence_after();
        uint32_t accum = 0;
        #pragma unroll
        for (int tp = 0; tp < 9; ++tp) {
          const int dy = tp / 3 - 1, dx = tp % 3 - 1;
          if (!row_used(a, dy)) continue;
          const int s = (a.gr + dy) % kWsRing;
          #pragma unroll
          for (int j = 0; j < CIN / 16; ++j) {
            const uint64_t ad = ring_sw<CIN>()
                                    ? umma_desc_sw128(Ring + (uint32_t)(s * kSlotSW + (dx + 1) * 128 + j * 32))
                                    : adesc0 + (uint64_t)((s * kRowB + (dx + 1) * 16 + 2 * j * kPlaneW) >> 4);
            const uint64_t bd = bdesc0 + (uint64_t)((tp * NOUT * CIN * 2 + j * 256) >> 4);
            umma_bf16(tmem + (uint32_t)b * NCOLS, ad, bd, idesc, accum);
            accum = 1u;
          }
        }
        umma_commit(smem_u32(&accf[b]));
        issued = true;
        // release the rows the next tile does not read
        if (tile + 1 < t1) {
          const Pos n = advance(a);
          for (int dy = -1; dy <= 1; ++dy) {
            if (!row_used(a, dy)) continue;
            const int r = a.gr + dy;
            const int ndy = r - n.gr;
            const bool kept = n.tx == a.tx && ndy >= -1 && ndy <= 1 && row_used(n, ndy);
            if (!kept) umma_commit(smem_u32(&empty[r % kWsRing]));
          }
        }
      }
      // every MMA issued has completed before tensor memory is freed
      if (issued) {
        umma_commit(smem_u32(&done));
        if (!mbar_wait(smem_u32(&done), 0)) atomicExch(err, 1);
      }
    }
  } else {
    // ------------------------------------------------------------- epilogue
    const int quarter = warp & 3, half = warp >> 2;  // lane quarter, column half
    const int m = quarter * 32 + lane;
    const int c_lo = half * CPW;                       // this warp's first column
    Pos a = first;
    int it = 0;
    for (long long tile = t0; tile < t1 && !s_stop && half < NSPLIT; ++tile, ++it, a = advance(a)) {
      const int b = it & 1;
      const int x0 = a.tx * kM, x = x0 + m;
      const long long p = (long long)a.gr * W + x;
      // the ReLU mask of this pixel's columns, fetched before the wait
      uint4 am[CPW / 8];
      if (mode == 2) {
        #pragma unroll
        for (int c = 0; c < CPW / 8; ++c)
          am[c] = x < W ? __ldg(reinterpret_cast<const uint4 *>(aux + p * NOUT + c_lo) + c) : make_uint4(0, 0, 0, 0);
      }
      const bool ok = mbar_wait(smem_u32(&accf[b]), (uint32_t)((it >> 1) & 1));
      if (!ok) stop();
      if (__any_sync(0xffffffffu, !ok)) break;
      tc_fence_after();
      uint32_t r[CPW];
      const uint32_t lane_addr = tmem + (uint32_t)b * NCOLS + ((uint32_t)(quarter * 32) << 16) + (uint32_t)c_lo;
      #pragma unroll
      for (int c0 = 0; c0 < CPW; c0 += 16) tmem_ld16_nowait(lane_addr + c0, r + c0);
      tmem_ld_wait();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&acce[b]));
      if (mode == 1) {
        if (x < W && c_lo < nstore) {
          float *o = (float *)out + p * nstore;
          if (nstore == 4 && c_lo == 0) {
            *reinterpret_cast<float4 *>(o) =
                make_float4(__uint_as_float(r[0]) + s_bias[0], __uint_as_float(r[1]) + s_bias[1],
                            __uint_as_float(r[2]) + s_bias[2], __uint_as_float(r[3]) + s_bias[3]);
          } else {
            #pragma unroll
            for (int q = 0; q < CPW; ++q)
              if (c_lo + q < nstore) o[c_lo + q] = __uint_as_float(r[q]) + s_bias[c_lo + q];
          }
        }
        continue;
      }
      uint32_t pk[CPW / 2];
      #pragma unroll
      for (int q = 0; q < CPW / 2; ++q) {
        const float v0 = __uint_as_float(r[2 * q]), v1 = __uint_as_float(r[2 * q + 1]);
        float lo, hi;
        if (mode == 0) {
          lo = fmaxf(v0 + s_bias[c_lo + 2 * q], 0.f);
          hi = fmaxf(v1 + s_bias[c_lo + 2 * q + 1], 0.f);
        } else {
          const uint32_t aw = (&am[q / 4].x)[q % 4];
          const __nv_bfloat162 a2 = *reinterpret_cast<const __nv_bfloat162 *>(&aw);
          lo = __low2float(a2) > 0.f ? v0 : 0.f;
          hi = __high2float(a2) > 0.f ? v1 : 0.f;
        }
        const __nv_bfloat162 b2 = __floats2bfloat162_rn(lo, hi);
        pk[q] = *reinterpret_cast<const uint32_t *>(&b2);
      }
      if (!tma) {
        if (x < W) {
          uint4 *o = reinterpret_cast<uint4 *>((__nv_bfloat16 *)out + p * NOUT + c_lo);
          #pragma unroll
          for (int c = 0; c < CPW / 8; ++c) o[c] = make_uint4(pk[4 * c], pk[4 * c + 1], pk[4 * c + 2], pk[4 * c + 3]);
        }
        continue;
      }
      // staging tile it & 1: the store issued from it two tiles ago has read
      // it (thread 0 issues every store, so it is the one that can tell)
      const int sb = it & 1;
      if (it >= 2) {
        if (tid == 0) {
          bulk_wait_read1();
          mbar_arrive(smem_u32(&sfree[sb]));
        }
        if (!mbar_wait(smem_u32(&sfree[sb]), (uint32_t)(((it >> 1) - 1) & 1))) {
          stop();
          break;
        }
      }
      uint8_t *row = stg_p + sb * STG + m * 128;
      #pragma unroll
      for (int c = 0; c < CPW / 8; ++c) {  // 16-byte chunk cc of the pixel's 128 bytes, 128-byte swizzle
        const int cc = c_lo / 8 + c;
        *reinterpret_cast<uint4 *>(row + ((cc ^ (m & 7)) << 4)) =
            make_uint4(pk[4 * c], pk[4 * c + 1], pk[4 * c + 2], pk[4 * c + 3]);
      }
      fence_async_smem();  // this thread's staging writes, ordered before the TMA store reads them
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&swritten[sb]));
      if (tid == 0) {
        if (!mbar_wait(smem_u32(&swritten[sb]), (uint32_t)((it >> 1) & 1))) {
          stop();
          break;
        }
        tma_store3(&tmap, Stg + (uint32_t)(sb * STG), 0, x0, a.gr);
        bulk_commit();
      }
    }
    if (tid == 0) bulk_wait_all();
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, 2 * NCOLS);
}

// ----------------------------------------------------------------------------
// Weight gradient: dw[t][n][c] += sum_p in[src(p, t)][c] g[p][n]
// Tile rows r = (t - t0) * CIN + c for TPT = 128 / CIN taps starting at
// t0 = blockIdx.y * TPT; K = pixels, 64 per stage; CTA x covers ppc pixels.
template <int CIN, int NOUT>
__global__ void __launch_bounds__(kThreads) k_wgrad_tc(const __nv_bfloat16 *__restrict__ in,
                                                       const __nv_bfloat16 *__restrict__ g, float *dw, long long npix,
                                                       int H, int W, int periodic_x, long long ppc, int *err) {
  constexpr int TPT = kM / CIN;
  constexpr int KP = 64;                  // pixels per stage
  constexpr int KG = KP / 8;              // K groups (8 pixels) per stage
  constexpr int A_BYTES = kM * KP * 2;    // 128 rows x 64 pixels
  constexpr int B_BYTES = NOUT * KP * 2;
  constexpr int STAGE = A_BYTES + B_BYTES;
  constexpr uint32_t NCOLS = NOUT < 32 ? 32 : NOUT;
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t tmem_slot;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int t0 = blockIdx.y * TPT;
  const long long pbeg = (long long)blockIdx.x * ppc;
  const long long pend = min(npix, pbeg + ppc);
  const int nstage = (int)((pend - pbeg + KP - 1) / KP);

  if (warp == 0) tmem_alloc(smem_u32(&tmem_slot), NCOLS);
  if (tid == 0) {
    mbar_init(smem_u32(&mbar[0]), 1);
    mbar_init(smem_u32(&mbar[1]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  constexpr uint32_t idesc = umma_idesc(kM, NOUT, 1, 1);
  uint32_t phase[2] = {0, 0};
  bool ok = true;
  int issued[2] = {0, 0};

  for (int st = 0; st < nstage; ++st) {
    const int s = st & 1;
    uint8_t *A = smem + s * STAGE, *B = A + A_BYTES;
    if (st >= 2) {
      if (!mbar_wait(smem_u32(&mbar[s]), phase[s])) ok = false;
      phase[s] ^= 1;
    }
    const long long pk = pbeg + (long long)st * KP;
    // A (MN-major): core (g, kg) = 8 pixels x 8 channels at (g*KG + kg)*128,
    // pixel k of the group at k*16; row group g = (tap, channel chunk)
    for (int q = tid; q < (kM / 8) * KP; q += kThreads) {
      const int g = q / KP, k = q % KP;
      const int r0 = g * 8, t = t0 + r0 / CIN, c = r0 % CIN;
      const long long p = pk + k;
      long long src = (t < 9 && p < pend) ? tap_src(p, t, H, W, periodic_x) : -1;
      if (src >= npix) src = -1;
      const uint32_t dst = smem_u32(A) + (uint32_t)((g * KG + k / 8) * 128 + (k % 8) * 16);
      cp_async16(dst, src >= 0 ? (const void *)(in + src * CIN + c) : (const void *)in, src >= 0);
    }
    // B (MN-major): core (gn, kg) = 8 pixels x 8 output channels
    for (int q = tid; q < (NOUT / 8) * KP; q += kThreads) {
      const int gn = q / KP, k = q % KP;
      const long long p = pk + k;
      const uint32_t dst = smem_u32(B) + (uint32_t)((gn * KG + k / 8) * 128 + (k % 8) * 16);
      cp_async16(dst, p < pend ? (const void *)(g + p * NOUT + gn * 8) : (const void *)g, p < pend);
    }
    cp_async_wait_all();
    fence_async_smem();
    __syncthreads();
    if (tid == 0 && ok) {
      tc_fence_after();
      #pragma unroll
      for (int j = 0; j < KP / 16; ++j) {
        const uint64_t ad = umma_desc(smem_u32(A) + j * 256, 128, KG * 128);
        const uint64_t bd = umma_desc(smem_u32(B) + j * 256, 128, KG * 128);
        umma_bf16(tmem, ad, bd, idesc, (st > 0 || j > 0) ? 1u : 0u);
      }
      umma_commit(smem_u32(&mbar[s]));
    }
    issued[s]++;
    __syncthreads();
  }
  for (int s = 0; s < 2; ++s)
    if (issued[s] > 0 && nstage > 0) {
      // stages s, s+2, ...: the outstanding phase of mbar[s] is the last one
      if (!mbar_wait(smem_u32(&mbar[s]), phase[s])) ok = false;
    }
  tc_fence_after();
  if (!ok) {
    if (tid == 0) atomicExch(err, 1);
  } else if (nstage > 0) {
    const int row = warp * 32 + lane;
    const int t = t0 + row / CIN, c = row % CIN;
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
    #pragma unroll
    for (int c0 = 0; c0 < NOUT; c0 += 16) {
      float v[16];
      tmem_ld16(lane_addr + c0, v);
      if (t < 9)
        for (int q = 0; q < 16; ++q) atomicAdd(dw + ((long long)t * NOUT + c0 + q) * CIN + c, v[q]);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, NCOLS);
}

// dynamic shared memory per CTA; with 64 accumulator columns at least 29 KB,
// so that at most 7 CTAs share an SM's 512 tensor-memory columns
template <int NOUT>
size_t smem_floor(size_t b) { return NOUT > 32 && b < 29 * 1024 ? 29 * 1024 : b; }
template <int CIN, int NOUT>
size_t conv_smem() { return smem_floor<NOUT>(2 * (size_t)(kM * CIN * 2 + NOUT * CIN * 2)); }
template <int CIN, int NOUT>
size_t wgrad_smem() { return smem_floor<NOUT>(2 * (size_t)(kM * 64 * 2 + NOUT * 64 * 2)); }

template <int CIN, int NOUT>
size_t ws_smem() {
  return 1024 + (ws_tma<CIN, NOUT>() ? 2 * (size_t)kM * NOUT * 2 : 0) + (size_t)9 * NOUT * CIN * 2 +
         (size_t)ring_bytes<CIN>();  // 64 -> 64: 1 + 32 + 72 + 102 KB
}

// cuTensorMapEncodeTiled through the runtime's driver entry-point table (the
// library links no libcuda)
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return (PFN_cuTensorMapEncodeTiled_v12000)f;
  }();
  return fn;
}

template <int CIN, int NOUT>
cudaError_t conv_ws_launch(const __nv_bfloat16 *in, const __nv_bfloat16 *w, const float *bias,
                           const __nv_bfloat16 *aux, void *out, long long npix, int H, int W, int periodic_x, int mode,
                           int nstore, int *err, cudaStream_t s) {
  const size_t sm = ws_smem<CIN, NOUT>();
  cudaError_t e = cudaFuncSetAttribute(k_conv_ws<CIN, NOUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  const long long hw = (long long)H * W;
  const int nimg = (int)(npix / hw);
  const long long NR = (long long)nimg * H;
  const long long ntiles = NR * ((W + kM - 1) / kM);
  // output tensor map: [image rows][W][NOUT] BF16, box = one tile (128 pixels
  // x 64 channels), 128-byte swizzle; pixels past W in a tile are not stored
  CUtensorMap tm;
  memset(&tm, 0, sizeof tm);
  if (ws_tma<CIN, NOUT>() && mode != 1) {
    auto enc = tensor_map_encoder();
    if (!enc || NR > 0x7fffffffLL || ((uintptr_t)out & 15u)) return cudaErrorInvalidValue;
    const cuuint64_t dims[3] = {(cuuint64_t)NOUT, (cuuint64_t)W, (cuuint64_t)NR};
    const cuuint64_t strides[2] = {(cuuint64_t)NOUT * 2, (cuuint64_t)W * NOUT * 2};
    const cuuint32_t box[3] = {(cuuint32_t)NOUT, (cuuint32_t)kM, 1u};
    const cuuint32_t estr[3] = {1u, 1u, 1u};
    if (enc(&tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, out, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return cudaErrorInvalidValue;
  }
  int dev = 0, nsm = 148, per = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_conv_ws<CIN, NOUT>, kWsThreads, sm);
  const int tmem_cap = 512 / (2 * (NOUT < 32 ? 32 : NOUT));
  per = per < 1 ? 1 : (per > tmem_cap ? tmem_cap : per);
  const long long grid = ntiles < (long long)nsm * per ? ntiles : (long long)nsm * per;
  k_conv_ws<CIN, NOUT><<<(unsigned)grid, kWsThreads, sm, s>>>(in, w, bias, aux, out, nimg, H, W, periodic_x, mode,
                                                               nstore, err, tm);
  return cudaGetLastError();
}

template <int CIN, int NOUT>
cudaError_t conv_launch(const __nv_bfloat16 *in, const __nv_bfloat16 *w, const float *bias, const __nv_bfloat16 *aux,
                        void *out, long long npix, int H, int W, int periodic_x, int mode, int nstore, int *err,
                        cudaStream_t s) {
  // whole images: the persistent warp-specialised form
  if (npix % ((long long)H * W) == 0)
    return conv_ws_launch<CIN, NOUT>(in, w, bias, aux, out, npix, H, W, periodic_x, mode, nstore, err, s);
  const size_t sm = conv_smem<CIN, NOUT>();
  cudaError_t e = cudaFuncSetAttribute(k_conv_tc<CIN, NOUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  const unsigned grid = (unsigned)((npix + kM - 1) / kM);
  k_conv_tc<CIN, NOUT><<<grid, kThreads, sm, s>>>(in, w, bias, aux, out, npix, H, W, periodic_x, mode, nstore, err);
  return cudaGetLastError();
}

template <int CIN, int NOUT>
cudaError_t wgrad_launch(const __nv_bfloat16 *in, const __nv_bfloat16 *g, float *dw, long long npix, int H, int W,
                         int periodic_x, int *err, cudaStream_t s) {
  const size_t sm = wgrad_smem<CIN, NOUT>();
  cudaError_t e = cudaFuncSetAttribute(k_wgrad_tc<CIN, NOUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  constexpr int TPT = kM / CIN;
  const int ytiles = (9 + TPT - 1) / TPT;
  // split K over about 4 waves of CTAs; pixels per CTA a multiple of 64
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  long long target = (long long)nsm * 8 / ytiles;
  if (target < 1) target = 1;
  long long ppc = (npix + target - 1) / target;
  ppc = (ppc + 63) / 64 * 64;
  if (ppc < 64) ppc = 64;
  const unsigned gx = (unsigned)((npix + ppc - 1) / ppc);
  k_wgrad_tc<CIN, NOUT><<<dim3(gx, ytiles), kThreads, sm, s>>>(in, g, dw, npix, H, W, periodic_x, ppc, err);
  return cudaGetLastError();
}

}  // namespace

cudaError_t cnn_conv(int cin, int nout, const __nv_bfloat16 *in, const __nv_bfloat16 *w, const float *bias,
                     const __nv_bfloat16 *aux, void *out, long long npix, int H, int W, int periodic_x, int mode,
                     int nstore, int *err, cudaStream_t s) {
  if (cin == 16 && nout == 64) return conv_launch<16, 64>(in, w, bias, aux, out, npix, H, W, periodic_x, mode, nstore, err, s);
  if (cin == 64 && nout == 64) return conv_launch<64, 64>(in, w, bias, aux, out, npix, H, W, periodic_x, mode, nstore, err, s);
  if (cin == 64 && nout == 16) return conv_launch<64, 16>(in, w, bias, aux, out, npix, H, W, periodic_x, mode, nstore, err, s);
  if (cin == 16 && nout == 16) return conv_launch<16, 16>(in, w, bias, aux, out, npix, H, W, periodic_x, mode, nstore, err, s);
  return cudaErrorInvalidValue;
}

cudaError_t cnn_wgrad(int cin, int nout, const __nv_bfloat16 *in, const __nv_bfloat16 *g, float *dw, long long npix,
                      int H, int W, int periodic_x, int *err, cudaStream_t s) {
  if (cin == 16 && nout == 64) return wgrad_launch<16, 64>(in, g, dw, npix, H, W, periodic_x, err, s);
  if (cin == 64 && nout == 64) return wgrad_launch<64, 64>(in, g, dw, npix, H, W, periodic_x, err, s);
  if (cin == 64 && nout == 16) return wgrad_launch<64, 16>(in, g, dw, npix, H, W, periodic_x, err, s);
  return cudaErrorInvalidValue;
}
