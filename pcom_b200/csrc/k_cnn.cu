// k_cnn.cu -- the learned subgrid closure: a 5-layer 3x3 convolutional
// network (input channels u, v, T, S and the specific-volume anomaly per
// model level; 64 hidden channels; outputs the du, dv, dT, dS tendency
// residuals), trained and evaluated with the kernels below.
//
// Every convolution is an implicit GEMM on the 5th-generation tensor cores:
// BF16 operands staged in shared memory in a UMMA canonical layout (128-byte
// swizzle for 64-channel rows brought in by TMA tensor loads, "interleave"
// without swizzle otherwise), one elected thread issuing tcgen05.mma
// (kind::f16, FP32 accumulation in tensor memory), completion tracked with
// tcgen05.commit on mbarriers, and the epilogue reading the accumulator
// with tcgen05.ld and writing 64-channel rows with TMA tensor stores.
// Forward and data-gradient convolutions are K-major GEMMs (rows = pixels,
// K = input channel, N = the three row taps x output channels, summed over
// the three column taps); the weight gradient is an MN-major GEMM (rows =
// tap x input channel, N = output channels, K = pixels) split over CTAs with
// FP32 atomics.
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

// one test each of two mbarrier phases, issued together so that their
// latencies overlap; bit 0 = the first complete, bit 1 = the second
__device__ __forceinline__ uint32_t mbar_test2(uint32_t mbar0, uint32_t parity0, uint32_t mbar1, uint32_t parity1) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t.reg .b32 a, b;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 q, [%3], %4;\n\t"
      "selp.b32 a, 1, 0, p;\n\tselp.b32 b, 2, 0, q;\n\tor.b32 %0, a, b;\n\t}\n"
      : "=r"(done)
      : "r"(mbar0), "r"(parity0), "r"(mbar1), "r"(parity1)
      : "memory");
  return done;
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

// ----------------------------------------------------------------------------
// Persistent row-streaming convolution (the form every whole-image
// convolution takes).
//
// A tile is 128 consecutive pixels of one image row (tile column tx covers
// pixels 128 tx ..); each CTA owns a contiguous run of output rows of one or
// two tile columns.  Instead of gathering three input rows per output row,
// it streams every input row once and multiplies it by the weights of all
// three row taps at once: for input row i the B operand stacks the weights
// of taps dy = -1, 0, +1 (target t = dy + 1), so one MMA with N = 3 x BW
// (BW = the output channels, at least 32) adds the contributions of row i to
// output rows i + 1, i and i - 1.  Output rows live in a ring of 8
// accumulator blocks of BW columns in tensor memory, output q of the CTA in
// block 7 - (q % 8): the blocks of outputs i + 1, i, i - 1 are then adjacent
// (lowest column first), except where the ring wraps, where the MMA is split
// in two.  The first contribution to an output row is the MMA that starts
// its block (accumulate = 0), issued as its own MMA where its neighbours
// accumulate.  The one thread that issues MMAs is the limit of this kernel:
// a tcgen05.mma of M = 128 took ~110 cycles to issue whatever its N up to
// 192 (operands at a new address each time), so N = 192 does three times
// the work of N = 64 in the same issue slot.  Per 64-channel input row:
// 3 column taps x 4 K steps = 12 MMAs (plus the splits).
//
// Roles (warps), handing work over through mbarriers:
//   warps 0-7   epilogue: output q goes to the four warps of parity q % 2,
//               warp w draining lane quarter w % 4 (32 pixels, all
//               columns) with tcgen05.ld, freeing the block, applying bias +
//               ReLU (or the ReLU mask) and storing; 64-channel BF16 rows go
//               through the warp's own 4 KB staging tile in the 128-byte
//               swizzled layout and one TMA tensor store per warp
//   warps 8-11  loads.  64-channel inputs: warp 8 brings each 130-pixel
//               input row (tile + one halo pixel each side) into its ring
//               slot with one TMA tensor load (128-byte swizzle, zero fill
//               outside the image); warp 9 waits for it, writes the
//               wrapped-around halo pixel of a zonally periodic grid (which
//               the tensor load fills with zero) and releases the slot to
//               the MMA thread.  16-channel inputs: the four warps stream the
//               row with cp.async into 8-channel planes (no swizzle).
//   warp 12     MMA: one thread waits for the row and for the blocks it
//               starts to be drained, issues the MMAs, and commits the
//               release of the slot and "block full" for each output row
//               the row completes.
// Every wait is bounded: a wait that gives up sets the error flag and a
// shared stop flag, and every role leaves its loop; the MMA thread waits
// (bounded) for its MMAs and the load warp for its tensor loads before
// tensor memory is freed and the CTA exits.
constexpr int kRing = 6;           // input row slots
constexpr int kBlocks = 8;         // accumulator blocks (output rows) in tensor memory
constexpr int kRowPix = kM + 2;    // pixels per input row slot
constexpr int kRowB = kRowPix * 16;            // plane layout: one slot of one plane (2,080 bytes)
constexpr int kPlaneW = kRing * kRowB + 16;    // padded plane (12,496 bytes)
constexpr int kSlotSW = 17 * 1024;             // swizzled layout: 130 rows of 128 bytes, 1024-byte aligned
constexpr int kRowsThreads = 13 * 32;          // 8 epilogue + 4 load + 1 MMA warps

template <int CIN>
__host__ __device__ constexpr bool row_tma() { return CIN == 64; }
template <int CIN>
__host__ __device__ constexpr int ring_bytes() { return row_tma<CIN>() ? kRing * kSlotSW : (CIN / 8) * kPlaneW; }
template <int NOUT>
__host__ __device__ constexpr int blk_w() { return NOUT < 32 ? 32 : NOUT; }
template <int NOUT>
__host__ __device__ constexpr bool store_tma() { return NOUT == 64; }

// tcgen05.mma with each descriptor given as its two 32-bit words
__device__ __forceinline__ void umma_bf16_w(uint32_t tmem_d, uint32_t a_lo, uint32_t a_hi, uint32_t b_lo, uint32_t b_hi,
                                            uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t.reg .b64 ad, bd;\n\tsetp.ne.b32 p, %6, 0;\n\tmov.b64 ad, {%1, %2};\n\t"
      "mov.b64 bd, {%3, %4};\n\ttcgen05.mma.cta_group::1.kind::f16 [%0], ad, bd, %5, p;\n\t}\n" ::"r"(tmem_d),
      "r"(a_lo), "r"(a_hi), "r"(b_lo), "r"(b_hi), "r"(idesc), "r"(accumulate));
}
// start-address step (16-byte units) of the A operand of column tap dx, K
// step j within a ring slot: dx pixels in, K columns j * 16 in
template <int CIN>
__host__ __device__ constexpr uint32_t a_step(int dx, int j) {
  return row_tma<CIN>() ? (uint32_t)(dx * 8 + j * 2) : (uint32_t)(dx + j * (2 * kPlaneW / 16));
}

__device__ __forceinline__ void cp_async_arrive_noinc(uint32_t mbar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(mbar) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void tma_load3(uint32_t dst, const CUtensorMap *map, int c0, int c1, int c2, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
          dst),
      "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(mbar)
      : "memory");
}
__device__ __forceinline__ void tma_store3(const CUtensorMap *map, uint32_t src, int c0, int c1, int c2) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(map),
               "r"(src), "r"(c0), "r"(c1), "r"(c2)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// One tile column's run of output rows [rb, re] (global image rows, all
// images stacked) out of a CTA's tiles [t, t1); tiles are numbered tile
// column first.  Its input rows are rb - 1 .. re + 1, those of the same
// images.
struct RowRun {
  int tx, rb, re, ilo, ihi;
};
__device__ __forceinline__ bool next_run(long long &t, long long t1, int NR, int H, RowRun &r) {
  if (t >= t1) return false;
  r.tx = (int)(t / NR);
  r.rb = (int)(t % NR);
  long long end = (long long)(r.tx + 1) * NR;
  if (end > t1) end = t1;
  r.re = r.rb + (int)(end - t) - 1;
  r.ilo = r.rb - (r.rb % H > 0 ? 1 : 0);
  r.ihi = r.re + (r.re % H < H - 1 ? 1 : 0);
  t = end;
  return true;
}

// (in the MODE 1 instantiation the BF16 epilogue after its `continue` is
// unreachable by design)
#pragma nv_diag_suppress 128
// MODE (compile time, so that each epilogue holds only its own registers):
// 0 = + bias, ReLU, BF16 out; 1 = + bias, FP32 out, first nstore channels;
// 2 = ReLU mask from aux, BF16 out
template <int CIN, int NOUT, int MODE>
__global__ void __launch_bounds__(kRowsThreads, 1) k_conv_rows(const __nv_bfloat16 *__restrict__ in,
                                                            const __nv_bfloat16 *__restrict__ w,
                                                            const float *__restrict__ bias,
                                                            const __nv_bfloat16 *__restrict__ aux, void *out, int nimg,
                                                            int H, int W, int periodic_x, int nstore, int *err,
                                                            const __grid_constant__ CUtensorMap tmap_in,
                                                            const __grid_constant__ CUtensorMap tmap_out) {
  constexpr int mode = MODE;
  constexpr int KC = CIN / 8, KJ = CIN / 16;  // 16-byte chunks, K steps of one pixel
  constexpr int BW = blk_w<NOUT>();
  constexpr int WT_BYTES = BW * CIN * 2;      // one target's weights of one column tap
  constexpr int W_BYTES = 9 * WT_BYTES;       // [column tap][target][BW rows][CIN]
  constexpr int STG = 32 * NOUT * 2;          // one epilogue warp's staging tile
  constexpr uint32_t NCOLS = kBlocks * BW;
  constexpr uint32_t ROW_TX = kRowPix * 128;  // bytes of one 64-channel tensor load
  static_assert(!row_tma<CIN>() || (W_BYTES % 1024 == 0 && STG % 1024 == 0), "swizzled slots need 1024-byte alignment");
  static_assert(3 * BW <= 256, "N of one MMA");
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ __align__(16) float s_bias[NOUT];
  __shared__ __align__(8) uint64_t full[kRing], tmab[kRing], empty[kRing], bfull[kBlocks], bempty[kBlocks], done;
  __shared__ uint32_t tmem_slot;
  __shared__ volatile int s_stop;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  // 1024-byte aligned base: swizzled staging tiles and ring slots need it
  const uint32_t base = (smem_u32(smem_raw) + 1023u) & ~1023u;
  uint8_t *const sbase = smem_raw + (base - smem_u32(smem_raw));
  const bool tma_out = store_tma<NOUT>() && mode != 1;
  const uint32_t Stg = base, Wsm = base + (store_tma<NOUT>() ? 8 * STG : 0), Ring = Wsm + W_BYTES;
  const int ntx = (W + kM - 1) / kM;
  const int NR = nimg * H;
  const long long ntiles = (long long)NR * ntx;
  const long long chunk = (ntiles + gridDim.x - 1) / gridDim.x;
  const long long t0 = (long long)blockIdx.x * chunk;
  const long long t1 = t0 + chunk < ntiles ? t0 + chunk : ntiles;

  if (warp == 0) tmem_alloc(smem_u32(&tmem_slot), NCOLS);
  if (tid == 0) {
    for (int q = 0; q < kRing; ++q) {
      mbar_init(smem_u32(&full[q]), row_tma<CIN>() ? 1 : 32 * 4);  // halo writer, or one arrival per load thread
      mbar_init(smem_u32(&tmab[q]), 1);
      mbar_init(smem_u32(&empty[q]), 1);
    }
    for (int q = 0; q < kBlocks; ++q) {
      mbar_init(smem_u32(&bfull[q]), 1);
      mbar_init(smem_u32(&bempty[q]), 4);  // the four epilogue warps of the row
    }
    mbar_init(smem_u32(&done), 1);
    s_stop = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // weights, resident for the kernel's lifetime: for column tap dx the B
  // operand is 3 BW rows, row t BW + n = tap (dy = t - 1, dx) output channel
  // n (zero for n >= NOUT)
  for (int q = tid; q < 9 * BW * KC; q += kRowsThreads) {
    const int dx = q / (3 * BW * KC), r = q % (3 * BW * KC), rr = r / KC, c = r % KC;
    const int tg = rr / BW, n = rr % BW;
    const bool ok = n < NOUT;
    cp_async16(Wsm + (uint32_t)(dx * 3 * WT_BYTES + ((rr / 8) * KC + c) * 128 + (rr % 8) * 16),
               ok ? (const void *)(w + ((long long)(tg * 3 + dx) * NOUT + n) * CIN + c * 8) : (const void *)w, ok);
  }
  for (int q = tid; q < NOUT; q += kRowsThreads) s_bias[q] = mode == 2 ? 0.f : bias[q];
  cp_async_wait_all();
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  auto stop = [&]() {
    s_stop = 1;
    atomicExch(err, 1);
  };
  RowRun run;

  if (warp == 8 && row_tma<CIN>()) {
    // ----------------------------------------------------- tensor loads
    if (lane == 0) {
      int k = 0;
      long long t = t0;
      bool ok = true;
      while (ok && !s_stop && next_run(t, t1, NR, H, run)) {
        for (int i = run.ilo; i <= run.ihi && !s_stop; ++i, ++k) {
          const int s = k % kRing, n = k / kRing;
          if (n > 0 && !mbar_wait(smem_u32(&empty[s]), (uint32_t)((n - 1) & 1))) {
            stop();
            ok = false;
            break;
          }
          mbar_expect_tx(smem_u32(&tmab[s]), ROW_TX);
          tma_load3(Ring + (uint32_t)(s * kSlotSW), &tmap_in, 0, run.tx * kM - 1, i, smem_u32(&tmab[s]));
        }
      }
      // no tensor load may still be writing when the CTA exits: the last one
      // of each slot has landed (the consumer may have stopped early)
      for (int s = 0; s < kRing && s < k; ++s) {
        const int n = (k - 1 - s) / kRing;  // uses of slot s: the last is k' = s + n kRing
        mbar_wait(smem_u32(&tmab[s]), (uint32_t)(n & 1));
      }
    }
  } else if (warp == 9 && row_tma<CIN>()) {
    // ---------------------------------------- periodic halo, slot release
    int k = 0;
    long long t = t0;
    bool go = true;
    while (go && !s_stop && next_run(t, t1, NR, H, run)) {
      const int x0 = run.tx * kM;
      const bool wl = periodic_x && run.tx == 0, wr = periodic_x && x0 + kM >= W;
      for (int i = run.ilo; i <= run.ihi && !s_stop; ++i, ++k) {
        const int s = k % kRing, n = k / kRing;
        const int ok = __shfl_sync(0xffffffffu, lane == 0 ? (int)mbar_wait(smem_u32(&tmab[s]), (uint32_t)(n & 1)) : 0, 0);
        if (!ok) {
          if (lane == 0) stop();
          go = false;
          break;
        }
        // the pixel left of x = 0 is x = W - 1; right of x = W - 1 is x = 0
        const int c = lane & 7;
        const bool left = lane < 8 && wl, right = lane >= 8 && lane < 16 && wr;
        if (left || right) {
          const int u = left ? 0 : W - x0 + 1, xs = left ? W - 1 : 0;
          const uint4 v = __ldg(reinterpret_cast<const uint4 *>(in + ((long long)i * W + xs) * CIN) + c);
          *reinterpret_cast<uint4 *>(sbase + (Ring - base) + s * kSlotSW + u * 128 + ((c ^ (u & 7)) << 4)) = v;
          fence_async_smem();
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_u32(&full[s]));
      }
    }
  } else if (warp >= 8 && warp < 12 && !row_tma<CIN>()) {
    // ------------------------------------------------- cp.async row loads
    const int lt = tid - 8 * 32;
    int k = 0;
    long long t = t0;
    bool go = true;
    while (go && !s_stop && next_run(t, t1, NR, H, run)) {
      const int x0 = run.tx * kM;
      for (int i = run.ilo; i <= run.ihi && !s_stop; ++i, ++k) {
        const int s = k % kRing, n = k / kRing;
        if (n > 0 && !mbar_wait(smem_u32(&empty[s]), (uint32_t)((n - 1) & 1))) {
          stop();
          go = false;
          break;
        }
        for (int q = lt; q < kRowPix * KC; q += 32 * 4) {
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
          cp_async16(Ring + (uint32_t)(c * kPlaneW + s * kRowB + u * 16),
                     ok ? (const void *)(in + ((long long)i * W + xx) * CIN + c * 8) : (const void *)in, ok);
        }
        cp_async_arrive_noinc(smem_u32(&full[s]));
      }
    }
    cp_async_wait_all();
  } else if (warp == 12) {
    // ------------------------------------------------------------------ MMA
    if (lane == 0) {
      // descriptors as a 32-bit low word (start address, leading byte
      // offset) over a fixed high word: the offsets added below stay inside
      // the 14-bit start field (shared-memory addresses < 256 KB)
      const uint64_t adesc0 = row_tma<CIN>() ? umma_desc_sw128(Ring) : umma_desc(Ring, kPlaneW, 128);
      const uint64_t bdesc0 = umma_desc(Wsm, 128, KC * 128);
      const uint32_t a_hi = (uint32_t)(adesc0 >> 32), b_hi = (uint32_t)(bdesc0 >> 32);
      const uint32_t a_lo0 = (uint32_t)adesc0, b_lo0 = (uint32_t)bdesc0;
      constexpr uint32_t SLOT16 = (row_tma<CIN>() ? kSlotSW : kRowB) / 16;  // one ring slot, 16-byte units
      constexpr uint32_t WT16 = WT_BYTES / 16;
      int qbase = 0, s = 0;  // s: ring slot of the current row
      uint32_t ph = 0;       // parity of slot s's current fill
      // the next row's slot and first block, tested right after this row's
      // MMAs are issued, while they run (a test took ~400 cycles while the
      // MMAs read shared memory; two in a row at the top of each row left
      // the tensor pipe idle)
      uint32_t pre_ok = 0;
      bool pre = false;
      bool issued = false, go = true;
      long long t = t0;
      while (go && !s_stop && next_run(t, t1, NR, H, run)) {
        int y = run.ilo % H;  // image row of input row i
        for (int i = run.ilo; i <= run.ihi; ++i) {
          // targets: 0 = output i + 1 (tap dy = -1), 1 = output i, 2 = output i - 1
          const bool v0 = i + 1 <= run.re && y < H - 1, v1 = i >= run.rb && i <= run.re, v2 = i - 1 >= run.rb && y > 0;
          const int ta = v0 ? 0 : (v1 ? 1 : 2), tb = v2 ? 2 : (v1 ? 1 : 0);
          const int q0 = qbase + (i + 1 - run.rb);  // output number of target 0 (q of target t: q0 - t)
          const bool nw1 = y == 0;                  // output i starts here (no row above in its image)
          bool ok = true;
          // blocks this row starts: drained of their previous output
          if (v0 && q0 >= kBlocks && !(pre && (pre_ok & 2u)))
            ok = mbar_spin(smem_u32(&bempty[7 - (q0 & 7)]), (uint32_t)(((q0 >> 3) - 1) & 1));
          if (ok && v1 && nw1 && q0 - 1 >= kBlocks)
            ok = mbar_spin(smem_u32(&bempty[7 - ((q0 - 1) & 7)]), (uint32_t)((((q0 - 1) >> 3) - 1) & 1));
          if (ok && !(pre && (pre_ok & 1u))) ok = mbar_spin(smem_u32(&full[s]), ph);
          // another role's stop is seen within 8 rows (a shared-memory read
          // waits behind the MMAs' operand reads; this thread's own waits
          // are bounded either way)
          if (!ok || ((i & 7) == 0 && s_stop)) {
            if (!ok) stop();
            go = false;
            break;
          }
          // The row's MMAs.  A run of adjacent targets shares one MMA; target
          // t starts a new run where target t - 1 is invalid or its block is
          // not adjacent (the ring wraps between them) and, on the first
          // step, where a block that starts here meets one that accumulates.
          // The issuing thread is this kernel's limit: with the runs worked
          // out in the loop, runtime branches and 64-bit descriptor
          // arithmetic per MMA, it issued one MMA per ~235 cycles with every
          // other role switched off; the straight-line sequences below add
          // compile-time offsets to 32-bit words.
          // the other steps: one run from ta, or two where the ring wraps
          // between targets 0 and 1 or 1 and 2
          const int r2 = (ta == 0 && tb >= 1 && (q0 & 7) == 0) ? 1 : ((ta <= 1 && tb == 2 && ((q0 - 1) & 7) == 0) ? 2 : -1);
          const uint32_t a_lo = a_lo0 + (uint32_t)s * SLOT16;
          // cp.async rows (generic proxy) need a proxy fence before the
          // MMAs read them; tensor-loaded rows are async-proxy writes and
          // their halo writer fences before it releases the slot
          if (!row_tma<CIN>()) fence_async_smem();
          tc_fence_after();
          if (ta == 0 && tb == 2 && r2 < 0 && !nw1) {
            // the common row: outputs i + 1, i, i - 1 in adjacent blocks, only
            // output i + 1 starting: step 0 = [i + 1] (starts its block) and
            // [i, i - 1]; the other steps one MMA over all three
            const uint32_t c0 = tmem + (uint32_t)((7 - (q0 & 7)) * BW);
            umma_bf16_w(c0, a_lo, a_hi, b_lo0, b_hi, umma_idesc(kM, BW, 0, 0), 0u);
            umma_bf16_w(c0 + BW, a_lo, a_hi, b_lo0 + WT16, b_hi, umma_idesc(kM, 2 * BW, 0, 0), 1u);
            #pragma unroll
            for (int st = 1; st < 3 * KJ; ++st)
              umma_bf16_w(c0, a_lo + a_step<CIN>(st / KJ, st % KJ), a_hi,
                          b_lo0 + (uint32_t)((st / KJ) * 3 * WT16 + (st % KJ) * 16), b_hi, umma_idesc(kM, 3 * BW, 0, 0),
                          1u);
          } else {
            const bool nw[3] = {true, nw1, false};
            const bool v[3] = {v0, v1, v2};
            // step 0 (column tap 0, K step 0)
            #pragma unroll
            for (int tt = 0; tt < 3; ++tt) {
              const bool adj = tt > 0 && v[tt - 1] && ((q0 - tt + 1) & 7) != 0;  // joins target tt - 1
              if (v[tt] && !(adj && nw[tt] == nw[tt - (tt > 0)])) {
                int e = tt;  // last target of the first-step run starting at tt
                #pragma unroll
                for (int u = tt + 1; u < 3; ++u)
                  if (e == u - 1 && v[u] && ((q0 - u + 1) & 7) != 0 && nw[u] == nw[tt]) e = u;
                umma_bf16_w(tmem + (uint32_t)((7 - ((q0 - tt) & 7)) * BW), a_lo, a_hi, b_lo0 + (uint32_t)tt * WT16, b_hi,
                            umma_idesc(kM, (e - tt + 1) * BW, 0, 0), nw[tt] ? 0u : 1u);
              }
            }
            // steps 1 .. 3 KJ - 1: column tap dx = st / KJ, K step j = st % KJ
            const uint32_t colA = tmem + (uint32_t)((7 - ((q0 - ta) & 7)) * BW);
            const uint32_t idA = umma_idesc(kM, ((r2 < 0 ? tb : r2 - 1) - ta + 1) * BW, 0, 0);
            const uint32_t bA = b_lo0 + (uint32_t)ta * WT16;
            if (r2 < 0) {
              #pragma unroll
              for (int st = 1; st < 3 * KJ; ++st)
                umma_bf16_w(colA, a_lo + a_step<CIN>(st / KJ, st % KJ), a_hi,
                            bA + (uint32_t)((st / KJ) * 3 * WT16 + (st % KJ) * 16), b_hi, idA, 1u);
            } else {
              const uint32_t colB = tmem + (uint32_t)((7 - ((q0 - r2) & 7)) * BW);
              const uint32_t idB = umma_idesc(kM, (tb - r2 + 1) * BW, 0, 0);
              const uint32_t bB = b_lo0 + (uint32_t)r2 * WT16;
              #pragma unroll
              for (int st = 1; st < 3 * KJ; ++st) {
                const uint32_t ad = a_lo + a_step<CIN>(st / KJ, st % KJ);
                const uint32_t boff = (uint32_t)((st / KJ) * 3 * WT16 + (st % KJ) * 16);
                umma_bf16_w(colA, ad, a_hi, bA + boff, b_hi, idA, 1u);
                umma_bf16_w(colB, ad, a_hi, bB + boff, b_hi, idB, 1u);
              }
            }
          }
          // row i + 1 of the same run: its slot, and the block of its output
          // i + 2 (output q0 + 1), whose drain it needs (the block's first
          // use needs none: a test of the phase before its first reads 1)
          pre = i + 1 <= run.ihi;
          if (pre)
            pre_ok = mbar_test2(smem_u32(&full[s + 1 == kRing ? 0 : s + 1]), s + 1 == kRing ? ph ^ 1u : ph,
                                smem_u32(&bempty[7 - ((q0 + 1) & 7)]), (uint32_t)((((q0 + 1) >> 3) - 1) & 1));
          issued = true;
          umma_commit(smem_u32(&empty[s]));
          if (v2) umma_commit(smem_u32(&bfull[7 - ((q0 - 2) & 7)]));
          if (v1 && y == H - 1) umma_commit(smem_u32(&bfull[7 - ((q0 - 1) & 7)]));
          if (++y == H) y = 0;
          if (++s == kRing) {
            s = 0;
            ph ^= 1u;
          }
        }
        qbase += run.re - run.rb + 1;
      }
      // every MMA issued has completed before tensor memory is freed
      if (issued) {
        umma_commit(smem_u32(&done));
        if (!mbar_wait(smem_u32(&done), 0)) atomicExch(err, 1);
      }
    }
  } else if (warp < 8) {
    // ------------------------------------------------------------- epilogue
    const int quarter = warp & 3, par = warp >> 2;
    const int m = quarter * 32 + lane;
    // mode 0: the bias in registers (read from shared memory per row it
    // took ~1,500 of the ~2,700 cycles of a 64-channel row's conversion
    // while the MMAs stream their operands)
    float breg[mode == 0 ? NOUT : 1];
    #pragma unroll
    for (int c = 0; c < (mode == 0 ? NOUT : 1); ++c) breg[c] = mode == 0 ? s_bias[c] : 0.f;
    const uint32_t stg = Stg + (uint32_t)(warp * STG);
    uint8_t *const stg_p = sbase + warp * STG;
    int q = 0;
    bool go = true;
    long long t = t0;
    while (go && !s_stop && next_run(t, t1, NR, H, run)) {
      const int x0 = run.tx * kM, x = x0 + m;
      for (int o = run.rb; o <= run.re; ++o, ++q) {
        if ((q & 1) != par) continue;
        const int b = 7 - (q & 7);
        const long long p = (long long)o * W + x;
        uint4 am[NOUT / 8];  // the ReLU mask of this pixel, fetched before the wait
        if (mode == 2) {
          #pragma unroll
          for (int c = 0; c < NOUT / 8; ++c)
            am[c] = x < W ? __ldg(reinterpret_cast<const uint4 *>(aux + p * NOUT) + c) : make_uint4(0, 0, 0, 0);
        }
        const bool ok = mbar_wait(smem_u32(&bfull[b]), (uint32_t)((q >> 3) & 1));
        if (!ok) stop();
        if (__any_sync(0xffffffffu, !ok)) {
          go = false;
          break;
        }
        tc_fence_after();
        uint32_t r[NOUT];
        const uint32_t lane_addr = tmem + (uint32_t)(b * BW) + ((uint32_t)(quarter * 32) << 16);
        #pragma unroll
        for (int c0 = 0; c0 < NOUT; c0 += 16) tmem_ld16_nowait(lane_addr + c0, r + c0);
        tmem_ld_wait();
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_u32(&bempty[b]));
        if (mode == 1) {
          if (x < W) {
            float *o4 = (float *)out + p * nstore;
            if (nstore == 4) {
              *reinterpret_cast<float4 *>(o4) =
                  make_float4(__uint_as_float(r[0]) + s_bias[0], __uint_as_float(r[1]) + s_bias[1],
                              __uint_as_float(r[2]) + s_bias[2], __uint_as_float(r[3]) + s_bias[3]);
            } else {
              #pragma unroll
              for (int c = 0; c < NOUT; ++c)
                if (c < nstore) o4[c] = __uint_as_float(r[c]) + s_bias[c];
            }
          }
          continue;
        }
        uint32_t pk[NOUT / 2];
        #pragma unroll
        for (int c = 0; c < NOUT / 2; ++c) {
          const float a0 = __uint_as_float(r[2 * c]), a1 = __uint_as_float(r[2 * c + 1]);
          float lo, hi;
          if (mode == 0) {
            lo = fmaxf(a0 + breg[(2 * c) % (mode == 0 ? NOUT : 1)], 0.f);
            hi = fmaxf(a1 + breg[(2 * c + 1) % (mode == 0 ? NOUT : 1)], 0.f);
          } else {
            const uint32_t aw = (&am[c / 4].x)[c % 4];
            const __nv_bfloat162 a2 = *reinterpret_cast<const __nv_bfloat162 *>(&aw);
            lo = __low2float(a2) > 0.f ? a0 : 0.f;
            hi = __high2float(a2) > 0.f ? a1 : 0.f;
          }
          const __nv_bfloat162 b2 = __floats2bfloat162_rn(lo, hi);
          pk[c] = *reinterpret_cast<const uint32_t *>(&b2);
        }
        if (!tma_out) {
          if (x < W) {
            uint4 *o16 = reinterpret_cast<uint4 *>((__nv_bfloat16 *)out + p * NOUT);
            #pragma unroll
            for (int c = 0; c < NOUT / 8; ++c) o16[c] = make_uint4(pk[4 * c], pk[4 * c + 1], pk[4 * c + 2], pk[4 * c + 3]);
          }
          continue;
        }
        // this warp's previous store has read its staging tile
        if (lane == 0) bulk_wait_read0();
        __syncwarp();
        uint8_t *row = stg_p + lane * 128;
        #pragma unroll
        for (int c = 0; c < NOUT / 8; ++c)  // 16-byte chunk c of the pixel's 128 bytes, 128-byte swizzle
          *reinterpret_cast<uint4 *>(row + ((c ^ (lane & 7)) << 4)) =
              make_uint4(pk[4 * c], pk[4 * c + 1], pk[4 * c + 2], pk[4 * c + 3]);
        fence_async_smem();  // the staging writes, ordered before the TMA store reads them
        __syncwarp();
        if (lane == 0 && x0 + quarter * 32 < W) {
          tma_store3(&tmap_out, stg, 0, x0 + quarter * 32, o);
          bulk_commit();
        }
      }
    }
    if (lane == 0) bulk_wait_all();
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, NCOLS);
}
#pragma nv_diag_default 128

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
size_t rows_smem() {
  return 1024 + (store_tma<NOUT>() ? 8 * (size_t)32 * NOUT * 2 : 0) + (size_t)9 * blk_w<NOUT>() * CIN * 2 +
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

// [image rows][W][C] BF16 activations as a 3-D tensor map with a box of
// box_w pixels x C channels, 128-byte swizzle
bool act_tensor_map(CUtensorMap *tm, const void *p, int C, int W, int NR, int box_w) {
  auto enc = tensor_map_encoder();
  if (!enc || ((uintptr_t)p & 15u)) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)NR};
  const cuuint64_t strides[2] = {(cuuint64_t)C * 2, (cuuint64_t)W * C * 2};
  const cuuint32_t box[3] = {(cuuint32_t)C, (cuuint32_t)box_w, 1u};
  const cuuint32_t estr[3] = {1u, 1u, 1u};
  return enc(tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void *>(p), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int CIN, int NOUT, int MODE>
cudaError_t conv_rows_launch_m(const __nv_bfloat16 *in, const __nv_bfloat16 *w, const float *bias,
                               const __nv_bfloat16 *aux, void *out, long long npix, int H, int W, int periodic_x,
                               int nstore, int *err, cudaStream_t s) {
  constexpr int mode = MODE;
  const size_t sm = rows_smem<CIN, NOUT>();
  cudaError_t e =
      cudaFuncSetAttribute(k_conv_rows<CIN, NOUT, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  const long long hw = (long long)H * W;
  const long long NRl = npix / hw;
  if (NRl * H > 0x7fffffffLL) return cudaErrorInvalidValue;
  const int nimg = (int)NRl, NR = nimg * H;
  const long long ntiles = (long long)NR * ((W + kM - 1) / kM);
  // input rows: one box = the 130 pixels of a tile and its halo; output:
  // one box = an epilogue warp's 32 pixels; pixels past W are zero-filled
  // (loads) or not written (stores)
  CUtensorMap tin, tout;
  memset(&tin, 0, sizeof tin);
  memset(&tout, 0, sizeof tout);
  if (row_tma<CIN>() && !act_tensor_map(&tin, in, CIN, W, NR, kRowPix)) return cudaErrorInvalidValue;
  if (store_tma<NOUT>() && mode != 1 && !act_tensor_map(&tout, out, NOUT, W, NR, 32)) return cudaErrorInvalidValue;
  int dev = 0, nsm = 148, per = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_conv_rows<CIN, NOUT, MODE>, kRowsThreads, sm);
  const int tmem_cap = 512 / (kBlocks * blk_w<NOUT>());
  per = per < 1 ? 1 : (per > tmem_cap ? tmem_cap : per);
  const long long grid = ntiles < (long long)nsm * per ? ntiles : (long long)nsm * per;
  if (grid < 1) return cudaSuccess;
  k_conv_rows<CIN, NOUT, MODE><<<(unsigned)grid, kRowsThreads, sm, s>>>(in, w, bias, aux, out, nimg, H, W,
                                                                         periodic_x, nstore, err, tin, tout);
  return cudaGetLastError();
}

template <int CIN, int NOUT>
cudaError_t conv_rows_launch(const __nv_bfloat16 *in, const __nv_bfloat16 *w, const float *bias,
                             const __nv_bfloat16 *aux, void *out, long long npix, int H, int W, int periodic_x,
                             int mode, int nstore, int *err, cudaStream_t s) {
  if (mode == 0) return conv_rows_launch_m<CIN, NOUT, 0>(in, w, bias, aux, out, npix, H, W, periodic_x, nstore, err, s);
  if (mode == 1) return conv_rows_launch_m<CIN, NOUT, 1>(in, w, bias, aux, out, npix, H, W, periodic_x, nstore, err, s);
  if (mode == 2) return conv_rows_launch_m<CIN, NOUT, 2>(in, w, bias, aux, out, npix, H, W, periodic_x, nstore, err, s);
  return cudaErrorInvalidValue;
}

template <int CIN, int NOUT>
cudaError_t conv_launch(const __nv_bfloat16 *in, const __nv_bfloat16 *w, const float *bias, const __nv_bfloat16 *aux,
                        void *out, long long npix, int H, int W, int periodic_x, int mode, int nstore, int *err,
                        cudaStream_t s) {
  // whole images: the persistent row-streaming form
  if (npix % ((long long)H * W) == 0)
    return conv_rows_launch<CIN, NOUT>(in, w, bias, aux, out, npix, H, W, periodic_x, mode, nstore, err, s);
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
