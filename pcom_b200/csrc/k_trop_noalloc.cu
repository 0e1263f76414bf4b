// k_trop_noalloc.cu -- pcom_gpu_trop_noalloc: the barotropic subcycle for
// callers that cannot allocate device memory.
//
// Who needs it: host frameworks that own every byte of device memory and
// hand it out from their own pool -- a coupled-model driver that sizes its
// pool for all components at start-up, or a serving stack whose caching
// allocator already holds the GPU -- so a cudaMalloc from inside this library
// would fail or break the framework's memory budget.  Such callers can own the
// inputs and outputs, but not the scratch the subcycle needs.  This entry
// point keeps that scratch in one fixed array compiled into the library
// (g_trop_scratch below, about 3.2 MB, held by every GPU that loads the
// library until the process exits) and never allocates.
//
// Limits: ni*nj <= PCOM_NOALLOC_MAX_POINTS and ni, nj <= PCOM_NOALLOC_MAX_DIM
// (PCOM_NOALLOC_MAX_POINTS covers the 1-degree 362 x 162 domain); larger
// domains are rejected.  Every call uses the same array, so two calls that
// overlap on the GPU (different streams, or different host threads) race.
// The first call on a device (in each CUDA context of that device) looks up
// the array's device address with cudaGetSymbolAddress; make that first call
// before any stream capture.  Each call waits on the caller's stream twice
// (for the metric check and for the kernel's status words), so it returns
// after the subcycle has finished on the GPU.
#include <mutex>

#include "../../include/pcom_gpu.h"
#include "pcom_dev.cuh"
#include "pcom_kernels.h"

namespace {

constexpr long long kMaxPts = PCOM_NOALLOC_MAX_POINTS;
constexpr int kMaxDim = PCOM_NOALLOC_MAX_DIM;
// layout (in doubles): 6 ping-pong planes (ch, ub, vb x 2), 8 metric vectors
// (dxy and rh of grids 1..4), then 8 words of barrier/flag state
constexpr long long kOffMetric = 6 * kMaxPts;
constexpr long long kOffWords = kOffMetric + 8LL * kMaxDim;
constexpr long long kScratch = kOffWords + 8;

static __device__ __align__(256) double g_trop_scratch[kScratch];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
// device address of g_trop_scratch per device, with the context it was looked
// up in: a cudaDeviceReset destroys that context, the module is loaded again
// in the next one and the array may move, so a new context means a new lookup
double *g_addr[kMaxDevices] = {};
void *g_ctx[kMaxDevices] = {};

// the calling thread's current driver context (cuCtxGetCurrent through the
// runtime's driver entry-point table; the library links no libcuda)
typedef int (*ctx_get_fn)(void **);
void *current_context() {
  static ctx_get_fn fn = [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return (ctx_get_fn)f;
  }();
  void *ctx = nullptr;
  if (!fn || fn(&ctx) != 0) return nullptr;
  return ctx;
}

// 1-D copies of the j-only metrics and a check that dx%x(1) depends on i
// only and dx%x(2), rh on j only (lat-lon grids, main.f90:408-493)
__global__ void k_noalloc_metrics(pcom_trop_io io, int ni, int nj, double *vec, unsigned *bad) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  for (int j = t; j < nj; j += gridDim.x * blockDim.x) {
    for (int g = 0; g < 4; ++g) {
      const double y = io.dxy[g][(long long)ni * j], r = io.rh[g][(long long)ni * j];
      vec[g * kMaxDim + j] = y;
      vec[(4 + g) * kMaxDim + j] = r;
      for (int i = 0; i < ni; ++i) {
        const long long q = i + (long long)ni * j;
        if (io.dxy[g][q] != y || io.rh[g][q] != r || io.dxx[g][q] != io.dxx[g][i]) atomicOr(bad, 1u);
      }
    }
  }
}

int error(int code, const char *msg) { return pcom_set_error(code, msg); }

}  // namespace

extern "C" int pcom_gpu_trop_noalloc(const pcom_trop_io *io, void *stream_) {
  if (!io) return error(PCOM_ERR_ARG, "pcom_gpu_trop_noalloc: null argument");
  const int ni = io->glo_ni + 2, nj = io->glo_nj + 2;
  if (io->glo_ni < 2 || io->glo_nj < 2) return error(PCOM_ERR_ARG, "pcom_gpu_trop_noalloc: domain too small");
  if (ni > kMaxDim || nj > kMaxDim || (long long)ni * nj > kMaxPts)
    return error(PCOM_ERR_ARG,
                 "pcom_gpu_trop_noalloc: domain exceeds the fixed scratch (ni*nj <= PCOM_NOALLOC_MAX_POINTS, "
                 "ni, nj <= PCOM_NOALLOC_MAX_DIM)");
  if (io->dtbt <= 0 || io->dtbc <= 0 || io->dtbc % io->dtbt != 0)
    return error(PCOM_ERR_ARG, "pcom_gpu_trop_noalloc: dtbc must be a positive multiple of dtbt");
  cudaStream_t s = (cudaStream_t)stream_;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return error(PCOM_ERR_CUDA, "pcom_gpu_trop_noalloc: no usable current device");
  double *base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    void *ctx = current_context();  // null before the runtime's first use of the device
    if (!ctx || !g_addr[dev] || g_ctx[dev] != ctx) {
      // the host-side symbol is not a device address: look the address up
      // once per device (and context), with that device current
      double *ptr = nullptr;
      cudaError_t e = cudaGetSymbolAddress((void **)&ptr, g_trop_scratch);
      if (e != cudaSuccess || !ptr) return error(PCOM_ERR_CUDA, "pcom_gpu_trop_noalloc: cudaGetSymbolAddress failed");
      ctx = current_context();  // the lookup has initialised the context
      if (!ctx) return error(PCOM_ERR_CUDA, "pcom_gpu_trop_noalloc: cannot read the current CUDA context");
      g_addr[dev] = ptr;
      g_ctx[dev] = ctx;
    }
    base = g_addr[dev];
  }
  double *vec = base + kOffMetric;
  unsigned *words = (unsigned *)(base + kOffWords);  // [0..1] barrier, [2..3] error flags, [4] metric check
  // the barrier count/generation, the error flags and the metric check start at zero
  if (cudaMemsetAsync(words, 0, 8 * sizeof(double), s) != cudaSuccess)
    return error(PCOM_ERR_CUDA, "pcom_gpu_trop_noalloc: clearing the barrier words failed");
  k_noalloc_metrics<<<(nj + 127) / 128, 128, 0, s>>>(*io, ni, nj, vec, words + 4);
  unsigned bad = 0;
  if (cudaMemcpyAsync(&bad, words + 4, sizeof bad, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return error(PCOM_ERR_CUDA, "pcom_gpu_trop_noalloc: metric check failed to run");
  if (bad) return error(PCOM_ERR_ARG, "pcom_gpu_trop_noalloc: metrics are not those of a lat-lon grid");

  Dev D{};
  D.ni = ni; D.nj = nj; D.nim = ni - 1; D.njm = nj - 1; D.glo_ni = io->glo_ni; D.glo_nj = io->glo_nj;
  D.j_lo = 1; D.j_hi = nj;
  D.bt = io->dtbt; D.bc = io->dtbc; D.nstep = io->dtbc / io->dtbt * 2;
  D.n2 = (long long)ni * nj;
  pcom_dev_consts((io->flags & PCOM_LIT_R8) != 0, D.c);
  for (int g = 1; g <= 4; ++g) {
    D.dxx[g] = io->dxx[g - 1];
    D.dxy[g] = io->dxy[g - 1];
    D.rh[g] = io->rh[g - 1];
    D.dxy1d[g] = vec + (g - 1) * kMaxDim;
    D.rh1d[g] = vec + (4 + g - 1) * kMaxDim;
  }
  D.separable = 1;
  D.lev_t = io->lev_t; D.lev_u = io->lev_u;
  D.prh_t = io->prh_t; D.prh_u = io->prh_u;
  D.cor = io->cor; D.am = (double *)io->am1; D.graphihx = io->graphihx; D.graphihy = io->graphihy;
  D.ut = (double *)io->ut; D.vt = (double *)io->vt;
  for (int q = 0; q < 4; ++q) { D.bphi[q] = (double *)io->bphi[q]; D.bgra[q] = (double *)io->bgraphi[q]; }
  D.chc = io->chc; D.chp = io->chp; D.mch = io->mch; D.mch2 = io->mch2;
  D.ubc = io->ubc; D.vbc = io->vbc; D.ubp = io->ubp; D.vbp = io->vbp; D.acch = io->acch;
  for (int q = 0; q < 2; ++q) {
    D.tr_ch[q] = base + (0 + q) * kMaxPts;
    D.tr_ub[q] = base + (2 + q) * kMaxPts;
    D.tr_vb[q] = base + (4 + q) * kMaxPts;
  }
  D.bar = words;
  D.err = (int *)(words + 2);

  // tiling: the resident kernel with the fewest tiles that are co-resident
  int bx = 0, by = 0, best = 1 << 30;
  const int mb = trop_res_max_blocks(24, 18);
  for (int ty = 6; ty <= 40; ++ty)
    for (int tx = 6; tx <= 60; ++tx) {
      if (!trop_res_fits(tx, ty)) continue;
      const int nt = ((io->glo_ni + tx - 1) / tx) * ((nj + ty - 1) / ty);
      if (nt > mb) continue;
      if (nt < best || (nt == best && (tx + 4) * (ty + 4) < (bx + 4) * (by + 4))) { best = nt; bx = tx; by = ty; }
    }
  if (bx == 0 || trop_res_max_blocks(bx, by) < best)
    return error(PCOM_ERR_ARG, "pcom_gpu_trop_noalloc: the domain does not fit one co-resident tile per CTA");
  if (launch_trop_res(D, bx, by, s) != cudaSuccess)
    return error(PCOM_ERR_CUDA, "pcom_gpu_trop_noalloc: kernel launch failed");
  int flags[2] = {0, 0};
  if (cudaMemcpyAsync(flags, D.err, sizeof flags, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return error(PCOM_ERR_CUDA, "pcom_gpu_trop_noalloc: kernel failed");
  if (flags[0]) return error(PCOM_ERR_TIMEOUT, "pcom_gpu_trop_noalloc: a grid barrier gave up waiting");
  return PCOM_OK;
}
