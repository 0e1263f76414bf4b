// cnn.cu -- the closure network on the device: parameters (FP32 master
// copies, BF16 operand copies in the forward and transposed-flipped layouts),
// forward pass, masked mean-square loss, backward pass (tensor-core data and
// weight gradients from k_cnn.cu, bias gradients) and Adam, behind the C ABI
// of include/pcom_cnn.h.
//
// Layers (3x3, 'same'): 16 -> 64 -> 64 -> 64 -> 64 -> 16, ReLU between; the
// first layer's inputs 5..15 and the last layer's outputs 4..15 are zero
// padding of the 5 input and 4 output channels (the UMMA K and N granules).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pcom_cnn.h"
#include "cnn_kernels.h"

namespace {

thread_local std::string g_cnn_error;
int cfail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_cnn_error = buf;
  return code;
}
#define CC(call)                                                                                 \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess) return cfail(PCOM_CNN_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

constexpr int kLayers = 5;
constexpr int kK[kLayers] = {16, 64, 64, 64, 64};  // input channels (padded)
constexpr int kN[kLayers] = {64, 64, 64, 64, 16};  // output channels (padded)
constexpr int kRealIn = 5, kRealOut = 4;           // real input / output channels

long long wsize(int l) { return 9LL * kN[l] * kK[l]; }

// ---------------------------------------------------------------- kernels
__global__ void k_to_bf16(const float *w, __nv_bfloat16 *o, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    o[i] = __float2bfloat16(w[i]);
}
// dgrad layout: wd[t][k][n] = w[8 - t][n][k]
__global__ void k_flip_t(const float *w, __nv_bfloat16 *wd, int N, int K) {
  const long long n9 = 9LL * N * K;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n9; i += (long long)gridDim.x * blockDim.x) {
    const int t = (int)(i / ((long long)N * K));
    const int r = (int)(i % ((long long)N * K));
    const int k = r / N, n = r % N;  // wd index (t, k, n)
    wd[i] = __float2bfloat16(w[((long long)(8 - t) * N + n) * K + k]);
  }
}
// bias gradient: db[n] += sum_p g[p][n]
__global__ void k_colsum(const __nv_bfloat16 *g, int N, long long npix, float *db) {
  const long long gid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long nthr = (long long)gridDim.x * blockDim.x;
  const int n = (int)(gid % N);
  float s = 0.f;
  for (long long p = gid / N; p < npix; p += nthr / N) s += __bfloat162float(g[p * N + n]);
  atomicAdd(db + n, s);
}
__global__ void k_mask_count(const float *mask, long long n, double *cnt) {
  double s = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    s += mask[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(cnt, s);
}
// loss = sum mask (y - t)^2 / count; g = d loss / d y (BF16, 16 channels)
__global__ void k_loss(const float *y, const float *t, const float *mask, long long npix, const double *cnt,
                       double *loss, __nv_bfloat16 *g) {
  const double c = *cnt;
  const float sc = c > 0 ? (float)(2.0 / c) : 0.f;
  double s = 0.0;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npix; p += (long long)gridDim.x * blockDim.x) {
    #pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float m = mask[p * 4 + q];
      const float d = (y[p * 4 + q] - t[p * 4 + q]) * m;
      s += (double)d * d;
      g[p * 16 + q] = __float2bfloat16(sc * d);
    }
    #pragma unroll
    for (int q = 4; q < 16; ++q) g[p * 16 + q] = __float2bfloat16(0.f);
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0 && c > 0) atomicAdd(loss, s / c);
}
// Adam (Kingma & Ba 2015) on the FP32 master parameters
__global__ void k_adam(float *w, const float *g, float *m, float *v, long long n, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}
// zero the padded channels of the first and last layers (kept exactly 0)
__global__ void k_zero_pad(float *w1, float *w5, float *b5) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 9 * 64 * 16) {
    const int k = i % 16;
    if (k >= kRealIn) w1[i] = 0.f;
  }
  if (i < 9 * 16 * 64) {
    const int n = (i / 64) % 16;
    if (n >= kRealOut) w5[i] = 0.f;
  }
  if (i < 16 && i >= kRealOut) b5[i] = 0.f;
}

}  // namespace

struct pcom_cnn {
  int H = 0, W = 0, max_img = 0, periodic_x = 1;
  cudaStream_t stream = nullptr;
  bool own_stream = true;  // created here (destroyed here), or the caller's
  long long nparam = 0;
  float *param = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;  // FP32, [W1 b1 ... W5 b5]
  __nv_bfloat16 *wf[kLayers] = {}, *wd[kLayers] = {};                   // operand copies
  __nv_bfloat16 *act[kLayers] = {};                                     // act[0] = input copy, act[l] = layer l output
  __nv_bfloat16 *gbuf[2] = {};                                          // gradient ping-pong (64 ch)
  __nv_bfloat16 *gout = nullptr;                                        // d loss / d y (16 ch)
  float *y = nullptr;
  double *scal = nullptr;  // [0] mask count, [1] loss
  int *err = nullptr;
  long long step = 0;
  std::vector<void *> allocs;
  long long woff[kLayers], boff[kLayers];
  ~pcom_cnn() {
    for (void *p : allocs) cudaFree(p);
  }
  template <class T>
  int alloc(T **p, size_t n) {
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, n * sizeof(T));
    if (e != cudaSuccess) return cfail(PCOM_CNN_ERR_CUDA, "cudaMalloc(%zu): %s", n * sizeof(T), cudaGetErrorString(e));
    // zeroed on the owning stream and finished before the buffer is handed
    // out: a plain cudaMemset would run on the legacy stream, which
    // non-blocking streams are not ordered after, and synchronous copies on
    // the legacy stream are not ordered after the owning stream either
    cudaMemsetAsync(q, 0, n * sizeof(T), stream);
    cudaStreamSynchronize(stream);
    allocs.push_back(q);
    *p = (T *)q;
    return PCOM_CNN_OK;
  }
};

namespace {

int refresh_operands(pcom_cnn *c) {
  k_zero_pad<<<(9 * 64 * 16 + 255) / 256, 256, 0, c->stream>>>(c->param + c->woff[0], c->param + c->woff[4],
                                                                c->param + c->boff[4]);
  for (int l = 0; l < kLayers; ++l) {
    k_to_bf16<<<256, 256, 0, c->stream>>>(c->param + c->woff[l], c->wf[l], wsize(l));
    if (l > 0) k_flip_t<<<256, 256, 0, c->stream>>>(c->param + c->woff[l], c->wd[l], kN[l], kK[l]);
  }
  CC(cudaGetLastError());
  return PCOM_CNN_OK;
}

int check_err(pcom_cnn *c) {
  int e = 0;
  CC(cudaMemcpyAsync(&e, c->err, sizeof e, cudaMemcpyDeviceToHost, c->stream));
  CC(cudaStreamSynchronize(c->stream));
  if (e) {
    cudaMemsetAsync(c->err, 0, sizeof(int), c->stream);
    return cfail(PCOM_CNN_ERR_TIMEOUT, "a tensor-core kernel gave up waiting for its MMAs (bounded wait)");
  }
  return PCOM_CNN_OK;
}

int forward(pcom_cnn *c, const __nv_bfloat16 *x, long long npix) {
  const __nv_bfloat16 *in = x;
  for (int l = 0; l < kLayers; ++l) {
    const float *b = c->param + c->boff[l];
    cudaError_t e;
    if (l < kLayers - 1)
      e = cnn_conv(kK[l], kN[l], in, c->wf[l], b, nullptr, c->act[l + 1 < kLayers ? l + 1 : 0], npix, c->H, c->W,
                   c->periodic_x, 0, 0, c->err, c->stream);
    else
      e = cnn_conv(kK[l], kN[l], in, c->wf[l], b, nullptr, c->y, npix, c->H, c->W, c->periodic_x, 1, kRealOut, c->err,
                   c->stream);
    if (e != cudaSuccess) return cfail(PCOM_CNN_ERR_CUDA, "conv layer %d: %s", l + 1, cudaGetErrorString(e));
    in = c->act[l + 1 < kLayers ? l + 1 : 0];
  }
  return PCOM_CNN_OK;
}

// loss and gradients for the current parameters (grad zeroed first)
int backward(pcom_cnn *c, const __nv_bfloat16 *x, const float *target, const float *mask, long long npix) {
  CC(cudaMemsetAsync(c->grad, 0, c->nparam * sizeof(float), c->stream));
  CC(cudaMemsetAsync(c->scal, 0, 2 * sizeof(double), c->stream));
  k_mask_count<<<592, 256, 0, c->stream>>>(mask, npix * 4, c->scal);
  k_loss<<<592, 256, 0, c->stream>>>(c->y, target, mask, npix, c->scal, c->scal + 1, c->gout);
  CC(cudaGetLastError());
  // layer inputs: x for layer 1, act[l] for layer l+1 (l = 1..4)
  auto layer_in = [&](int l) -> const __nv_bfloat16 * { return l == 0 ? x : c->act[l]; };
  const __nv_bfloat16 *g = c->gout;  // d loss / d (pre-activation of layer l)
  for (int l = kLayers - 1; l >= 0; --l) {
    cudaError_t e = cnn_wgrad(kK[l], kN[l], layer_in(l), g, c->grad + c->woff[l], npix, c->H, c->W, c->periodic_x,
                              c->err, c->stream);
    if (e != cudaSuccess) return cfail(PCOM_CNN_ERR_CUDA, "wgrad layer %d: %s", l + 1, cudaGetErrorString(e));
    k_colsum<<<592, 256, 0, c->stream>>>(g, kN[l], npix, c->grad + c->boff[l]);
    if (l == 0) break;
    // d loss / d (pre-activation of layer l-1) = conv^T(g) * (act[l] > 0)
    __nv_bfloat16 *gn = c->gbuf[l & 1];
    e = cnn_conv(kN[l], kK[l], g, c->wd[l], nullptr, c->act[l], gn, npix, c->H, c->W, c->periodic_x, 2, 0, c->err,
                 c->stream);
    if (e != cudaSuccess) return cfail(PCOM_CNN_ERR_CUDA, "dgrad layer %d: %s", l + 1, cudaGetErrorString(e));
    g = gn;
  }
  CC(cudaGetLastError());
  return PCOM_CNN_OK;
}

}  // namespace

extern "C" {

int pcom_cnn_last_error(char *buf, int32_t len) {
  if (buf && len > 0) {
    strncpy(buf, g_cnn_error.c_str(), (size_t)len - 1);
    buf[len - 1] = 0;
  }
  return (int)g_cnn_error.size();
}

int64_t pcom_cnn_param_count(void) {
  long long n = 0;
  for (int l = 0; l < kLayers; ++l) n += wsize(l) + kN[l];
  return n;
}

int pcom_cnn_create(int32_t H, int32_t W, int32_t max_images, int32_t periodic_x, pcom_cnn **out) {
  if (!out || H < 1 || W < 3 || max_images < 1) return cfail(PCOM_CNN_ERR_ARG, "bad dimensions");
  pcom_cnn *c = new pcom_cnn();
  c->H = H; c->W = W; c->max_img = max_images; c->periodic_x = periodic_x ? 1 : 0;
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { delete c; return cfail(PCOM_CNN_ERR_CUDA, "stream: %s", cudaGetErrorString(e)); }
  long long off = 0;
  for (int l = 0; l < kLayers; ++l) {
    c->woff[l] = off; off += wsize(l);
    c->boff[l] = off; off += kN[l];
  }
  c->nparam = off;
  const long long npix = (long long)H * W * max_images;
  int rc = 0;
  auto A = [&](auto **p, size_t n) { if (!rc) rc = c->alloc(p, n); };
  A(&c->param, off); A(&c->grad, off); A(&c->m, off); A(&c->v, off);
  for (int l = 0; l < kLayers; ++l) { A(&c->wf[l], wsize(l)); A(&c->wd[l], wsize(l)); }
  for (int l = 1; l < kLayers; ++l) A(&c->act[l], npix * 64);
  A(&c->gbuf[0], npix * 64); A(&c->gbuf[1], npix * 64);
  A(&c->gout, npix * 16);
  A(&c->y, npix * 4);
  A(&c->scal, 2);
  A(&c->err, 1);
  if (rc) { cudaStreamDestroy(c->stream); delete c; return rc; }
  *out = c;
  return PCOM_CNN_OK;
}

int pcom_cnn_destroy(pcom_cnn *c) {
  if (!c) return PCOM_CNN_OK;
  cudaStreamSynchronize(c->stream);
  cudaStream_t s = c->stream;
  const bool own = c->own_stream;
  delete c;
  if (own) cudaStreamDestroy(s);
  return PCOM_CNN_OK;
}

int pcom_cnn_set_stream(pcom_cnn *c, void *stream) {
  if (!c) return cfail(PCOM_CNN_ERR_ARG, "null network");
  CC(cudaStreamSynchronize(c->stream));
  // only a stream this network created is destroyed; a caller's stays theirs
  if (c->own_stream) cudaStreamDestroy(c->stream);
  if (stream) {
    c->stream = (cudaStream_t)stream;
    c->own_stream = false;
  } else {
    CC(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    c->own_stream = true;
  }
  return PCOM_CNN_OK;
}

int pcom_cnn_set_params(pcom_cnn *c, const float *host, int64_t n) {
  if (!c || !host || n != c->nparam) return cfail(PCOM_CNN_ERR_ARG, "need %lld parameters", c ? c->nparam : 0LL);
  CC(cudaMemcpyAsync(c->param, host, n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  CC(cudaMemsetAsync(c->m, 0, n * sizeof(float), c->stream));
  CC(cudaMemsetAsync(c->v, 0, n * sizeof(float), c->stream));
  c->step = 0;
  int rc = refresh_operands(c);
  if (rc) return rc;
  CC(cudaStreamSynchronize(c->stream));
  return PCOM_CNN_OK;
}

int pcom_cnn_get_params(pcom_cnn *c, float *host, int64_t n) {
  if (!c || !host || n != c->nparam) return cfail(PCOM_CNN_ERR_ARG, "need %lld parameters", c ? c->nparam : 0LL);
  CC(cudaMemcpyAsync(host, c->param, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  CC(cudaStreamSynchronize(c->stream));
  return PCOM_CNN_OK;
}

int pcom_cnn_forward(pcom_cnn *c, const void *x, float *y, int32_t nimg) {
  if (!c || !x || !y || nimg < 1 || nimg > c->max_img) return cfail(PCOM_CNN_ERR_ARG, "bad arguments");
  const long long npix = (long long)c->H * c->W * nimg;
  int rc = forward(c, (const __nv_bfloat16 *)x, npix);
  if (rc) return rc;
  CC(cudaMemcpyAsync(y, c->y, npix * 4 * sizeof(float), cudaMemcpyDeviceToDevice, c->stream));
  return check_err(c);
}

int pcom_cnn_forward_async(pcom_cnn *c, const void *x, float *y, int32_t nimg) {
  if (!c || !x || !y || nimg < 1 || nimg > c->max_img) return cfail(PCOM_CNN_ERR_ARG, "bad arguments");
  const long long npix = (long long)c->H * c->W * nimg;
  int rc = forward(c, (const __nv_bfloat16 *)x, npix);
  if (rc) return rc;
  CC(cudaMemcpyAsync(y, c->y, npix * 4 * sizeof(float), cudaMemcpyDeviceToDevice, c->stream));
  return PCOM_CNN_OK;
}

int pcom_cnn_gradient(pcom_cnn *c, const void *x, const float *target, const float *mask, int32_t nimg,
                      float *grad_host, double *loss) {
  if (!c || !x || !target || !mask || nimg < 1 || nimg > c->max_img) return cfail(PCOM_CNN_ERR_ARG, "bad arguments");
  const long long npix = (long long)c->H * c->W * nimg;
  int rc = forward(c, (const __nv_bfloat16 *)x, npix);
  if (!rc) rc = backward(c, (const __nv_bfloat16 *)x, target, mask, npix);
  if (rc) return rc;
  if (grad_host) CC(cudaMemcpyAsync(grad_host, c->grad, c->nparam * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  if (loss) CC(cudaMemcpyAsync(loss, c->scal + 1, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  return check_err(c);
}

int pcom_cnn_train_step(pcom_cnn *c, const void *x, const float *target, const float *mask, int32_t nimg, float lr,
                        double *loss) {
  if (!c || !x || !target || !mask || nimg < 1 || nimg > c->max_img) return cfail(PCOM_CNN_ERR_ARG, "bad arguments");
  const long long npix = (long long)c->H * c->W * nimg;
  int rc = forward(c, (const __nv_bfloat16 *)x, npix);
  if (!rc) rc = backward(c, (const __nv_bfloat16 *)x, target, mask, npix);
  if (rc) return rc;
  c->step++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - powf(b1, (float)c->step), c2 = 1.f - powf(b2, (float)c->step);
  k_adam<<<592, 256, 0, c->stream>>>(c->param, c->grad, c->m, c->v, c->nparam, lr, b1, b2, 1e-8f, c1, c2);
  rc = refresh_operands(c);
  if (rc) return rc;
  if (loss) CC(cudaMemcpyAsync(loss, c->scal + 1, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  return check_err(c);
}

int pcom_cnn_conv_layer(int32_t cin, int32_t nout, const void *in, const void *w, const float *bias, const void *aux,
                        void *out, int64_t npix, int32_t H, int32_t W, int32_t periodic_x, int32_t mode, int32_t nstore,
                        void *stream) {
  int *err = nullptr;
  cudaStream_t s = (cudaStream_t)stream;
  CC(cudaMalloc(&err, sizeof(int)));
  CC(cudaMemsetAsync(err, 0, sizeof(int), s));
  cudaError_t e = cnn_conv(cin, nout, (const __nv_bfloat16 *)in, (const __nv_bfloat16 *)w, bias,
                           (const __nv_bfloat16 *)aux, out, npix, H, W, periodic_x, mode, nstore, err, s);
  int h = 0;
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaMemcpy(&h, err, sizeof h, cudaMemcpyDeviceToHost);
  cudaFree(err);
  if (e != cudaSuccess) return cfail(PCOM_CNN_ERR_CUDA, "conv: %s", cudaGetErrorString(e));
  if (h) return cfail(PCOM_CNN_ERR_TIMEOUT, "conv: bounded MMA wait gave up");
  return PCOM_CNN_OK;
}

int pcom_cnn_wgrad_layer(int32_t cin, int32_t nout, const void *in, const void *g, float *dw, int64_t npix, int32_t H,
                         int32_t W, int32_t periodic_x, void *stream) {
  int *err = nullptr;
  cudaStream_t s = (cudaStream_t)stream;
  CC(cudaMalloc(&err, sizeof(int)));
  CC(cudaMemsetAsync(err, 0, sizeof(int), s));
  cudaError_t e = cnn_wgrad(cin, nout, (const __nv_bfloat16 *)in, (const __nv_bfloat16 *)g, dw, npix, H, W, periodic_x,
                            err, s);
  int h = 0;
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaMemcpy(&h, err, sizeof h, cudaMemcpyDeviceToHost);
  cudaFree(err);
  if (e != cudaSuccess) return cfail(PCOM_CNN_ERR_CUDA, "wgrad: %s", cudaGetErrorString(e));
  if (h) return cfail(PCOM_CNN_ERR_TIMEOUT, "wgrad: bounded MMA wait gave up");
  return PCOM_CNN_OK;
}

}  // extern "C"
