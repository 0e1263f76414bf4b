// cnn_oracle.cpp -- CPU restatement of the closure network (test
// infrastructure only): 3x3 'same' convolutions over NHWC images with zero
// padding in y and optional wrap-around in x, their data and weight
// gradients, and the 5-layer network's masked mean-square loss with its
// gradient by back-propagation, all accumulated in FP64.
//
// With round_bf16 = 1 the network reproduces the device path's rounding
// points (BF16 weights, BF16 activations after ReLU, BF16 gradients at the
// layer boundaries) so GPU gradients can be compared at BF16 tolerance; with
// round_bf16 = 0 it is plain FP64 arithmetic, which the tests check against
// central finite differences of the loss.  There is no reference counterpart
// (the reference has no learned component); the layer definitions follow
// include/pcom_cnn.h.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

float bf16r(float x) {  // round to nearest even BF16, kept as float
  uint32_t u;
  std::memcpy(&u, &x, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return x;
  const uint32_t lsb = (u >> 16) & 1u;
  u += 0x7fffu + lsb;
  u &= 0xffff0000u;
  float r;
  std::memcpy(&r, &u, 4);
  return r;
}

long long tap_src(long long p, int t, int H, int W, int periodic_x) {
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

// out[p][n] = sum_t sum_c in[src(p,t)][c] w[t][n][c] (FP64 accumulation)
void conv_acc(int cin, int nout, const double *in, const double *w, long long npix, int H, int W, int px, double *out) {
#pragma omp parallel for schedule(static)
  for (long long p = 0; p < npix; ++p)
    for (int n = 0; n < nout; ++n) {
      double s = 0.0;
      for (int t = 0; t < 9; ++t) {
        const long long q = tap_src(p, t, H, W, px);
        if (q < 0) continue;
        const double *wr = w + ((long long)t * nout + n) * cin;
        const double *xr = in + q * cin;
        for (int c = 0; c < cin; ++c) s += xr[c] * wr[c];
      }
      out[p * nout + n] = s;
    }
}

// d in[q][c] = sum_t sum_n g[p][n] w[t][n][c] with q = src(p, t)
void conv_back_data(int cin, int nout, const double *g, const double *w, long long npix, int H, int W, int px,
                    double *din) {
  std::fill(din, din + npix * cin, 0.0);
  for (long long p = 0; p < npix; ++p)
    for (int t = 0; t < 9; ++t) {
      const long long q = tap_src(p, t, H, W, px);
      if (q < 0) continue;
      for (int n = 0; n < nout; ++n) {
        const double gv = g[p * nout + n];
        const double *wr = w + ((long long)t * nout + n) * cin;
        for (int c = 0; c < cin; ++c) din[q * cin + c] += gv * wr[c];
      }
    }
}

// pixels split into contiguous per-thread ranges, each summed into its own
// buffer; the buffers are added in thread order (deterministic for a given
// thread count)
void conv_back_weight(int cin, int nout, const double *in, const double *g, long long npix, int H, int W, int px,
                      double *dw) {
  const long long nw = 9LL * nout * cin;
  const int nt = std::max(1, omp_get_max_threads());
  std::vector<double> part((size_t)(nt * nw), 0.0);
#pragma omp parallel num_threads(nt)
  {
    const int tid = omp_get_thread_num(), nth = omp_get_num_threads();
    const long long p0 = npix * tid / nth, p1 = npix * (tid + 1) / nth;
    double *acc = part.data() + (size_t)tid * nw;
    for (long long p = p0; p < p1; ++p)
      for (int t = 0; t < 9; ++t) {
        const long long q = tap_src(p, t, H, W, px);
        if (q < 0) continue;
        for (int n = 0; n < nout; ++n) {
          const double gv = g[p * nout + n];
          double *d = acc + ((long long)t * nout + n) * cin;
          for (int c = 0; c < cin; ++c) d[c] += in[q * cin + c] * gv;
        }
      }
  }
  for (int t = 0; t < nt; ++t)
    for (long long i = 0; i < nw; ++i) dw[i] += part[(size_t)t * nw + i];
}

constexpr int L = 5;
constexpr int K_[L] = {16, 64, 64, 64, 64};
constexpr int N_[L] = {64, 64, 64, 64, 16};

}  // namespace

extern "C" {

// single layer, FP32 in/out: mode 0 bias + ReLU, 1 bias (first nstore
// channels), 2 times (aux > 0)
void orc_cnn_conv(int cin, int nout, const float *in, const float *w, const float *bias, const float *aux, float *out,
                  long long npix, int H, int W, int px, int mode, int nstore) {
  std::vector<double> xi(in, in + npix * cin), wi(w, w + 9LL * nout * cin), o((size_t)(npix * nout));
  conv_acc(cin, nout, xi.data(), wi.data(), npix, H, W, px, o.data());
  for (long long p = 0; p < npix; ++p)
    for (int n = 0; n < nout; ++n) {
      const double v = o[p * nout + n];
      if (mode == 0) out[p * nout + n] = (float)std::fmax(v + bias[n], 0.0);
      else if (mode == 1) { if (n < nstore) out[p * nstore + n] = (float)(v + bias[n]); }
      else out[p * nout + n] = aux[p * nout + n] > 0.f ? (float)v : 0.f;
    }
}

void orc_cnn_wgrad(int cin, int nout, const float *in, const float *g, double *dw, long long npix, int H, int W,
                   int px) {
  std::vector<double> xi(in, in + npix * cin), gi(g, g + npix * nout);
  conv_back_weight(cin, nout, xi.data(), gi.data(), npix, H, W, px, dw);
}

long long orc_cnn_param_count() {
  long long n = 0;
  for (int l = 0; l < L; ++l) n += 9LL * N_[l] * K_[l] + N_[l];
  return n;
}

// loss = sum mask (y - target)^2 / sum mask and its gradient (FP64) for the
// network with parameters `par`, inputs x [npix][16]
double orc_cnn_loss_grad(const float *par, const float *x, const float *target, const float *mask, long long npix,
                         int H, int W, int px, int round_bf16, double *grad) {
  auto R = [&](double v) -> double { return round_bf16 ? (double)bf16r((float)v) : v; };
  std::vector<long long> woff(L), boff(L);
  long long off = 0;
  for (int l = 0; l < L; ++l) { woff[l] = off; off += 9LL * N_[l] * K_[l]; boff[l] = off; off += N_[l]; }
  std::vector<std::vector<double>> w(L), act(L + 1);
  for (int l = 0; l < L; ++l) {
    w[l].resize(9LL * N_[l] * K_[l]);
    for (size_t i = 0; i < w[l].size(); ++i) w[l][i] = R(par[woff[l] + i]);
  }
  act[0].assign(x, x + npix * 16);
  for (auto &v : act[0]) v = R(v);
  for (int l = 0; l < L; ++l) {
    act[l + 1].resize((size_t)(npix * N_[l]));
    conv_acc(K_[l], N_[l], act[l].data(), w[l].data(), npix, H, W, px, act[l + 1].data());
    for (long long p = 0; p < npix; ++p)
      for (int n = 0; n < N_[l]; ++n) {
        double &v = act[l + 1][p * N_[l] + n];
        v += par[boff[l] + n];
        if (l < L - 1) v = R(std::fmax(v, 0.0));
        else v = round_bf16 ? (double)(float)v : v;
      }
  }
  double cnt = 0.0, loss = 0.0;
  for (long long i = 0; i < npix * 4; ++i) cnt += mask[i];
  std::vector<double> g((size_t)(npix * 16), 0.0);
  for (long long p = 0; p < npix; ++p)
    for (int q = 0; q < 4; ++q) {
      const double d = (act[L][p * 16 + q] - target[p * 4 + q]) * mask[p * 4 + q];
      loss += d * d;
      g[p * 16 + q] = R(2.0 * d / cnt);
    }
  loss /= cnt;
  std::fill(grad, grad + off, 0.0);
  for (int l = L - 1; l >= 0; --l) {
    conv_back_weight(K_[l], N_[l], act[l].data(), g.data(), npix, H, W, px, grad + woff[l]);
    for (long long p = 0; p < npix; ++p)
      for (int n = 0; n < N_[l]; ++n) grad[boff[l] + n] += g[p * N_[l] + n];
    if (l == 0) break;
    std::vector<double> gi((size_t)(npix * K_[l]));
    conv_back_data(K_[l], N_[l], g.data(), w[l].data(), npix, H, W, px, gi.data());
    for (long long i = 0; i < npix * K_[l]; ++i) gi[i] = act[l][i] > 0.0 ? R(gi[i]) : 0.0;
    g.swap(gi);
  }
  return loss;
}

}  // extern "C"
