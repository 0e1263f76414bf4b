// cnn_kernels.h -- launchers of the closure network's tensor-core kernels
// (internal to libpcomgpu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

// 3x3 convolution as a tcgen05 implicit GEMM (see k_cnn.cu for the modes);
// (cin, nout) in {(16, 64), (64, 64), (64, 16), (16, 16)}
cudaError_t cnn_conv(int cin, int nout, const __nv_bfloat16 *in, const __nv_bfloat16 *w, const float *bias,
                     const __nv_bfloat16 *aux, void *out, long long npix, int H, int W, int periodic_x, int mode,
                     int nstore, int *err, cudaStream_t s);
// weight gradient dw[9][nout][cin] += (accumulates into dw)
cudaError_t cnn_wgrad(int cin, int nout, const __nv_bfloat16 *in, const __nv_bfloat16 *g, float *dw, long long npix,
                      int H, int W, int periodic_x, int *err, cudaStream_t s);
