// pcom_kernels.h -- launchers of the device kernels (internal to libpcomgpu).
#pragma once
#include <cuda_runtime.h>
#include "pcom_dev.cuh"

// batched forms: member m = blockIdx.z reads its Dev from dPs[m]
struct BatchShape {
  int n;                      // members
  int glo_ni, ni, nj, nk;     // the largest extents over the members
};
enum {
  BK_ALPHA_TOBOT, BK_PGRA2D, BK_UV2D, BK_UPWELLING, BK_READYC3D, BK_CLIN, BK_SMAG, BK_SSH, BK_TS, BK_DEN_PRHO
};

// batched barotropic subcycle: one persistent launch over the tiles of all members
struct TileRef {
  int m, r0, j0, tw, th;  // member, first interior ring column (0-based), first row, width, height
};

// mixed path: the resident kernel with FP32 arithmetic outside the bottom pressure
cudaError_t launch_trop_mixed(const Dev &P, int TX, int TY, unsigned long long epoch, cudaStream_t s);
int trop_mixed_max_blocks(int TX, int TY);

// the launchers of the FP64/FP32 step kernels, in an exact (no FMA
// contraction) and a contracted build; a translation unit that defines one of
// them is compiled with PCOM_KNS set to the namespace it defines
namespace kx_exact {
#include "pcom_launchers.inc"
}
namespace kx_fma {
#include "pcom_launchers.inc"
}
#ifndef PCOM_KNS
#define PCOM_KNS kx_exact
#endif

// the model constants (literal precision per PCOM_LIT_R8)
void pcom_dev_consts(bool r8, DevConsts &c);
// set the message returned by pcom_gpu_last_error; returns code
int pcom_set_error(int code, const char *msg);

// watchdog: count non-finite values of a field over wet points of the T or U
// grid (mask from lev), atomically added into *count
void launch_nonfinite(const double *f, const int *lev, int nk, long long n2, int planes, unsigned long long *count,
                      cudaStream_t s);
