// pcom_kernels.h -- launchers of the device kernels (internal to libpcomgpu).
#pragma once
#include <cuda_runtime.h>
#include "pcom_dev.cuh"

template <typename R>
void launch_alpha_tobot(const DevT<R> &P, cudaStream_t s);
template <typename R>
void launch_pgra2d(const DevT<R> &P, cudaStream_t s);
template <typename R>
void launch_uv2d(const DevT<R> &P, int mode, cudaStream_t s);
template <typename R>
void launch_upwelling(const DevT<R> &P, int with_acw, cudaStream_t s);
template <typename R>
void launch_readyc3d(const DevT<R> &P, cudaStream_t s);
template <typename R>
void launch_clin(const DevT<R> &P, cudaStream_t s);
template <typename R>
void launch_smag(const DevT<R> &P, cudaStream_t s);
template <typename R>
void launch_ssh(const DevT<R> &P, cudaStream_t s);
template <typename R>
void launch_ts(const DevT<R> &P, cudaStream_t s);
template <typename R>
void launch_den_prho(const DevT<R> &P, cudaStream_t s);

// batched forms: member m = blockIdx.z reads its Dev from dPs[m]
struct BatchShape {
  int n;                      // members
  int glo_ni, ni, nj, nk;     // the largest extents over the members
};
enum {
  BK_ALPHA_TOBOT, BK_PGRA2D, BK_UV2D, BK_UPWELLING, BK_READYC3D, BK_CLIN, BK_SMAG, BK_SSH, BK_TS, BK_DEN_PRHO
};
void launch_batch(int kernel, const Dev *dPs, const BatchShape &b, int arg, cudaStream_t s);

size_t trop_smem_bytes(int TX, int TY);
cudaError_t launch_trop(const Dev &P, int TX, int TY, int nblocks, cudaStream_t s);
int trop_max_blocks(int TX, int TY);
// resident variant: one tile per CTA, one region point per thread
size_t trop_res_smem_bytes(int TX, int TY);
bool trop_res_fits(int TX, int TY);
cudaError_t launch_trop_res(const Dev &P, int TX, int TY, cudaStream_t s);
int trop_res_max_blocks(int TX, int TY);
// the same with reciprocal divisions (handle path)
size_t trop_fast_smem_bytes(int TX, int TY);
cudaError_t launch_trop_fast(const Dev &P, int TX, int TY, unsigned long long epoch, cudaStream_t s);
// the resident kernel's synchronisation skeleton (latency floor), same grid
cudaError_t launch_trop_floor(const Dev &P, int TX, int TY, unsigned long long epoch, cudaStream_t s);
int trop_fast_max_blocks(int TX, int TY);
// mixed path: the resident kernel with FP32 arithmetic outside the bottom pressure
cudaError_t launch_trop_mixed(const Dev &P, int TX, int TY, unsigned long long epoch, cudaStream_t s);
int trop_mixed_max_blocks(int TX, int TY);
// batched barotropic subcycle: one persistent launch over the tiles of all members
struct TileRef {
  int m, r0, j0, tw, th;  // member, first interior ring column (0-based), first row, width, height
};

// mixed path, domains too large for the resident kernel: the multi-tile
// kernel with the resident mixed kernel's precision; its per-step FP32
// coefficients (MC_*), masks and FP32 velocity ping-pong live in scratch the
// handle allocates (trop_multi_mixed_scratch_bytes)
enum { MC_BXN, MC_BXS, MC_BYE, MC_BYW, MC_SAM, MC_COR, MC_UT, MC_VT, MC_PRHU, MC_RPRHT, MC_RDEN, MC_COUNT };
struct MultiMixed {
  float *cf;            // [MC_COUNT][n2]
  unsigned char *fl;    // bit 0: lev_u >= 1, bit 1: lev_t >= 1
  float *ub[2], *vb[2]; // barotropic velocities between substeps
  float *vs0[2];        // the first substep's viscosity (u, v)
};
size_t trop_multi_mixed_scratch_bytes(long long n2);
void trop_multi_mixed_bind(MultiMixed &M, void *scratch, long long n2);
int trop_multi_mixed_max_blocks(int TX, int TY);
cudaError_t launch_trop_multi_mixed(const Dev &P, const MultiMixed &M, const TileRef *dtiles, int ntiles, int TX,
                                    int TY, int nblocks, unsigned long long *cnt, int *err, cudaStream_t s);

size_t trop_batch_smem(int TX, int TY);
int trop_batch_max_blocks(int TX, int TY);
cudaError_t launch_trop_batch(const Dev *dPs, const TileRef *dtiles, int ntiles, int TX, int TY, int nblocks,
                              unsigned long long *cnt, int *err, cudaStream_t s);
// the same kernel over the tiles of one domain P (passed by value)
cudaError_t launch_trop_multi(const Dev &P, const TileRef *dtiles, int ntiles, int TX, int TY, int nblocks,
                              unsigned long long *cnt, int *err, cudaStream_t s);
// resident form: one tile per CTA, coefficients in registers (the fast
// kernel over a tile list); all tiles of the group must be co-resident
int trop_group_max_blocks(int TX, int TY);
cudaError_t launch_trop_group(const Dev *dPs, const TileRef *dtiles, int ntiles, int TX, int TY,
                              unsigned long long *cnt, int *err, cudaStream_t s);

// the model constants (literal precision per PCOM_LIT_R8)
void pcom_dev_consts(bool r8, DevConsts &c);
// set the message returned by pcom_gpu_last_error; returns code
int pcom_set_error(int code, const char *msg);

// watchdog: count non-finite values of a field over wet points of the T or U
// grid (mask from lev), atomically added into *count
void launch_nonfinite(const double *f, const int *lev, int nk, long long n2, int planes, unsigned long long *count,
                      cudaStream_t s);
