// ep2d_noalloc.cu -- the RVE averaging for callers that cannot allocate device memory.
//
// Some callers hold every byte of device memory through their own allocator (a host
// framework's caching allocator, a fixed pool sized at start-up) and may not call
// cudaMalloc: a library allocation would grow or fragment memory they account for,
// and cudaMalloc/cudaFree synchronise the device.  ep2d_average_fields_noalloc serves
// them: the caller passes its own device arrays and its own output buffer, and the
// reduction's per-block partial sums go to a fixed array in this file instead of to
// memory the library would allocate.
//
// The array is a file-scope __device__ variable: every GPU that loads the library holds
// it (kMaxBlocks x NAVG doubles, 176 KiB) until the process exits.  Host code must not
// use its name as an address -- on the host the name is only a stand-in -- so the first
// call on each device looks its device address up with cudaGetSymbolAddress while that
// device is current, and passes that pointer to the kernels.  The address belongs to the
// device's current context: after a cudaDeviceReset the module is loaded again, possibly
// elsewhere, so the lookup is keyed on the context too and the first call in a new
// context repeats it.  That first call (per device, and again after a reset) should come
// before any stream capture.  Every call overwrites all the partials it later reads, so
// nothing needs clearing between calls; calls that overlap on the GPU would share the
// array and race.
#include <cuda.h>

#include <cmath>
#include <mutex>
#include <string>

#include "ep2d.h"
#include "ep2d_rve.hpp"
#include "ep2d_types.hpp"

namespace ep2d {
namespace {

constexpr int kRowsPerBlock = 4;
constexpr int kMaxBlocks = 2048;  // rows (ny - 2) up to 8192, i.e. ny <= 8194
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_avg_scratch[kMaxBlocks * NAVG];

std::mutex g_scratch_mu;
double* g_scratch_dev[kMaxDevices] = {};
CUcontext g_scratch_ctx[kMaxDevices] = {};  // the context each cached address belongs to

// cuCtxGetCurrent through the runtime's driver entry point (no link against libcuda)
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
CtxGetCurrentFn ctx_get_current() {
  static CtxGetCurrentFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<CtxGetCurrentFn>(p);
  }();
  return fn;
}

// The scratch array's device address on the current device, looked up once per device
// and context.
int scratch_on_current_device(double** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return fail(EP2D_ERR_NODEV, std::string("no current CUDA device: ") + cudaGetErrorString(e));
  CtxGetCurrentFn get = ctx_get_current();
  if (!get) return fail(EP2D_ERR_CUDA, "cuCtxGetCurrent is not available from the CUDA driver");
  // the context current on this thread; null before the runtime has made one current,
  // which the lookup below does (cudaGetSymbolAddress initialises the device's primary
  // context; nothing here allocates)
  CUcontext ctx = nullptr;
  if (get(&ctx) != CUDA_SUCCESS) ctx = nullptr;
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!ctx || !g_scratch_dev[dev] || g_scratch_ctx[dev] != ctx) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_avg_scratch);
    if (e != cudaSuccess || !p)
      return fail(EP2D_ERR_CUDA, std::string("cudaGetSymbolAddress of the averaging scratch: ") +
                                     cudaGetErrorString(e));
    if (!ctx && (get(&ctx) != CUDA_SUCCESS || !ctx))
      return fail(EP2D_ERR_CUDA, "no current CUDA context after the scratch lookup");
    g_scratch_dev[dev] = static_cast<double*>(p);
    g_scratch_ctx[dev] = ctx;
  }
  *out = g_scratch_dev[dev];
  return EP2D_OK;
}

// Per-block partial sums of EffPlast2D.cu:456-490 over the reference's own layout
// (P, tauXX, tauYY: nX per row; tauXY: nX - 1; Ux: nX + 1; Uy: nX).  Same rows per
// block and element order per thread as the library's pitched averaging kernel.
__global__ void k_average_reference_layout(long nX, long nY, double dX, double dY, const double* __restrict__ P,
                                           const double* __restrict__ txx, const double* __restrict__ tyy,
                                           const double* __restrict__ txy, const double* __restrict__ Ux,
                                           const double* __restrict__ Uy, double nu0, int perOffsetX,
                                           int perOffsetY, double* __restrict__ partials) {
  double acc[NAVG];
#pragma unroll
  for (int k = 0; k < NAVG; k++) acc[k] = 0.0;
  const long jb = 1 + (long)blockIdx.x * kRowsPerBlock;
  const long je = (jb + kRowsPerBlock < nY - 1) ? jb + kRowsPerBlock : nY - 1;
  for (long j = jb; j < je; j++) {
    for (long i = 1 + threadIdx.x; i < nX - 1; i += blockDim.x) {
      const long q = j * nX + i;
      const double pv = P[q], xv = txx[q], yv = tyy[q];
      acc[0] += xv - pv;
      acc[1] += yv - pv;
      acc[2] += txy[j * (nX - 1) + i];
      acc[2] += nu0 * (xv + yv - 2.0 * pv);
      if (i > perOffsetX && i < nX - perOffsetX && j > perOffsetY && j < nY - perOffsetY) {
        const long c = j * (nX - 1) + i, cm = (j - 1) * (nX - 1) + i;
        const long x0 = j * (nX + 1) + i, xm = (j - 1) * (nX + 1) + i, xp = (j + 1) * (nX + 1) + i;
        const long y0 = j * nX + i, yp = (j + 1) * nX + i;
        acc[4] += xv - pv;
        acc[5] += yv - pv;
        acc[6] += 0.25 * (txy[cm - 1] + txy[cm] + txy[c - 1] + txy[c]);
        acc[7] += nu0 * (xv + yv - 2.0 * pv);
        acc[8] += (Ux[x0 + 1] - Ux[x0]) / dX;
        acc[9] += (Uy[yp] - Uy[y0]) / dY;
        acc[10] += 0.125 * ((Ux[x0] - Ux[xm]) / dY + (Uy[y0] - Uy[y0 - 1]) / dX + (Ux[x0 + 1] - Ux[xm + 1]) / dY +
                            (Uy[y0 + 1] - Uy[y0]) / dX + (Ux[xp] - Ux[x0]) / dY + (Uy[yp] - Uy[yp - 1]) / dX +
                            (Ux[xp + 1] - Ux[x0 + 1]) / dY + (Uy[yp + 1] - Uy[yp]) / dX);
      }
    }
  }
  __shared__ double red[NAVG][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NAVG; k++) {
    double v = acc[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[k][w] = v;
  }
  __syncthreads();
  if (threadIdx.x < NAVG) {
    double v = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) v += red[threadIdx.x][q];
    partials[(size_t)blockIdx.x * NAVG + threadIdx.x] = v;
  }
}

// Sums the partials in block order and divides as EffPlast2D.cu:491-503 does.
__global__ void k_average_finish(const double* __restrict__ partials, int nblocks, double div_all, double div_xy,
                                 double div_inner, double* __restrict__ out) {
  const int k = threadIdx.x;
  if (k >= NAVG) return;
  double v = 0.0;
  for (int b = 0; b < nblocks; b++) v += partials[(size_t)b * NAVG + k];
  // out: sigma[0..3], sigma_per[0..3], eps_per[0..2]; sigma[3] is never accumulated
  const double div = (k == 2) ? div_xy : (k < 4 ? div_all : div_inner);
  out[k] = (k == 3 ? 0.0 : v) / div;
}

}  // namespace
}  // namespace ep2d

using ep2d::fail;

extern "C" int ep2d_average_fields_noalloc(int32_t nx, int32_t ny, const double pa[EP2D_NPARS], const double* p,
                                           const double* tau_xx, const double* tau_yy, const double* tau_xy,
                                           const double* ux, const double* uy, double* out_dev, void* stream) {
  if (!pa || !p || !tau_xx || !tau_yy || !tau_xy || !ux || !uy || !out_dev)
    return fail(EP2D_ERR_ARG, "null argument");
  if (nx < 3 || ny < 3) return fail(EP2D_ERR_ARG, "the grid must be at least 3 x 3");
  const int nblocks = (ny - 2 + ep2d::kRowsPerBlock - 1) / ep2d::kRowsPerBlock;
  if (nblocks > ep2d::kMaxBlocks)
    return fail(EP2D_ERR_ARG, "ny = " + std::to_string(ny) + " exceeds " +
                                  std::to_string(ep2d::kMaxBlocks * ep2d::kRowsPerBlock + 2) +
                                  ", the largest grid the scratch-free averaging supports");
  // the checks of the library's parameter validation that concern the averaging
  for (int k = 0; k < EP2D_NPARS; k++)
    if (!std::isfinite(pa[k])) return fail(EP2D_ERR_ARG, "pa[" + std::to_string(k) + "] is not finite");
  if (!(pa[0] > 0.0) || !(pa[1] > 0.0)) return fail(EP2D_ERR_ARG, "dX and dY must be positive");
  if (!(pa[10] >= 1.0) || pa[10] > 64.0) return fail(EP2D_ERR_ARG, "N (pores per side) must be in [1, 64]");
  if (!(3.0 * pa[3] + pa[4] != 0.0)) return fail(EP2D_ERR_ARG, "3 K0 + G0 must not be zero");
  // an error left by the caller's earlier work is reported as such, not as this call's
  const cudaError_t pending = cudaPeekAtLastError();
  if (pending != cudaSuccess)
    return fail(EP2D_ERR_CUDA, std::string("a CUDA error from earlier work is pending (nothing launched): ") +
                                   cudaGetErrorString(pending));
  double* scratch = nullptr;
  const int rc = ep2d::scratch_on_current_device(&scratch);
  if (rc) return rc;
  // host scalars as the reference computes them (EffPlast2D.cu:453-454, :1569)
  const long nX = nx, nY = ny;
  const double K0 = pa[3], G0 = pa[4], nPores = pa[10];
  const double nu0 = (1.5 * K0 - G0) / (3.0 * K0 + G0);
  const int perOffsetX = static_cast<int>(nX / nPores);
  const int perOffsetY = static_cast<int>(nY / nPores);
  const double div_all = static_cast<double>(nX * nY);
  const double div_xy = static_cast<double>((nX - 1) * (nY - 1));
  const double div_inner = static_cast<double>((nX - 2 * perOffsetX) * (nY - 2 * perOffsetY));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  ep2d::k_average_reference_layout<<<nblocks, 256, 0, s>>>(nX, nY, pa[0], pa[1], p, tau_xx, tau_yy, tau_xy, ux, uy,
                                                          nu0, perOffsetX, perOffsetY, scratch);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    ep2d::k_average_finish<<<1, 32, 0, s>>>(scratch, nblocks, div_all, div_xy, div_inner, out_dev);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) return fail(EP2D_ERR_CUDA, std::string("scratch-free averaging: ") + cudaGetErrorString(e));
  return EP2D_OK;
}
