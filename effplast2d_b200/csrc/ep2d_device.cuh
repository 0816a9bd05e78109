// ep2d_device.cuh -- sm_100a kernels of the pseudo-transient elastoplastic RVE solver.
//
// Device layout (one RVE): every field is a row-major array with x (i) fastest and one
// common row pitch (a multiple of 32 elements, >= nx + 1), so the reference's arrays
// (EffPlast2D.cu:1577-1604: n x n nodes, (n-1)^2 corners, (n+1) x n and n x (n+1)
// faces) all index as base[j * pitch + i].  Displacements are double-buffered
// (ping-pong) so that one launch can read the old field in its halo while writing the
// new one; velocities are updated in place (each face reads only its own old value).
//
// Materials are not stored as K/G arrays: a one-byte mask per node carries
//   M_MAT    node inside a pore by SetMaterials' test  -> K = 0.01 K0, G = 0.01 G0
//   M_NODE   node inside a pore by ComputeStress' test -> P = tauXX = tauYY = 0
//   M_CORNER corner (i, j) inside a pore               -> tauXY = 0
//   M_MAT_R  M_MAT of node (i + 1, j)                   (the corner's lower-right node)
// which reproduces K, G (EffPlast2D.cu:708-728) and the kernel masks (:77-97) exactly
// while moving 1 byte per cell instead of 16 (K, G) plus 8 (P0, identically 0).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "ep2d_types.hpp"

namespace ep2d {

// ---------------------------------------------------------------------------------
// Pore tests.
//
// host_pore_test: SetMaterials' / ComputeEffParams' test (EffPlast2D.cu:719-720,
// :523-524, :539-540).  The reference evaluates it on the CPU, operation by operation;
// the *_rn intrinsics below are never contracted into fused multiply-adds, so the
// device result is bit-identical to the host one.
// ---------------------------------------------------------------------------------
__device__ __forceinline__ bool host_pore_test(double x, double y, double Lx, double Ly, double nPores,
                                               double rad) {
  const double ax = __dmul_rn(__dmul_rn(0.5, Lx), __dsub_rn(1.0, __ddiv_rn(1.0, nPores)));
  const double ay = __dmul_rn(__dmul_rn(0.5, Ly), __dsub_rn(1.0, __ddiv_rn(1.0, nPores)));
  const double sx = __ddiv_rn(Lx, nPores), sy = __ddiv_rn(Ly, nPores);
  for (int k = 0; k < nPores; k++) {
    for (int l = 0; l < nPores; l++) {
      const double a = __dadd_rn(__dsub_rn(x, ax), __dmul_rn(sx, (double)k));
      const double b = __dadd_rn(__dsub_rn(y, ay), __dmul_rn(sy, (double)l));
      if (__dsqrt_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b))) < rad) return true;
    }
  }
  return false;
}

// Face / node positions of the host-side tests, exact (no contraction).
__device__ __forceinline__ double host_pos(double h, long n_minus, long idx) {
  // -0.5 * h * n_minus + h * idx, evaluated as the reference's host code does
  return __dadd_rn(__dmul_rn(__dmul_rn(-0.5, h), (double)n_minus), __dmul_rn(h, (double)idx));
}

// Mask setup: one thread per node.
__global__ void k_mask(Geo g, uint8_t* __restrict__ mask) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= g.nx || j >= g.ny) return;
  const long nX = g.nx, nY = g.ny;
  const double dX = g.dX, dY = g.dY, rad = g.rad, N = g.nPores;
  uint8_t m = 0;
  {  // SetMaterials, EffPlast2D.cu:713-726
    const double x = host_pos(dX, nX - 1, i);
    const double y = host_pos(dY, nY - 1, j);
    const double Lx = __dmul_rn(dX, (double)(nX - 1));
    const double Ly = __dmul_rn(dY, (double)(nY - 1));
    if (host_pore_test(x, y, Lx, Ly, N, rad)) m |= M_MAT;
    if (i + 1 < g.nx && host_pore_test(host_pos(dX, nX - 1, i + 1), y, Lx, Ly, N, rad)) m |= M_MAT_R;
  }
  // ComputeStress' own tests, EffPlast2D.cu:77-97, written as the reference writes them
  // so that the CUDA compiler treats the arithmetic the same way.
  for (int k = 0; k < N; k++) {
    for (int l = 0; l < N; l++) {
      if (sqrt((-0.5 * dX * (nX - 1) + dX * i - 0.5 * dX * (nX - 1) * (1.0 - 1.0 / N) + (dX * (nX - 1) / N) * k) *
                   (-0.5 * dX * (nX - 1) + dX * i - 0.5 * dX * (nX - 1) * (1.0 - 1.0 / N) + (dX * (nX - 1) / N) * k) +
               (-0.5 * dY * (nY - 1) + dY * j - 0.5 * dY * (nY - 1) * (1.0 - 1.0 / N) + (dY * (nY - 1) / N) * l) *
                   (-0.5 * dY * (nY - 1) + dY * j - 0.5 * dY * (nY - 1) * (1.0 - 1.0 / N) + (dY * (nY - 1) / N) * l)) < rad) {
        m |= M_NODE;
      }
      if (i < nX - 1 && j < nY - 1) {
        if (sqrt((-0.5 * dX * (nX - 2) + dX * i - 0.5 * dX * (nX - 1) * (1.0 - 1.0 / N) + (dX * (nX - 1) / N) * k) *
                     (-0.5 * dX * (nX - 2) + dX * i - 0.5 * dX * (nX - 1) * (1.0 - 1.0 / N) + (dX * (nX - 1) / N) * k) +
                 (-0.5 * dY * (nY - 2) + dY * j - 0.5 * dY * (nY - 1) * (1.0 - 1.0 / N) + (dY * (nY - 1) / N) * l) *
                     (-0.5 * dY * (nY - 2) + dY * j - 0.5 * dY * (nY - 1) * (1.0 - 1.0 / N) + (dY * (nY - 1) / N) * l)) < rad) {
          m |= M_CORNER;
        }
      }
    }
  }
  mask[(size_t)j * g.pitch + i] = m;
}

// ---------------------------------------------------------------------------------
// Affine preload / load increment (EffPlast2D.cu:349-381): U += affine strain field on
// every face, into both buffers.  The reference does this on the host; the *_rn
// arithmetic reproduces its rounding exactly.  zero_first: step 0 starts from U = 0
// (EffPlast2D.cu:329-333).
// ---------------------------------------------------------------------------------
__global__ void k_preload(Geo g, double* ux0, double* ux1, double* uy0, double* uy1, int src, double dUxdx,
                          double dUydy, double dUxdy, int zero_first) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const long nX = g.nx, nY = g.ny;
  const double dUydx = dUxdy;
  const double* uxs = src ? ux1 : ux0;
  const double* uys = src ? uy1 : uy0;
  if (i <= nX && j < nY) {  // Ux: (nX + 1) x nY
    const size_t q = (size_t)j * g.pitch + i;
    const double a = __dmul_rn(host_pos(g.dX, nX, i), dUxdx);
    const double b = __dmul_rn(host_pos(g.dY, nY - 1, j), dUxdy);
    const double v = __dadd_rn(zero_first ? 0.0 : uxs[q], __dadd_rn(a, b));
    ux0[q] = v;
    ux1[q] = v;
  }
  if (i < nX && j <= nY) {  // Uy: nX x (nY + 1)
    const size_t q = (size_t)j * g.pitch + i;
    const double a = __dmul_rn(host_pos(g.dY, nY, j), dUydy);
    const double b = __dmul_rn(host_pos(g.dX, nX - 1, i), dUydx);
    const double v = __dadd_rn(zero_first ? 0.0 : uys[q], __dadd_rn(a, b));
    uy0[q] = v;
    uy1[q] = v;
  }
}

// ---------------------------------------------------------------------------------
// FP64 state <-> FP32 bulk state.  Ua, the affine field of the preloads, at the faces'
// positions k_preload uses: Ux = Exx x + Exy y, Uy = Eyy y + Exy x (k_preload adds
// dUxdy to both, EffPlast2D.cu:370-381).  To FP32: u' = U - Ua rounded to float, into
// both buffers; back: U = Ua + u', into both buffers.  The velocities are float in both
// states and stay where they are.
// ---------------------------------------------------------------------------------
__device__ __forceinline__ double affine_ux(const Geo& g, int i, int j, double Exx, double Exy) {
  return __dadd_rn(__dmul_rn(host_pos(g.dX, g.nx, i), Exx), __dmul_rn(host_pos(g.dY, g.ny - 1, j), Exy));
}
__device__ __forceinline__ double affine_uy(const Geo& g, int i, int j, double Eyy, double Exy) {
  return __dadd_rn(__dmul_rn(host_pos(g.dY, g.ny, j), Eyy), __dmul_rn(host_pos(g.dX, g.nx - 1, i), Exy));
}

__global__ void k_to_f32(Geo g, const double* __restrict__ ux, const double* __restrict__ uy, float* ux32a,
                         float* ux32b, float* uy32a, float* uy32b, double Exx, double Eyy, double Exy) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const size_t q = (size_t)j * g.pitch + i;
  if (i <= g.nx && j < g.ny) {
    const float v = (float)__dsub_rn(ux[q], affine_ux(g, i, j, Exx, Exy));
    ux32a[q] = v;
    ux32b[q] = v;
  }
  if (i < g.nx && j <= g.ny) {
    const float v = (float)__dsub_rn(uy[q], affine_uy(g, i, j, Eyy, Exy));
    uy32a[q] = v;
    uy32b[q] = v;
  }
}

__global__ void k_from_f32(Geo g, const float* __restrict__ ux32, const float* __restrict__ uy32, double* uxa,
                           double* uxb, double* uya, double* uyb, double Exx, double Eyy, double Exy) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const size_t q = (size_t)j * g.pitch + i;
  if (i <= g.nx && j < g.ny) {
    const double v = __dadd_rn(affine_ux(g, i, j, Exx, Exy), (double)ux32[q]);
    uxa[q] = v;
    uxb[q] = v;
  }
  if (i < g.nx && j <= g.ny) {
    const double v = __dadd_rn(affine_uy(g, i, j, Eyy, Exy), (double)uy32[q]);
    uya[q] = v;
    uyb[q] = v;
  }
}

// ---------------------------------------------------------------------------------
// RVE averaging (EffPlast2D.cu:430-503) as a deterministic two-level reduction:
// per-block partials in a fixed order, then one block sums the partials in order.
// Sums: 0..3 sigma (sigma[3] stays 0 as in the reference), 4..7 sigmaPer, 8..10 epsPer.
// ---------------------------------------------------------------------------------

template <typename T>
__device__ __forceinline__ void block_sum_into(T (&acc)[NAVG], T* out) {
  __shared__ T red[NAVG][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NAVG; k++) {
    T v = acc[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[k][w] = v;
  }
  __syncthreads();
  if (threadIdx.x < NAVG) {
    T v = 0;
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) v += red[threadIdx.x][q];
    out[threadIdx.x] = v;
  }
}

// grid: one block per group of rows; block of 256 threads, x-fastest
__global__ void k_average(Geo g, const double* __restrict__ P, const double* __restrict__ txx,
                          const double* __restrict__ tyy, const double* __restrict__ txy,
                          const double* __restrict__ Ux, const double* __restrict__ Uy, double nu0, int perOffsetX,
                          int perOffsetY, int rows_per_block, double* __restrict__ partials) {
  const long nX = g.nx, nY = g.ny;
  const size_t pitch = (size_t)g.pitch;
  const double dX = g.dX, dY = g.dY;
  double acc[NAVG];
#pragma unroll
  for (int k = 0; k < NAVG; k++) acc[k] = 0.0;
  const long jb = 1 + (long)blockIdx.x * rows_per_block;
  const long je = (jb + rows_per_block < nY - 1) ? jb + rows_per_block : nY - 1;
  for (long j = jb; j < je; j++) {
    for (long i = 1 + threadIdx.x; i < nX - 1; i += blockDim.x) {
      const size_t q = j * pitch + i;
      const double pv = P[q], xv = txx[q], yv = tyy[q];
      acc[0] += xv - pv;
      acc[1] += yv - pv;
      acc[2] += txy[q];
      acc[2] += nu0 * (xv + yv - 2.0 * pv);
      if (i > perOffsetX && i < nX - perOffsetX && j > perOffsetY && j < nY - perOffsetY) {
        acc[4] += xv - pv;
        acc[5] += yv - pv;
        acc[6] += 0.25 * (txy[q - pitch - 1] + txy[q - pitch] + txy[q - 1] + txy[q]);
        acc[7] += nu0 * (xv + yv - 2.0 * pv);
        acc[8] += (Ux[q + 1] - Ux[q]) / dX;
        acc[9] += (Uy[q + pitch] - Uy[q]) / dY;
        acc[10] += 0.125 * ((Ux[q] - Ux[q - pitch]) / dY + (Uy[q] - Uy[q - 1]) / dX +
                            (Ux[q + 1] - Ux[q - pitch + 1]) / dY + (Uy[q + 1] - Uy[q]) / dX +
                            (Ux[q + pitch] - Ux[q]) / dY + (Uy[q + pitch] - Uy[q + pitch - 1]) / dX +
                            (Ux[q + pitch + 1] - Ux[q + 1]) / dY + (Uy[q + pitch + 1] - Uy[q + pitch]) / dX);
      }
    }
  }
  block_sum_into<double>(acc, partials + (size_t)blockIdx.x * NAVG);
}

__global__ void k_sum_partials(const double* __restrict__ partials, int nblocks, int width, double* __restrict__ out) {
  const int k = threadIdx.x;
  if (k >= width) return;
  double v = 0.0;
  for (int b = 0; b < nblocks; b++) v += partials[(size_t)b * width + k];
  out[k] = v;
}

// ---------------------------------------------------------------------------------
// Boundary sums of getDeltaP_honest (:825-853), getDeltaP_periodic (:854-882) and
// getTauInfty_honest (:925-942).  Element (row, col) of a flat reference index f is
// (f / nX, f % nX), so the reference's `j * nX + nY - 1` is kept literally.
// out: [0] dPx [1] dPy [2] dPperX [3] dPperY [4] tauX [5] tauY
// ---------------------------------------------------------------------------------
// For ny > 2 nx the reference's `j * nX + nY - 1` runs past its array (undefined
// behaviour there); such reads count as 0 here.
__device__ __forceinline__ double at_flat(const double* a, long f, long nX, long nY, size_t pitch) {
  if (f < 0 || f >= nX * nY) return 0.0;
  return a[(size_t)(f / nX) * pitch + (size_t)(f % nX)];
}

__global__ void k_boundary(Geo g, const double* __restrict__ P, const double* __restrict__ txx,
                           const double* __restrict__ tyy, double* __restrict__ out) {
  const long nX = g.nx, nY = g.ny;
  const size_t pitch = (size_t)g.pitch;
  double acc[NAVG];
#pragma unroll
  for (int k = 0; k < NAVG; k++) acc[k] = 0.0;
  for (long i = 1 + threadIdx.x; i < nX - 1; i += blockDim.x) {
    const long f0 = 0 * nX + i, f1 = (nY - 1) * nX + i;
    const double p0 = at_flat(P, f0, nX, nY, pitch), x0 = at_flat(txx, f0, nX, nY, pitch), y0 = at_flat(tyy, f0, nX, nY, pitch);
    const double p1 = at_flat(P, f1, nX, nY, pitch), x1 = at_flat(txx, f1, nX, nY, pitch), y1 = at_flat(tyy, f1, nX, nY, pitch);
    acc[0] += x0 - p0;
    acc[0] += y0 - p0;
    acc[0] += x1 - p1;
    acc[0] += y1 - p1;
    acc[4] += x0 - y0;
    acc[4] += x1 - y1;
  }
  for (long j = 1 + threadIdx.x; j < nY - 1; j += blockDim.x) {
    const long f0 = j * nX + 0, f1 = j * nX + nY - 1;
    const double p0 = at_flat(P, f0, nX, nY, pitch), x0 = at_flat(txx, f0, nX, nY, pitch), y0 = at_flat(tyy, f0, nX, nY, pitch);
    const double p1 = at_flat(P, f1, nX, nY, pitch), x1 = at_flat(txx, f1, nX, nY, pitch), y1 = at_flat(tyy, f1, nX, nY, pitch);
    acc[1] += x0 - p0;
    acc[1] += y0 - p0;
    acc[1] += x1 - p1;
    acc[1] += y1 - p1;
    acc[5] += x0 - y0;
    acc[5] += x1 - y1;
  }
  if (g.nPores > 2) {
    const int nP = (int)g.nPores;
    const long r0 = nY / nP, r1 = nY * (nP - 1) / nP;
    for (long i = nX / nP + threadIdx.x; i < nX * (nP - 1) / nP; i += blockDim.x) {
      const long f0 = r0 * nX + i, f1 = r1 * nX + i;
      const double p0 = at_flat(P, f0, nX, nY, pitch), p1 = at_flat(P, f1, nX, nY, pitch);
      acc[2] += at_flat(txx, f0, nX, nY, pitch) - p0;
      acc[2] += at_flat(tyy, f0, nX, nY, pitch) - p0;
      acc[2] += at_flat(txx, f1, nX, nY, pitch) - p1;
      acc[2] += at_flat(tyy, f1, nX, nY, pitch) - p1;
    }
    const long c0 = nX / nP, c1 = nX * (nP - 2) / nP;
    for (long j = nY / nP + threadIdx.x; j < nY * (nP - 1) / g.nPores; j += blockDim.x) {
      const long f0 = j * nX + c0, f1 = j * nX + c1;
      const double p0 = at_flat(P, f0, nX, nY, pitch), p1 = at_flat(P, f1, nX, nY, pitch);
      acc[3] += at_flat(txx, f0, nX, nY, pitch) - p0;
      acc[3] += at_flat(tyy, f0, nX, nY, pitch) - p0;
      acc[3] += at_flat(txx, f1, nX, nY, pitch) - p1;
      acc[3] += at_flat(tyy, f1, nX, nY, pitch) - p1;
    }
  }
  block_sum_into<double>(acc, out);
}

// Gather of the hole-edge samples (EffPlast2D.cu:552-595): idx[k] encodes field
// (0 = Ux, 1 = Uy) in bit 62 and the reference's flat index in the low bits.
__global__ void k_gather(Geo g, const double* __restrict__ Ux, const double* __restrict__ Uy,
                         const unsigned long long* __restrict__ idx, int n, double* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const unsigned long long e = idx[k];
  const bool isy = (e >> 62) & 1ull;
  const unsigned long long fl = e & ((1ull << 62) - 1);
  const unsigned long long w = isy ? (unsigned long long)g.nx : (unsigned long long)g.nx + 1;
  const double* a = isy ? Uy : Ux;
  out[k] = a[(fl / w) * (unsigned long long)g.pitch + fl % w];
}

// SaveAnStatic2D's numerical fields (EffPlast2D.cu:1109-1134) from the state with the
// displacements zeroed inside the pores (EffPlast2D.cu:514-547).  Output unpadded.
__global__ void k_static_fields(Geo g, const double* __restrict__ Ux, const double* __restrict__ Uy,
                                const double* __restrict__ P, const double* __restrict__ txx,
                                const double* __restrict__ tyy, const double* __restrict__ txy,
                                double* __restrict__ unu, double* __restrict__ j1, double* __restrict__ j2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const long nX = g.nx, nY = g.ny;
  if (i >= nX || j >= nY) return;
  const size_t pitch = (size_t)g.pitch;
  const double Lx = __dmul_rn(g.dX, (double)(nX - 1)), Ly = __dmul_rn(g.dY, (double)(nY - 1));
  auto uxz = [&](long fi, long fj) {
    return host_pore_test(host_pos(g.dX, nX, fi), host_pos(g.dY, nY - 1, fj), Lx, Ly, g.nPores, g.rad)
               ? 0.0 : Ux[fj * pitch + fi];
  };
  auto uyz = [&](long fi, long fj) {
    return host_pore_test(host_pos(g.dX, nX - 1, fi), host_pos(g.dY, nY, fj), Lx, Ly, g.nPores, g.rad)
               ? 0.0 : Uy[fj * pitch + fi];
  };
  const double ux = 0.5 * (uxz(i, j) + uxz(i + 1, j));
  const double uy = 0.5 * (uyz(i, j) + uyz(i, j + 1));
  unu[j * nX + i] = sqrt(ux * ux + uy * uy);
  if (i < nX - 1 && j < nY - 1) {
    const size_t q = j * pitch + i;
    const double Sxx = 0.25 * (-P[q] + txx[q] + -P[q + 1] + txx[q + 1] + -P[q + pitch] + txx[q + pitch] +
                               -P[q + pitch + 1] + txx[q + pitch + 1]);
    const double Syy = 0.25 * (-P[q] + tyy[q] + -P[q + 1] + tyy[q + 1] + -P[q + pitch] + tyy[q + pitch] +
                               -P[q + pitch + 1] + tyy[q + pitch + 1]);
    const double Sxy = txy[q];
    j1[j * (nX - 1) + i] = 0.5 * (Sxx + Syy);
    j2[j * (nX - 1) + i] = 0.5 * ((Sxx - Syy) * (Sxx - Syy) + 4.0 * Sxy * Sxy);
  }
}


// The plastic-zone map and the stresses in polar coordinates around the centre that
// get_sigma_2D.m:170-194 computes after its solve, here from the recorded final state.
// plastic = (node yields) + (yielding corners among the four around the node), as
// Plast + PlastXY there; a node yields if its recorded (returned) J2 reached coh (to
// 1e-12 relative), a corner if its recorded trial J2XY exceeds coh.  In the plastic zone
// (plastic > 0): the numerical sigma_rr, sigma_phiphi from tauXX - P, tauYY - P and
// tauXYav rotated to polar axes, and the analytic ones
// -P0 + sign(load) 2 coh (log(sqrt(r)) [+ 1]) / sqrt(2), P0 = 0; zero elsewhere and
// inside the pore (r < rad).  Output unpadded, node (i, j) at j*nx + i.
// mask != nullptr: the zone accumulated by the tracking launches (M_YN of the node,
// M_YC of the corners around it: get_sigma_2D.m:126-138, :170-173); else from the
// recorded state (J2 at coh after the return, J2XY above coh).
__global__ void k_polar_fields(Geo g, const double* __restrict__ P, const double* __restrict__ txx,
                               const double* __restrict__ tyy, const double* __restrict__ txyav,
                               const double* __restrict__ j2, const double* __restrict__ j2xy,
                               const uint8_t* __restrict__ mask, double sgn, double* __restrict__ snrr,
                               double* __restrict__ snff, double* __restrict__ sarr, double* __restrict__ saff,
                               uint8_t* __restrict__ plast) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int nx = g.nx, ny = g.ny;
  if (i >= nx || j >= ny) return;
  const size_t pitch = (size_t)g.pitch, q = j * pitch + i;
  const double coh = g.coh;
  int count = mask ? ((mask[q] & M_YN) ? 1 : 0) : ((j2[q] >= coh * (1.0 - 1e-12)) ? 1 : 0);
  for (int dj = -1; dj <= 0; dj++)
    for (int di = -1; di <= 0; di++) {
      const int ci = i + di, cj = j + dj;
      if (ci >= 0 && ci < nx - 1 && cj >= 0 && cj < ny - 1 &&
          (mask ? (mask[cj * pitch + ci] & M_YC) != 0 : j2xy[cj * pitch + ci] > coh))
        count++;
    }
  const double x = -0.5 * g.dX * (nx - 1) + g.dX * i;
  const double y = -0.5 * g.dY * (ny - 1) + g.dY * j;
  const double r = sqrt(x * x + y * y);
  const double s = y / r, c = x / r;
  const double sxx = txx[q] - P[q], syy = tyy[q] - P[q], sxy = txyav[q];
  double a = 0.0, b = 0.0, ar = 0.0, af = 0.0;
  if (count > 0) {
    a = sxx * c * c + 2.0 * sxy * s * c + syy * s * s;
    b = sxx * s * s - 2.0 * sxy * s * c + syy * c * c;
    const double lg = log(sqrt(r));
    ar = sgn * 2.0 * coh * lg / sqrt(2.0);
    af = sgn * 2.0 * coh * (lg + 1.0) / sqrt(2.0);
  }
  if (r < g.rad) a = b = ar = af = 0.0;
  const size_t o = (size_t)j * nx + i;
  snrr[o] = a;
  snff[o] = b;
  sarr[o] = ar;
  saff[o] = af;
  plast[o] = (uint8_t)count;
}

__global__ void k_clear_track(Geo g, uint8_t* __restrict__ mask) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= g.nx || j >= g.ny) return;
  const size_t q = (size_t)j * g.pitch + i;
  mask[q] = (uint8_t)(mask[q] & ~(M_YN | M_YC));
}

// ---------------------------------------------------------------------------------
// Analytic static solution and error maps (SaveAnStatic2D, EffPlast2D.cu:1060-1292;
// getAnalytic* :989-1059).  Complex FP64 on the device.  The complex helpers follow the
// textbook definitions: product and quotient componentwise (quotient by Smith's
// method), log z = (log|z|, atan2), exp z = e^re (cos, sin), and the principal square
// root by the half-angle formulas; CUDA's real math functions do the rest.  Zone tests
// and positions use the non-contracting *_rn arithmetic so that every node falls in
// the same zone as in the reference's host evaluation.
// ---------------------------------------------------------------------------------
struct cplx {
  double re, im;
};
__device__ __forceinline__ cplx c_mk(double r, double i) { return cplx{r, i}; }
__device__ __forceinline__ cplx c_add(cplx a, cplx b) { return cplx{a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ cplx c_sub(cplx a, cplx b) { return cplx{a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ cplx c_addr(cplx a, double r) { return cplx{a.re + r, a.im}; }  // complex + real
__device__ __forceinline__ cplx c_rsub(double r, cplx a) { return cplx{r - a.re, 0.0 - a.im}; }  // real - complex
__device__ __forceinline__ cplx c_radd(double r, cplx a) { return cplx{r + a.re, a.im}; }  // real + complex
__device__ __forceinline__ cplx c_scale(double s, cplx a) { return cplx{s * a.re, s * a.im}; }
__device__ __forceinline__ cplx c_divr(cplx a, double s) { return cplx{a.re / s, a.im / s}; }
__device__ __forceinline__ cplx c_conj(cplx a) { return cplx{a.re, -a.im}; }
__device__ __forceinline__ cplx c_mul(cplx a, cplx b) {
  return cplx{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__device__ __forceinline__ cplx c_div(cplx a, cplx b) {  // Smith (1962)
  if (fabs(b.re) >= fabs(b.im)) {
    const double r = b.im / b.re, den = b.re + b.im * r;
    return cplx{(a.re + a.im * r) / den, (a.im - a.re * r) / den};
  }
  const double r = b.re / b.im, den = b.re * r + b.im;
  return cplx{(a.re * r + a.im) / den, (a.im * r - a.re) / den};
}
__device__ __forceinline__ cplx c_rdiv(double s, cplx b) { return c_div(cplx{s, 0.0}, b); }
__device__ __forceinline__ double c_abs(cplx a) { return hypot(a.re, a.im); }
__device__ __forceinline__ double c_arg(cplx a) { return atan2(a.im, a.re); }
__device__ __forceinline__ cplx c_log(cplx a) { return cplx{log(c_abs(a)), c_arg(a)}; }
__device__ __forceinline__ cplx c_exp(cplx a) {
  double s, c;
  sincos(a.im, &s, &c);
  const double e = exp(a.re);
  return cplx{e * c, e * s};
}
__device__ __forceinline__ cplx c_sqrt(cplx a) {  // principal branch, half-angle formulas
  if (a.re == 0.0 && a.im == 0.0) return cplx{0.0, a.im};
  const double m = c_abs(a);
  if (a.re >= 0.0) {
    const double t = sqrt(0.5 * (m + a.re));
    return cplx{t, a.im / (2.0 * t)};
  }
  const double t = sqrt(0.5 * (m - a.re));
  return cplx{fabs(a.im) / (2.0 * t), copysign(t, a.im)};
}

struct AnalyticCore {
  cplx zeta, w, dw, wv, Phi, Psi;
};

// getAnalytic, EffPlast2D.cu:989-1012
__device__ AnalyticCore an_core(const AnParams& a, double x, double y) {
  AnalyticCore o;
  const cplx z = c_mk(x, y);
  double signx = x > 0.0 ? 1.0 : -1.0;
  if (fabs(x) < 2.220446049250313e-16) signx = 1.0;
  o.zeta = c_divr(c_divr(c_add(z, c_scale(signx, c_sqrt(c_addr(c_mul(z, z), 4.0 * a.c0 * a.c0 * a.kappa)))), 2.0), a.c0);
  o.w = c_scale(a.c0, c_sub(o.zeta, c_rdiv(a.kappa, o.zeta)));
  o.dw = c_scale(a.c0, c_radd(1.0, c_rdiv(a.kappa, c_mul(o.zeta, o.zeta))));
  o.wv = c_scale(a.c0, c_sub(c_rdiv(1.0, o.zeta), c_scale(a.kappa, o.zeta)));
  o.Phi = c_rsub(-a.Y * a.xi / 2.0, c_scale(a.Y * a.xi, c_log(c_divr(c_div(o.w, o.zeta), a.rad))));
  o.Psi = c_div(c_mul(c_rdiv(-a.Y * a.xi, o.zeta), o.wv), o.dw);
  return o;
}

// getAnalyticUelast, EffPlast2D.cu:1014-1026
__device__ double an_u_elast_abs(const AnParams& a, double x, double y) {
  const AnalyticCore o = an_core(a, x, y);
  const cplx lg = c_log(c_divr(c_div(o.w, o.zeta), a.rad));
  const cplx phi = c_sub(c_mul(c_scale(-a.Y * a.xi, o.w), c_addr(lg, 0.5)), c_rdiv(2.0 * a.c0 * a.tauInfty, o.zeta));
  const cplx psi = c_scale(a.c0 * a.Y * a.xi, c_add(c_rdiv(1.0, o.zeta), c_scale(a.kappa, o.zeta)));
  const cplx dphi = c_mul(o.Phi, o.dw);
  const double k = 1.0 + 6.0 * a.G0 / (a.G0 + 3.0 * a.K0);
  const cplx U = c_divr(c_divr(c_sub(c_sub(c_scale(k, phi), c_mul(c_div(o.w, c_conj(o.dw)), c_conj(dphi))), c_conj(psi)), 2.0),
                        a.G0);
  return c_abs(U);
}

// getAnalyticUrHydro, EffPlast2D.cu:1027-1029
__device__ __forceinline__ double an_ur_hydro(const AnParams& a, double r) {
  return -0.5 * a.Y * a.rad * a.rad * exp((a.deltaP - a.Y) / a.Y) / (a.G0 * r);
}

// getAnalyticJelast, EffPlast2D.cu:1036-1051
__device__ void an_j_elast(const AnParams& a, double x, double y, double* J1, double* J2) {
  const AnalyticCore o = an_core(a, x, y);
  const cplx z = c_mk(x, y);
  const cplx dPhi = c_div(c_rdiv(-2.0 * a.xi * a.Y * a.kappa, o.zeta), c_addr(c_mul(o.zeta, o.zeta), -a.kappa));
  const double ang = -2.0 * c_arg(z);
  const cplx e = c_exp(c_mk(ang * 0.0, ang * 1.0));
  const cplx F = c_div(c_scale(2.0, c_add(c_mul(c_div(c_conj(o.w), o.dw), dPhi), o.Psi)), e);
  const double Srr = 2.0 * o.Phi.re - F.re / 2.0;
  const double Sff = 2.0 * o.Phi.re + F.re / 2.0;
  const double Srf = F.im / 2.0;
  *J1 = 0.5 * (Srr + Sff);
  *J2 = 0.5 * ((Srr - Sff) * (Srr - Sff) + 4.0 * Srf * Srf);
}

__device__ __forceinline__ double sq_rn(double v) { return __dmul_rn(v, v); }

// One thread per node; stats[blockIdx][8] = Umax, Usum, Un, J1max, J1sum, J2max, J2sum, Jn
__global__ void k_analytic(Geo g, AnParams a, const double* __restrict__ unu, const double* __restrict__ j1nu,
                           const double* __restrict__ j2nu, double* __restrict__ uan, double* __restrict__ eu,
                           double* __restrict__ j1an, double* __restrict__ j2an, double* __restrict__ ej1,
                           double* __restrict__ ej2, double* __restrict__ stats) {
  const long nX = g.nx, nY = g.ny;
  double st[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const long total = nX * nY;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const long j = e / nX, i = e - j * nX;
    const long q = j * nX + i;
    const double x = host_pos(g.dX, nX - 1, i), y = host_pos(g.dY, nY - 1, j);
    const double r2 = __dadd_rn(sq_rn(x), sq_rn(y));
    const double r = __dsqrt_rn(r2);
    double ua;
    if (__dadd_rn(__ddiv_rn(sq_rn(x), sq_rn(a.Rx)), __ddiv_rn(sq_rn(y), sq_rn(a.Ry))) > 1.0) {
      ua = a.hydro ? fabs(an_ur_hydro(a, r)) : an_u_elast_abs(a, x, y);
    } else if (__dadd_rn(__ddiv_rn(sq_rn(x), sq_rn(a.rx)), __ddiv_rn(sq_rn(y), sq_rn(a.ry))) > 1.0) {
      ua = fabs(an_ur_hydro(a, r));
    } else {
      ua = 0.0;
    }
    uan[q] = ua;
    double err = 0.0;
    const double un = unu[q];
    if (r2 > sq_rn(a.Rmin) && r2 < sq_rn(a.Rmax) && fabs(un) > a.eps) {
      err = fabs((ua - un) / ua);
      st[0] = fmax(st[0], err);
      st[1] += err;
      st[2] += 1.0;
      if (fabs(err) > 0.5) err = -0.5;
    }
    eu[q] = err;
    if (i < nX - 1 && j < nY - 1) {
      const long c = j * (nX - 1) + i;
      const double xs = __dadd_rn(x, __dmul_rn(0.5, g.dX)), ys = __dadd_rn(y, __dmul_rn(0.5, g.dY));
      const double rs2 = __dadd_rn(sq_rn(xs), sq_rn(ys));
      const double rs = __dsqrt_rn(rs2);
      double J1 = 0.0, J2 = 0.0;
      if (__dadd_rn(__ddiv_rn(sq_rn(xs), sq_rn(a.Rx)), __ddiv_rn(sq_rn(ys), sq_rn(a.Ry))) > 1.0) {
        if (a.hydro) {
          const double relR = a.rad / rs;
          const double Srr = -a.deltaP + relR * relR * a.Y * exp(a.deltaP / a.Y - 1);
          const double Sff = -a.deltaP - relR * relR * a.Y * exp(a.deltaP / a.Y - 1);
          J1 = 0.5 * (Srr + Sff);
          J2 = 0.5 * ((Srr - Sff) * (Srr - Sff));
        } else {
          an_j_elast(a, xs, ys, &J1, &J2);
        }
      } else if (__dadd_rn(__ddiv_rn(sq_rn(xs), sq_rn(a.rx)), __ddiv_rn(sq_rn(ys), sq_rn(a.ry))) > 1.0) {
        const double Srr = -2.0 * a.xi * a.Y * log(rs / a.rad);
        const double Sff = -2.0 * a.xi * a.Y * (1.0 + log(rs / a.rad));
        J1 = 0.5 * (Srr + Sff);
        J2 = 0.5 * ((Srr - Sff) * (Srr - Sff));
      }
      j1an[c] = J1;
      j2an[c] = J2;
      double e1 = 0.0, e2 = 0.0;
      if (rs2 > sq_rn(a.Rmin) && rs2 < sq_rn(a.Rmax)) {
        if (fabs(j1nu[c]) > a.eps) {
          e1 = fabs((J1 - j1nu[c]) / J1);
          st[3] = fmax(st[3], e1);
          st[4] += e1;
          if (fabs(e1) > 0.5) e1 = -0.5;
        }
        if (fabs(j2nu[c]) > a.eps) {
          e2 = fabs((J2 - j2nu[c]) / J2);
          st[5] = fmax(st[5], e2);
          st[6] += e2;
          if (fabs(e2) > 0.5) e2 = -0.5;
        }
        st[7] += 1.0;
      }
      ej1[c] = e1;
      ej2[c] = e2;
    }
  }
  // block reduction: max for 0, 3, 5; sums for the rest
  __shared__ double red[8][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    double v = st[k];
    const bool mx = (k == 0 || k == 3 || k == 5);
    for (int o = 16; o > 0; o >>= 1) {
      const double u = __shfl_down_sync(0xffffffffu, v, o);
      v = mx ? fmax(v, u) : v + u;
    }
    if (lane == 0) red[k][w] = v;
  }
  __syncthreads();
  if (threadIdx.x < 8) {
    const int k = threadIdx.x;
    const bool mx = (k == 0 || k == 3 || k == 5);
    double v = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) v = mx ? fmax(v, red[k][q]) : v + red[k][q];
    stats[(size_t)blockIdx.x * 8 + k] = v;
  }
}

}  // namespace ep2d
