// ep2d_stencil.cuh -- the per-cell arithmetic of one pseudo-time iteration, shared by
// every form of the fused iteration kernel (tile and stream, single RVE and batched).
//
// Each formula is written with explicit IEEE operations (__dadd_rn, __dmul_rn,
// __fma_rn, ...), which the compiler neither contracts nor reorders.  Every kernel
// that calls these functions therefore rounds every cell identically, whatever the
// surrounding code, the tile or segment shape, or the batch the RVE runs in; results
// of the kernel forms are equal bit for bit.  The operations follow the reference's
// expressions (EffPlast2D.cu:37-177) with four rewrites that change rounding only:
// divisions by dX, dY, 3 and rho are multiplications by host-computed reciprocals, the
// yield test compares J2^2 with coh^2, the return factor coh / J2 is coh * rsqrt(J2^2)
// (CUDA's double rsqrt, within 1 ulp; the factor within 2 ulp of the quotient), and
// the marked products and sums are fused.
#pragma once

#include "ep2d_types.hpp"

namespace ep2d {

// ComputeStress at a node (EffPlast2D.cu:43-60): P = -K div U, tau = 2G (eps - div/3).
// dux = Ux(i+1, j) - Ux(i, j), duy = Uy(i, j+1) - Uy(i, j).
__device__ __forceinline__ void node_trial(double dux, double duy, double K, double G2, double rdX, double rdY,
                                           double third, double& p, double& xx, double& yy) {
  const double exx = __dmul_rn(dux, rdX);
  const double eyy = __dmul_rn(duy, rdY);
  const double divU = __dadd_rn(exx, eyy);
  p = __dmul_rn(-K, divU);
  xx = __dmul_rn(G2, __fma_rn(-divU, third, exx));
  yy = __dmul_rn(G2, __fma_rn(-divU, third, eyy));
}

// The four node shear moduli around a corner, summed in the reference's order
// (EffPlast2D.cu:62-69) and scaled by 1/4 (exact).
__device__ __forceinline__ double corner_g4(int m00, int m10, int m01, int m11, double G0, double Gp) {
  const double s = __dadd_rn(__dadd_rn(__dadd_rn((m00 & M_MAT) ? Gp : G0, (m10 & M_MAT) ? Gp : G0),
                                       (m01 & M_MAT) ? Gp : G0),
                             (m11 & M_MAT) ? Gp : G0);
  return __dmul_rn(0.25, s);
}

// ComputeStress at a corner (EffPlast2D.cu:62-74): tauXY = G (dUx/dy + dUy/dx), with
// dxy = Ux(i+1, j+1) - Ux(i+1, j), dyx = Uy(i+1, j+1) - Uy(i, j+1).
__device__ __forceinline__ double corner_trial(double g4, double dxy, double dyx, double rdX, double rdY) {
  return __dmul_rn(g4, __fma_rn(dxy, rdY, __dmul_rn(dyx, rdX)));
}

// J2^2 at a node from the node deviators and tauXY averaged onto the node (:100-135).
__device__ __forceinline__ double node_j2sq(double xx, double yy, double tav) {
  return __fma_rn(xx, xx, __fma_rn(yy, yy, __dmul_rn(2.0, __dmul_rn(tav, tav))));
}

// J2^2 at a corner from the sums of the four node deviators around it (:137-145).
__device__ __forceinline__ double corner_j2sq(double sx, double sy, double t) {
  return __fma_rn(__dmul_rn(0.0625, sx), sx, __fma_rn(__dmul_rn(0.0625, sy), sy, __dmul_rn(2.0, __dmul_rn(t, t))));
}

// Radial return factor (ComputePlasticity, :147-177): coh / J2 where J2 > coh, else 1.
__device__ __forceinline__ double return_factor(double j2sq, double coh, double coh2) {
  return (j2sq > coh2) ? __dmul_rn(coh, rsqrt(j2sq)) : 1.0;
}

// corner_g4 for the 16 combinations of the four nodes' material bits, bit b of `bits`
// being node b in the order m00, m10, m01, m11; equal to corner_g4 bit for bit.
__device__ __forceinline__ double corner_g4_of_bits(int bits, double G0, double Gp) {
  return corner_g4(bits & 1, (bits >> 1) & 1, (bits >> 2) & 1, (bits >> 3) & 1, G0, Gp);
}

// ComputeDisp (:3-35): damped momentum update of one face velocity,
// v (1 - dt damp) + dt/rho (dA rA + dB rB).
__device__ __forceinline__ double face_velocity(double v, double c, double dtr, double dA, double rA, double dB,
                                                double rB) {
  return __fma_rn(v, c, __dmul_rn(dtr, __fma_rn(dA, rA, __dmul_rn(dB, rB))));
}

// Stress differences of a face: ((-p + p_n) + t) - t_n, in the reference's order.
__device__ __forceinline__ double face_diff(double p, double p_n, double t, double t_n) {
  return __dsub_rn(__dadd_rn(__dsub_rn(p_n, p), t), t_n);
}

// U += V dt
__device__ __forceinline__ double advance(double u, double v, double dT) { return __fma_rn(v, dT, u); }

}  // namespace ep2d
