// ep2d_stencil.cuh -- the per-cell arithmetic of one pseudo-time iteration, shared by
// every form of the fused iteration kernel (tile and stream, single RVE and batched).
//
// Each formula is written with explicit IEEE operations (__dadd_rn, __dmul_rn,
// __fma_rn, ...), which the compiler neither contracts nor reorders.  Every kernel
// that calls these functions therefore rounds every cell identically, whatever the
// surrounding code, the tile or segment shape, or the batch the RVE runs in; results
// of the kernel forms are equal bit for bit.  The operations follow the reference's
// expressions (EffPlast2D.cu:37-177) with rewrites that change rounding only: divisions
// by dX, dY, 3 and rho are multiplications by host-computed reciprocals (dt/rho folded
// into the face factors), the yield test compares J2^2 with coh^2 (16 J2^2 with 16 coh^2
// at corners), the return factor coh / J2 is coh * rsqrt(J2^2) (CUDA's double rsqrt,
// within 1 ulp; the factor within 2 ulp of the quotient), the four-term sums of the
// tauXY average and of the corner deviators add two pair sums (pair_sum4) instead of left
// to right, the averages' 1/4 is folded into the J2 formulas, and the marked products and
// sums are fused.
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

// J2^2 at a node from h = the four-corner tauXY sum (the average is h / 4):
// xx^2 + yy^2 + 2 (h/4)^2 = xx^2 + yy^2 + 0.125 h^2, two operations fewer than forming
// the average first.
__device__ __forceinline__ double node_j2sq_h(double xx, double yy, double h) {
  return __fma_rn(xx, xx, __fma_rn(yy, yy, __dmul_rn(__dmul_rn(0.125, h), h)));
}

// 16 J2^2 at a corner from the sums sx, sy of the four node deviators around it
// (:137-145): sx^2 + sy^2 + 32 t^2 = 16 ((sx/4)^2 + (sy/4)^2 + 2 t^2).  Its
// yield test compares with 16 coh^2 and its factor is 4 coh rsqrt(16 J2^2) = coh / J2,
// so the 1/16 is never applied.
__device__ __forceinline__ double corner_j2sq16(double sx, double sy, double t) {
  return __fma_rn(sx, sx, __fma_rn(sy, sy, __dmul_rn(__dmul_rn(32.0, t), t)));
}

// Radial return factor (ComputePlasticity, :147-177): coh / J2 where J2 > coh, else 1.
__device__ __forceinline__ double return_factor(double j2sq, double coh, double coh2) {
  return (j2sq > coh2) ? __dmul_rn(coh, rsqrt(j2sq)) : 1.0;
}

// ComputeDisp (:3-35): damped momentum update of one face velocity with the factors
// sA = dt/rho rA and sB = dt/rho rB formed on the host: v (1 - dt damp) + dA sA + dB sB.
__device__ __forceinline__ double face_velocity_s(double v, double c, double dA, double sA, double dB, double sB) {
  return __fma_rn(v, c, __fma_rn(dA, sA, __dmul_rn(dB, sB)));
}

// Normal-stress difference across a face, (t - p) - (t_n - p_n): the total stresses
// tau - P of the two nodes, each formed once per node (the stream form forms it before
// its one shuffle) and then subtracted.
__device__ __forceinline__ double stress_diff(double p, double p_n, double t, double t_n) {
  return __dsub_rn(__dsub_rn(t, p), __dsub_rn(t_n, p_n));
}

// U += V dt
__device__ __forceinline__ double advance(double u, double v, double dT) { return __fma_rn(v, dT, u); }

// ---- FP32 bulk ------------------------------------------------------------------
// The same formulas in FP32 (__f*_rn: neither contracted nor reordered), for the FP32
// stencil bulk.  Its displacements are the perturbation u' = U - Ua of the affine field
// Ua = (Exx x + Exy y, Eyy y) the preloads have applied (EffPlast2D.cu:349-381), held as
// three FP64 scalars: the strain of Ua is exactly (Exx, Eyy, Exy), so the node and
// corner strains are those constants plus the differences of u', which keeps the FP32
// differences small (u' ~ 1e-2 of U near the pores) instead of cancelling two FP32
// values of U itself.

__device__ __forceinline__ void node_trial(float dux, float duy, float exx0, float eyy0, float K, float G2, float rdX,
                                           float rdY, float third, float& p, float& xx, float& yy) {
  const float exx = __fadd_rn(__fmul_rn(dux, rdX), exx0);
  const float eyy = __fadd_rn(__fmul_rn(duy, rdY), eyy0);
  const float divU = __fadd_rn(exx, eyy);
  p = __fmul_rn(-K, divU);
  xx = __fmul_rn(G2, __fmaf_rn(-divU, third, exx));
  yy = __fmul_rn(G2, __fmaf_rn(-divU, third, eyy));
}
__device__ __forceinline__ float corner_trial(float g4, float dxy, float dyx, float exy0, float rdX, float rdY) {
  return __fmul_rn(g4, __fadd_rn(__fmaf_rn(dxy, rdY, __fmul_rn(dyx, rdX)), exy0));
}
__device__ __forceinline__ float node_j2sq(float xx, float yy, float tav) {
  return __fmaf_rn(xx, xx, __fmaf_rn(yy, yy, __fmul_rn(2.0f, __fmul_rn(tav, tav))));
}
__device__ __forceinline__ float node_j2sq_h(float xx, float yy, float h) {
  return __fmaf_rn(xx, xx, __fmaf_rn(yy, yy, __fmul_rn(__fmul_rn(0.125f, h), h)));
}
__device__ __forceinline__ float corner_j2sq16(float sx, float sy, float t) {
  return __fmaf_rn(sx, sx, __fmaf_rn(sy, sy, __fmul_rn(__fmul_rn(32.0f, t), t)));
}
__device__ __forceinline__ float face_velocity_s(float v, float c, float dA, float sA, float dB, float sB) {
  return __fmaf_rn(v, c, __fmaf_rn(dA, sA, __fmul_rn(dB, sB)));
}
__device__ __forceinline__ float return_factor(float j2sq, float coh, float coh2) {
  return (j2sq > coh2) ? __fmul_rn(coh, rsqrtf(j2sq)) : 1.0f;
}
__device__ __forceinline__ float stress_diff(float p, float p_n, float t, float t_n) {
  return __fsub_rn(__fsub_rn(t, p), __fsub_rn(t_n, p_n));
}
__device__ __forceinline__ float advance(float u, float v, float dT) { return __fmaf_rn(v, dT, u); }

// The sum of a 2x2 block as two pair sums, (a + b) + (c + d): the tauXY average onto a
// node (pairs = the block's rows) and the deviator sums onto a corner (pairs = its
// columns).  Every kernel form adds in this order, so a form may carry a pair sum from
// one row or lane to the next and still round like the others.
__device__ __forceinline__ double pair_sum4(double a, double b, double c, double d) {
  return __dadd_rn(__dadd_rn(a, b), __dadd_rn(c, d));
}
__device__ __forceinline__ float pair_sum4(float a, float b, float c, float d) {
  return __fadd_rn(__fadd_rn(a, b), __fadd_rn(c, d));
}

// explicit IEEE add, subtract, multiply of either precision
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double sqrt_rn(double a) { return __dsqrt_rn(a); }
__device__ __forceinline__ float sqrt_rn(float a) { return __fsqrt_rn(a); }

}  // namespace ep2d
