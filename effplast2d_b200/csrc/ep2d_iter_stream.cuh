// ep2d_iter_stream.cuh -- the fused iteration kernel, column-streaming form.
//
// Same iteration as ep2d_iter_f64.cuh (ComputeStress -> ComputeJ2 -> ComputePlasticity
// -> ComputeDisp, EffPlast2D.cu:3-177), same per-cell formulas (ep2d_stencil.cuh), a
// different mapping.  A warp owns 28 columns (lanes 2..29; lanes 0, 1, 30, 31 are
// halo) and a segment of rows; each lane keeps its column's values of the last few rows
// in registers and the warp marches up its segment one row per step.  At step r a lane
//   takes   Ux, Uy, Vx, Vy and the mask of row r+1 from its shared-memory ring,
//   forms   the trial stresses of row r (node and corner),
//   returns row r-1 (node: tauXY averaged onto the node from the clamped 2x2 corner
//           block; corner: tauXX, tauYY averaged onto the corner),
//   updates the faces of row r-1 (damped momentum, U += V dt).
// Rows reach the ring by cp.async (U and V as 16-byte column pairs), STREAM_DEPTH rows
// ahead of use, so each warp keeps that many rows of loads in flight without holding
// them in registers: the march is a
// chain of dependent steps, and without the ring a warp would wait one memory latency
// per row.  Neighbouring columns come from warp shuffles; a value a step needs from a
// neighbour that the previous step already fetched (the same quantity one row lower)
// is carried in a register instead of fetched again.  There is no block-wide barrier;
// each lane reads only the ring entries it wrote.
//
// Segments whose 32 columns and rows jA-2 .. jB+1 lie inside the grid away from its
// edges run the INTERIOR instantiation: no bounds tests, and the clamped 2x2 corner
// block of the node return is always the one below-left.  Segments touching an edge
// run the general one.  Both call the same formulas, so they round alike.
#pragma once

#include <type_traits>

#include "ep2d_stencil.cuh"
#include "ep2d_types.hpp"

namespace ep2d {

constexpr int STREAM_WARPS = 4;                 // warps per CTA (STREAM_COLS owned columns per warp)
constexpr int STREAM_DEPTH = 6;                 // rows of loads in flight per warp
// rows k-2 .. k+DEPTH live in the ring at step k: the faces of row k-2 read U and V of
// rows k-2 and k-1 from it, and the refill goes to the slot of row k-3
constexpr int STREAM_SLOTS = STREAM_DEPTH + 3;

// One row of a warp's 32 columns, as the ring holds it; m: the aligned 32-bit word of
// the byte mask that contains the lane's node.
template <typename TV>
struct StreamRow {
  double ux[32];
  double uy[32];
  TV vx[32];
  TV vy[32];
  uint32_t m[32];
};

// Shared memory of one warp: its ring, the 16-entry table of corner_g4 by the material
// bits of the four nodes around a corner, and (K, 2G) by the material bit of a node.
template <typename TV>
struct StreamWarpSmem {
  StreamRow<TV> ring[STREAM_SLOTS];
  double g4[16];
  double2 kg[2];
};

template <typename TV>
constexpr size_t stream_smem_bytes() {
  return sizeof(StreamWarpSmem<TV>) * STREAM_WARPS;
}

__device__ __forceinline__ double shfl_idx(double v, int src) { return __shfl_sync(0xffffffffu, v, src); }
__device__ __forceinline__ double shfl_dn(double v) { return __shfl_down_sync(0xffffffffu, v, 1); }
__device__ __forceinline__ double shfl_up1(double v) { return __shfl_up_sync(0xffffffffu, v, 1); }
__device__ __forceinline__ int shfl_dn_i(int v) { return __shfl_down_sync(0xffffffffu, v, 1); }

// cp.async of 4, 8 or 16 bytes; with ok == false nothing is read and the destination is
// zero-filled (src-size 0), `src` then only has to be a valid address.
template <int BYTES>
__device__ __forceinline__ void cp_async_zfill(void* dst, const void* src, bool ok) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(d), "l"(src), "n"(BYTES), "r"(ok ? BYTES : 0)
               : "memory");
}
// two consecutive elements of a field: 16 bytes (double) or 8 (float).  Through L1
// (.ca): neighbouring strips share their halo columns there; the L2-only form (.cg) ran
// 4 % slower at 2048^2.
template <typename T>
__device__ __forceinline__ void cp_async_pair_zfill(T* dst, const T* src, bool ok) {
  cp_async_zfill<(int)(2 * sizeof(T))>(dst, src, ok);
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// true if segment (strip, jA..jB) may run the INTERIOR instantiation: every lane's
// column in [0, nx-1] and at least one column from the right edge, rows jA-2 .. jB+1
// inside the grid with jA >= 3 and jB <= ny-2
__device__ __forceinline__ bool stream_interior(int nx, int ny, int strip, int jA, int jB) {
  return strip >= 1 && STREAM_COLS * strip + 29 <= nx - 3 && jA >= 3 && jB <= ny - 2;
}

template <bool PLASTIC, bool RECORD, bool INTERIOR, typename TV>
__device__ __forceinline__ void stream_task(const Geo& g, const Fields& f, const int src, const int strip,
                                            const int jA, const int jB, StreamWarpSmem<TV>& sm, double& vmx,
                                            double& vmy) {
  const int lane = threadIdx.x & 31;
  const int nx = g.nx, ny = g.ny;
  const int pitch = g.pitch;  // pitch * (ny + 1) < 2^31 (checked on the host)
  const int i = STREAM_COLS * strip - 2 + lane;
  const bool own = INTERIOR ? (lane >= 2 && lane < 2 + STREAM_COLS) : (lane >= 2 && lane < 2 + STREAM_COLS && i < nx);
  const double* __restrict__ ux = src ? f.ux[1] : f.ux[0];
  const double* __restrict__ uy = src ? f.uy[1] : f.uy[0];
  double* __restrict__ uxo = src ? f.ux[0] : f.ux[1];
  double* __restrict__ uyo = src ? f.uy[0] : f.uy[1];
  TV* __restrict__ fvx = static_cast<TV*>(f.vx);
  TV* __restrict__ fvy = static_cast<TV*>(f.vy);
  const uint8_t* __restrict__ mask = f.mask;

  const bool coln = INTERIOR || (i >= 0 && i < nx);   // column of nodes, Uy, Vy
  const int mshift = 8 * (i & 3);                     // pitch % 32 == 0: byte i & 3 of the word
  const int ln1 = min(lane + 1, 31);                  // the lane of column i + 1 (lane 31: unused)
  const int mshift1 = 8 * ((i + 1) & 3);

  // rows k_first .. k_last pass through the ring: U and the mask are needed up to row
  // r + 1 and V up to row r for steps r = jA - 2 .. jB.  U and V move in column pairs:
  // lanes 0..15 copy the 16 pairs of the warp's 32 columns of Ux (Vx), lanes 16..31
  // those of Uy (Vy), 16 (V as float: 8) bytes each; a pair starts on an even column at
  // a 16-byte aligned address (pitch % 32 == 0) and lies in its row as long as it starts
  // inside the pitch.  Columns past the grid read the row padding, which nothing writes
  // and which holds zeros, like the zero fill of rows and columns outside the arrays.
  const int k_first = jA - 2, k_last = jB + 1;
  const int half = lane >> 4;                                  // 0: Ux, Vx; 1: Uy, Vy
  const int pc = STREAM_COLS * strip - 2 + 2 * (lane & 15);    // first column of the pair
  const bool pair_in = INTERIOR || (pc >= 0 && pc < pitch);
  const int rows_of = half ? ny + 1 : ny;                      // Uy, Vy: rows 0 .. ny
  const double* __restrict__ u_src = half ? uy : ux;
  const TV* __restrict__ v_src = half ? fvy : fvx;
  auto issue = [&](int k, int slot) {
    StreamRow<TV>& row = sm.ring[slot];
    const bool ok = pair_in && (INTERIOR || (k >= 0 && k < rows_of));
    const int q = ok ? k * pitch + pc : 0;
    cp_async_pair_zfill<double>((half ? row.uy : row.ux) + 2 * (lane & 15), u_src + q, ok);
    cp_async_pair_zfill<TV>((half ? row.vy : row.vx) + 2 * (lane & 15), v_src + q, ok);
    const bool rm = INTERIOR || (coln && k >= 0 && k < ny);  // nodes
    cp_async_zfill<4>(&row.m[lane], mask + (rm ? ((k * pitch + i) & ~3) : 0), rm);
  };
  const double rdX = g.rdX, rdY = g.rdY, third = 1.0 / 3.0;
  const double coh = g.coh, coh2 = g.coh2;
  const double dT = g.dT, cX = g.cX, cY = g.cY, dtr = g.dtr;
  __syncwarp();  // the previous segment of this warp has stopped reading the tables
  if (lane < 16) sm.g4[lane] = corner_g4_of_bits(lane, g.G0, g.Gp);
  if (lane < 2) sm.kg[lane] = make_double2(lane ? g.Kp : g.K0, __dmul_rn(2.0, lane ? g.Gp : g.G0));
  __syncwarp();

  // Launched as a programmatic dependent of the previous iteration (single-RVE form),
  // this kernel may start before that one has finished; nothing above touches global
  // memory.  Wait for the previous grid to complete (its stores visible) before the
  // first load; without such a launch (the batched form) the wait returns at once.
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  int slot_wr = 0;
#pragma unroll 1
  for (int d = 0; d < STREAM_DEPTH; d++) {
    if (k_first + d <= k_last) issue(k_first + d, slot_wr);
    cp_async_commit();  // empty groups keep the count uniform
    slot_wr++;
  }

  // registers at step r (suffix _r: column i+1, _l: column i-1): U rows r (0) and r+1
  // (p), masks rows r and r+1; U and V of row r-1 and r are read back from the ring
  double ux0 = 0.0, uxp = 0.0, uy0 = 0.0, uyp = 0.0;
  double ux0_r = 0.0, uxp_r = 0.0;  // Ux(i+1, r), Ux(i+1, r+1)
  int mk0 = 0, mkp = 0, mk0_r = 0, mkp_r = 0;
  int g_lo = 0, g_hi = 0;  // material bits of nodes (i, i+1) in rows r and r+1
  // trial stresses: nodes rows r-1 (a) and r (b); corners rows r-3..r (c0..c3)
  double xa = 0.0, ya = 0.0, pb = 0.0, xb = 0.0, yb = 0.0, pa_ = 0.0;
  double xb_r = 0.0, yb_r = 0.0;  // node trial row r of column i+1; next step: row r-1
  double c0 = 0.0, c1 = 0.0, c2 = 0.0, c3 = 0.0;
  double c2_l = 0.0;  // corner trial row r-1 of column i-1; next step: row r-2
  // returned stresses: nodes rows r-2 (q) and r-1 (w); corners rows r-2 (cq), r-1 (cw)
  double pq = 0.0, yq = 0.0, pw = 0.0, xw = 0.0, yw = 0.0, cq = 0.0, cw = 0.0;
  double cw_l = 0.0;  // returned corner row r-1 of column i-1; next step: row r-2

  // slots of rows k, k-1, k-2
  int s_k = STREAM_SLOTS - 1, s_k1 = STREAM_SLOTS - 2, s_k2 = STREAM_SLOTS - 3;
  int k = k_first;
  // bring row k from the ring into the registers and refill the ring
  auto take_row = [&]() {
    cp_async_wait<STREAM_DEPTH - 1>();  // this lane's copies of row k have landed
    __syncwarp();                        // ... and every lane's (neighbours are read below)
    s_k2 = s_k1;
    s_k1 = s_k;
    s_k = (s_k + 1 == STREAM_SLOTS) ? 0 : s_k + 1;
    const StreamRow<TV>& row = sm.ring[s_k];
    ux0 = uxp; uxp = row.ux[lane];
    ux0_r = uxp_r; uxp_r = row.ux[ln1];
    uy0 = uyp; uyp = row.uy[lane];
    mk0 = mkp; mkp = (int)((row.m[lane] >> mshift) & 0xffu);
    mk0_r = mkp_r; mkp_r = (int)((row.m[ln1] >> mshift1) & 0xffu);
    g_lo = g_hi;
    g_hi = (mkp & M_MAT) | ((mkp_r & M_MAT) << 1);
    if (k + STREAM_DEPTH <= k_last) issue(k + STREAM_DEPTH, slot_wr);  // the slot of row k-3
    cp_async_commit();
    slot_wr = (slot_wr + 1 == STREAM_SLOTS) ? 0 : slot_wr + 1;
  };
  // Step r = k - 1 forms the trial stresses of row r, returns row r - 1 (STAGE >= 1)
  // and updates the faces of row r - 1 (STAGE 2).  The first owned face row, jA, needs
  // rows jA and jA - 1 returned, and those need the trials of rows jA - 2 .. jA: the
  // march opens with two trial-only steps (r = jA - 2, jA - 1) and one without faces
  // (r = jA), then takes one full step per owned row.
  auto step = [&](auto stage_c) {
    constexpr int STAGE = decltype(stage_c)::value;
    take_row();
    const int r = k - 1;

    // ---- trial stresses of row r.  The step body is branch-free: every lane evaluates
    // every formula (lanes a branch would mask run it in lockstep anyway) and a select
    // keeps the value or its default, so the compiler schedules whole rows as straight
    // code; only the stores are predicated.
    const double uyp_r = sm.ring[s_k].uy[ln1];
    double pn, xn, yn, cn;
    {
      const double2 kg = sm.kg[mk0 & M_MAT];
      double p_, x_, y_;
      node_trial(__dsub_rn(ux0_r, ux0), __dsub_rn(uyp, uy0), kg.x, kg.y, rdX, rdY, third, p_, x_, y_);
      const bool node_ok = (INTERIOR || (coln && r >= 0 && r < ny)) && !(mk0 & M_NODE);
      pn = node_ok ? p_ : 0.0;
      xn = node_ok ? x_ : 0.0;
      yn = node_ok ? y_ : 0.0;
      const double c_ =
          corner_trial(sm.g4[g_lo | (g_hi << 2)], __dsub_rn(uxp_r, ux0_r), __dsub_rn(uyp_r, uyp), rdX, rdY);
      const bool corner_ok = (INTERIOR || (i >= 0 && i < nx - 1 && r >= 0 && r < ny - 1)) && !(mk0 & M_CORNER);
      cn = corner_ok ? c_ : 0.0;
    }
    const double xa_r = xb_r, ya_r = yb_r;
    pa_ = pb; xa = xb; ya = yb;
    pb = pn; xb = xn; yb = yn;
    xb_r = shfl_dn(xb);
    yb_r = shfl_dn(yb);
    const double c1_l = c2_l;
    c0 = c1; c1 = c2; c2 = c3; c3 = cn;
    c2_l = shfl_up1(c2);

    // ---- return of row j = r - 1
    const int j = r - 1;
    double tav_o = 0.0, j2_o = 0.0, j2xy_o = 0.0;
    double cq_l = 0.0;
    if constexpr (STAGE >= 1) {
      double xr = xa, yr = ya, cr = c2;
      if (PLASTIC) {
        // node: tauXY averaged from the clamped 2x2 corner block (EffPlast2D.cu:109-135)
        double c00, c10, c01, c11;
        if (INTERIOR) {  // the block below-left: corners (i-1..i, j-1..j)
          c00 = c1_l; c10 = c1; c01 = c2_l; c11 = c2;
        } else {
          const int a = min(max(i - 1, 0), nx - 3) - i;  // -2, -1 or 0 inside the grid
          const int bsel = min(max(j - 1, 0), ny - 3) - j;
          const double cr0 = (bsel == 0) ? c2 : (bsel == -1 ? c1 : c0);  // row j + bsel
          const double cr1 = (bsel == 0) ? c3 : (bsel == -1 ? c2 : c1);  // row j + bsel + 1
          const int sa = min(max(lane + a, 0), 31), sb = min(max(lane + a + 1, 0), 31);
          c00 = shfl_idx(cr0, sa); c10 = shfl_idx(cr0, sb);
          c01 = shfl_idx(cr1, sa); c11 = shfl_idx(cr1, sb);
        }
        const double tav = __dmul_rn(0.25, __dadd_rn(__dadd_rn(__dadd_rn(c00, c10), c01), c11));
        const double nJ2sq = node_j2sq(xa, ya, tav);
        const bool node_in = INTERIOR || (coln && j >= 0 && j < ny);
        const double fn = node_in ? return_factor(nJ2sq, coh, coh2) : 1.0;
        // corner: node deviators (i..i+1, j..j+1) = rows a (j) and b (j+1)
        const double sx = __dadd_rn(__dadd_rn(__dadd_rn(xa, xa_r), xb), xb_r);
        const double sy = __dadd_rn(__dadd_rn(__dadd_rn(ya, ya_r), yb), yb_r);
        const double cJ2sq = corner_j2sq(sx, sy, c2);
        const bool corner_in = INTERIOR || (i >= 0 && i < nx - 1 && j >= 0 && j < ny - 1);
        const double fc = corner_in ? return_factor(cJ2sq, coh, coh2) : 1.0;
        if (RECORD) {
          tav_o = node_in ? __dmul_rn(tav, fn) : 0.0;
          j2_o = !node_in ? 0.0
                          : (fn != 1.0) ? __dsqrt_rn(node_j2sq(__dmul_rn(xa, fn), __dmul_rn(ya, fn), tav_o))
                                        : __dsqrt_rn(nJ2sq);
          j2xy_o = corner_in ? __dsqrt_rn(cJ2sq) : 0.0;
        }
        xr = __dmul_rn(xa, fn);
        yr = __dmul_rn(ya, fn);
        cr = __dmul_rn(c2, fc);
      }
      cq_l = cw_l;
      pq = pw; yq = yw; cq = cw;
      pw = pa_; xw = xr; yw = yr; cw = cr;
      cw_l = shfl_up1(cw);
    }

    // ---- faces of row j (owned rows [jA, jB)); U and V of row j from the ring.  A face
    // the reference leaves alone gets its old velocity back, unchanged.
    if constexpr (STAGE == 2) {
      const double pw_l = shfl_up1(pw), xw_l = shfl_up1(xw);
      const StreamRow<TV>& rj = sm.ring[s_k2];
      const double uxm = rj.ux[lane], uym = rj.uy[lane];
      const double vxm = (double)rj.vx[lane], vym = (double)rj.vy[lane];
      const TV vxs = (TV)face_velocity(vxm, cX, dtr, face_diff(pw, pw_l, xw, xw_l), rdX, __dsub_rn(cw_l, cq_l), rdY);
      const TV vys = (TV)face_velocity(vym, cY, dtr, face_diff(pw, pq, yw, yq), rdY, __dsub_rn(cq, cq_l), rdX);
      // the displacement moves by the stored velocity
      const double vx = (INTERIOR || (i > 0 && j > 0 && j < ny - 1)) ? (double)vxs : vxm;
      const double vy = (INTERIOR || (i > 0 && i < nx - 1 && j > 0)) ? (double)vys : vym;
      const double uxn = advance(uxm, vx, dT), uyn = advance(uym, vy, dT);
      if (own) {
        const int q = j * pitch + i;
        fvx[q] = (TV)vx;
        fvy[q] = (TV)vy;
        uxo[q] = uxn;
        uyo[q] = uyn;
        if (!INTERIOR) {
          if (i == nx - 1) {  // face column nx of Ux/Vx (lane + 1): never updated
            uxo[j * pitch + nx] = rj.ux[lane + 1];
            if (RECORD) vmx = fmax(vmx, fabs((double)rj.vx[lane + 1]));
          }
          if (j == ny - 1) {  // face row ny of Uy/Vy (row k-1 of the ring): never updated
            const StreamRow<TV>& rj1 = sm.ring[s_k1];
            uyo[ny * pitch + i] = rj1.uy[lane];
            if (RECORD) vmy = fmax(vmy, fabs((double)rj1.vy[lane]));
          }
        }
        if (RECORD) {
          vmx = fmax(vmx, fabs(vx));
          vmy = fmax(vmy, fabs(vy));
          f.p[q] = pw;
          f.txx[q] = xw;
          f.tyy[q] = yw;
          if (INTERIOR || (i < nx - 1 && j < ny - 1)) f.txy[q] = cw;
          if (PLASTIC) {
            f.txyav[q] = tav_o;
            f.j2[q] = j2_o;
            if (INTERIOR || (i < nx - 1 && j < ny - 1)) f.j2xy[q] = j2xy_o;
          }
        }
      }
    }
  };
  take_row();  // row jA - 2 only fills the registers
  k++;
  step(std::integral_constant<int, 0>{});
  k++;
  step(std::integral_constant<int, 0>{});
  k++;
  step(std::integral_constant<int, 1>{});
  k++;
#pragma unroll 2
  for (; k <= k_last; k++) step(std::integral_constant<int, 2>{});
}

template <bool PLASTIC, bool RECORD, typename TV>
__device__ __forceinline__ void stream_segment(const Geo& g, const Fields& f, int src, int strip, int seg, int seg_h,
                                               StreamWarpSmem<TV>& sm, double& vmx, double& vmy) {
  const int jA = seg * seg_h;
  const int jB = min(jA + seg_h, g.ny);
  if (stream_interior(g.nx, g.ny, strip, jA, jB))
    stream_task<PLASTIC, RECORD, true, TV>(g, f, src, strip, jA, jB, sm, vmx, vmy);
  else
    stream_task<PLASTIC, RECORD, false, TV>(g, f, src, strip, jA, jB, sm, vmx, vmy);
}

template <bool RECORD>
__device__ __forceinline__ void stream_fold_vmax(double vmx, double vmy, unsigned long long* vmax) {
  if (RECORD) {
    for (int o = 16; o > 0; o >>= 1) {
      vmx = fmax(vmx, __shfl_xor_sync(0xffffffffu, vmx, o));
      vmy = fmax(vmy, __shfl_xor_sync(0xffffffffu, vmy, o));
    }
    if ((threadIdx.x & 31) == 0) {
      atomicMax(&vmax[0], (unsigned long long)__double_as_longlong(vmx));
      atomicMax(&vmax[1], (unsigned long long)__double_as_longlong(vmy));
    }
  }
}

// One RVE: warp w of CTA b handles task b * STREAM_WARPS + w = (strip, segment).
template <bool PLASTIC, bool RECORD, typename TV>
__global__ void __launch_bounds__(32 * STREAM_WARPS) k_iter_stream(Geo g, Fields f, int src, int nstrips, int nsegs,
                                                                   int seg_h) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  StreamWarpSmem<TV>& sm = reinterpret_cast<StreamWarpSmem<TV>*>(smem_raw)[threadIdx.x >> 5];
  // let the next iteration's grid be scheduled now: it waits for this grid's completion
  // before reading anything (griddepcontrol.wait in stream_task)
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
  const int task = blockIdx.x * STREAM_WARPS + (threadIdx.x >> 5);
  if (task >= nstrips * nsegs) return;  // whole warp
  double vmx = 0.0, vmy = 0.0;
  stream_segment<PLASTIC, RECORD, TV>(g, f, src, task % nstrips, task / nstrips, seg_h, sm, vmx, vmy);
  stream_fold_vmax<RECORD>(vmx, vmy, f.vmax);
}

// Many RVEs: a persistent grid of warps walks the device-side list {rve, strip | seg << 16}
// (warps are independent, so a CTA's warps may work on different RVEs).  `parity` is the
// launch's position in the captured graph (mod 2), as for the tile form.
template <bool RECORD, typename TV>
__global__ void __launch_bounds__(32 * STREAM_WARPS) k_iter_stream_batch(const BatchEntry* __restrict__ ents,
                                                                         const int2* __restrict__ units,
                                                                         const int* __restrict__ nunits, int parity,
                                                                         int seg_h) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  StreamWarpSmem<TV>& sm = reinterpret_cast<StreamWarpSmem<TV>*>(smem_raw)[threadIdx.x >> 5];
  const int n = *nunits;
  const int nw = gridDim.x * STREAM_WARPS;
  for (int t = blockIdx.x * STREAM_WARPS + (threadIdx.x >> 5); t < n; t += nw) {
    const int2 u = units[t];
    const BatchEntry& e = ents[u.x];
    const int src = e.src0 ^ parity;
    double vmx = 0.0, vmy = 0.0;
    if (e.plastic) stream_segment<true, RECORD, TV>(e.g, e.f, src, u.y & 0xffff, u.y >> 16, seg_h, sm, vmx, vmy);
    else stream_segment<false, RECORD, TV>(e.g, e.f, src, u.y & 0xffff, u.y >> 16, seg_h, sm, vmx, vmy);
    stream_fold_vmax<RECORD>(vmx, vmy, e.f.vmax);
  }
}

}  // namespace ep2d
