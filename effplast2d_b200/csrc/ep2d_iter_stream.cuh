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
constexpr int STREAM_DEPTH = 4;                 // rows of loads in flight per warp
// rows k-2 .. k+DEPTH live in the ring at step k: the faces of row k-2 read U and V of
// rows k-2 and k-1 from it, and the refill goes to the slot of row k-3
constexpr int STREAM_SLOTS = STREAM_DEPTH + 3;

// One row of a warp's 32 columns, as the ring holds it; m: the aligned 32-bit word of
// the byte mask that contains the lane's node.  TU: displacement type (double; float
// for the FP32 bulk, whose displacements are perturbations of the affine field), TV:
// velocity type.
template <typename TU, typename TV>
struct StreamRow {
  TU ux[32];
  TU uy[32];
  TV vx[32];
  TV vy[32];
  uint32_t m[32];
};

// (K, 2G) of a node in the arithmetic type
template <typename T>
struct KG2 {
  T k, g2;
};

// Shared memory of one warp: its ring and two tables that fold the pore masks into the
// material constants, so that the interior step needs no select for them:
//   g4z[c]: corner_g4 of a corner by c = (mask(i,j) & (M_MAT | M_CORNER | M_MAT_R)) |
//           ((mask(i,j+1) & (M_MAT | M_MAT_R)) << 1), and 0 where the corner is in a pore
//           (bit 2, M_CORNER) -- the corner trial is then 0 * (...) = 0, as the
//           reference's tauXY = 0 (EffPlast2D.cu:89-92), up to the sign of the zero;
//   kgz[m]: (K, 2G) of a node by m = mask & (M_MAT | M_NODE), (0, 0) in a pore (M_NODE):
//           P and the deviators are then 0 (EffPlast2D.cu:79-85), up to the zero's sign.
// A zero's sign changes no sum, difference or product the iteration forms from it.
template <typename TU, typename TV>
struct StreamWarpSmem {
  StreamRow<TU, TV> ring[STREAM_SLOTS];
  TU g4z[32];
  KG2<TU> kgz[4];
};

// c = corner table index of the corner (i, j) from the mask bytes of nodes (i, j) and
// (i, j + 1); the four material bits of g4z's index: bit 0 node (i, j), bit 3 (i+1, j),
// bit 1 (i, j+1), bit 4 (i+1, j+1); bit 2 the corner's pore bit
__device__ __forceinline__ int corner_index(int m_j, int m_j1) {
  return (m_j & (M_MAT | M_CORNER | M_MAT_R)) | ((m_j1 & (M_MAT | M_MAT_R)) << 1);
}
__device__ __forceinline__ double g4z_entry(int c, double G0, double Gp) {
  return (c & 4) ? 0.0 : corner_g4(c & 1, (c >> 3) & 1, (c >> 1) & 1, (c >> 4) & 1, G0, Gp);
}

template <typename TU, typename TV>
constexpr size_t stream_smem_bytes() {
  return sizeof(StreamWarpSmem<TU, TV>) * STREAM_WARPS;
}

template <typename T>
__device__ __forceinline__ T shfl_idx(T v, int src) { return __shfl_sync(0xffffffffu, v, src); }
template <typename T>
__device__ __forceinline__ T shfl_dn(T v) { return __shfl_down_sync(0xffffffffu, v, 1); }
template <typename T>
__device__ __forceinline__ T shfl_up1(T v) { return __shfl_up_sync(0xffffffffu, v, 1); }
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

// The displacement arrays of a form: FP64 U, or the FP32 bulk's perturbations u'.
template <typename TU>
__device__ __forceinline__ TU* u_field(const Fields& f, bool y, int buf);
template <>
__device__ __forceinline__ double* u_field<double>(const Fields& f, bool y, int buf) {
  return y ? f.uy[buf] : f.ux[buf];
}
template <>
__device__ __forceinline__ float* u_field<float>(const Fields& f, bool y, int buf) {
  return y ? f.uy32[buf] : f.ux32[buf];
}

// One strip segment.  TU = double: the FP64 stencil (velocities stored as TV); TU =
// float: the FP32 bulk (arithmetic, u' and V in FP32; a RECORD launch then only folds
// max|V|, the FP64 convergence check reading it in double).
template <bool PLASTIC, bool RECORD, bool INTERIOR, typename TU, typename TV, bool TRACK = false>
__device__ __forceinline__ void stream_task(const Geo& g, const Fields& f, const int src, const int strip,
                                            const int jA, const int jB, StreamWarpSmem<TU, TV>& sm, double& vmx,
                                            double& vmy) {
  using T = TU;  // arithmetic type
  constexpr bool F32 = std::is_same<TU, float>::value;
  static_assert(!F32 || std::is_same<TV, float>::value, "the FP32 bulk stores velocities in FP32");
  constexpr bool REC_STRESS = RECORD && !F32;  // the FP32 bulk records no stresses
  const int lane = threadIdx.x & 31;
  const int nx = g.nx, ny = g.ny;
  const int pitch = g.pitch;  // pitch * (ny + 1) < 2^31 (checked on the host)
  const int i = STREAM_COLS * strip - 2 + lane;
  const bool own = INTERIOR ? (lane >= 2 && lane < 2 + STREAM_COLS) : (lane >= 2 && lane < 2 + STREAM_COLS && i < nx);
  const TU* __restrict__ ux = u_field<TU>(f, false, src);
  const TU* __restrict__ uy = u_field<TU>(f, true, src);
  TU* __restrict__ uxo = u_field<TU>(f, false, src ^ 1);
  TU* __restrict__ uyo = u_field<TU>(f, true, src ^ 1);
  TV* __restrict__ fvx = static_cast<TV*>(f.vx);
  TV* __restrict__ fvy = static_cast<TV*>(f.vy);
  const uint8_t* __restrict__ mask = f.mask;
  // TRACK: the yield bits go to the same bytes; other lanes only read the low bits,
  // which the stores leave as they are
  uint8_t* mask_w = const_cast<uint8_t*>(f.mask);

  const bool coln = INTERIOR || (i >= 0 && i < nx);   // column of nodes, Uy, Vy
  const int mshift = 8 * (i & 3);                     // pitch % 32 == 0: byte i & 3 of the word
  const int ln1 = min(lane + 1, 31);                  // the lane of column i + 1 (lane 31: unused)

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
  const TU* __restrict__ u_src = half ? uy : ux;
  const TV* __restrict__ v_src = half ? fvy : fvx;
  // live == false (rows past the segment's last, k_last): the copies only zero-fill
  auto issue = [&](int k, int slot, bool live) {
    StreamRow<TU, TV>& row = sm.ring[slot];
    const bool ok = live && pair_in && (INTERIOR || (k >= 0 && k < rows_of));
    const int q = ok ? k * pitch + pc : 0;
    cp_async_pair_zfill<TU>((half ? row.uy : row.ux) + 2 * (lane & 15), u_src + q, ok);
    cp_async_pair_zfill<TV>((half ? row.vy : row.vx) + 2 * (lane & 15), v_src + q, ok);
    const bool rm = live && (INTERIOR || (coln && k >= 0 && k < ny));  // nodes
    cp_async_zfill<4>(&row.m[lane], mask + (rm ? ((k * pitch + i) & ~3) : 0), rm);
  };
  const T rdX = (T)g.rdX, rdY = (T)g.rdY, third = (T)(1.0 / 3.0);
  const T coh = (T)g.coh, coh2 = (T)g.coh2, coh4 = (T)g.coh4, coh2x16 = (T)g.coh2x16;
  const T dT = (T)g.dT, cX = (T)g.cX, cY = (T)g.cY, dtrX = (T)g.dtrX, dtrY = (T)g.dtrY;
  const T exx0 = (T)g.exx0, eyy0 = (T)g.eyy0, exy0 = (T)g.exy0;  // FP32 bulk only
  __syncwarp();  // the previous segment of this warp has stopped reading the tables
  sm.g4z[lane] = (T)g4z_entry(lane, g.G0, g.Gp);
  if (lane < 4) {
    KG2<T> kg{(T)0, (T)0};
    if (!(lane & M_NODE)) kg = KG2<T>{(T)((lane & M_MAT) ? g.Kp : g.K0), (T)__dmul_rn(2.0, (lane & M_MAT) ? g.Gp : g.G0)};
    sm.kgz[lane] = kg;
  }
  __syncwarp();

  // Launched as a programmatic dependent of the previous iteration (single-RVE form),
  // this kernel may start before that one has finished; nothing above touches global
  // memory.  Wait for the previous grid to complete (its stores visible) before the
  // first load; without such a launch (the batched form) the wait returns at once.
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  int slot_wr = 0;
#pragma unroll 1
  for (int d = 0; d < STREAM_DEPTH; d++) {
    issue(k_first + d, slot_wr, k_first + d <= k_last);
    cp_async_commit();  // empty groups keep the count uniform
    slot_wr++;
  }

  // registers at step r (suffix _r: column i+1, _l: column i-1): U rows r (0) and r+1
  // (p), masks rows r and r+1; U and V of row r-1 and r are read back from the ring
  T ux0 = 0, uxp = 0, uy0 = 0, uyp = 0;
  T ux0_r = 0, uxp_r = 0;  // Ux(i+1, r), Ux(i+1, r+1)
  int mkm = 0, mk0 = 0, mkp = 0;  // mask bytes of node i in rows r-1, r and r+1
  // trial stresses: nodes rows r-1 (a) and r (b); corners rows r-3..r (c0..c3; the
  // interior needs rows r-1 and r only, with hs1 = the pair sum c(i-1) + c(i) of row r-2)
  T xa = 0, ya = 0, pb = 0, xb = 0, yb = 0, pa_ = 0;
  T c0 = 0, c1 = 0, c2 = 0, c3 = 0;
  T c2_l = 0;  // corner trial row r-1 of column i-1; next step: row r-2
  T hs1 = 0;
  // returned stresses: nodes rows r-2 (q) and r-1 (w); corners rows r-2 (cq), r-1 (cw)
  T pw = 0, xw = 0, yw = 0, cq = 0, cw = 0;
  // total normal stresses tau - P of row r-1 (sxw, syw) and syy of row r-2 (syq)
  T sxw = 0, syw = 0, syq = 0;
  T cw_l = 0;  // returned corner row r-1 of column i-1; next step: row r-2

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
    const StreamRow<TU, TV>& row = sm.ring[s_k];
    ux0 = uxp; uxp = row.ux[lane];
    ux0_r = uxp_r; uxp_r = row.ux[ln1];
    uy0 = uyp; uyp = row.uy[lane];
    mkm = mk0; mk0 = mkp; mkp = (int)((row.m[lane] >> mshift) & 0xffu);
    if (k + STREAM_DEPTH <= k_last) issue(k + STREAM_DEPTH, slot_wr, true);  // the slot of row k-3
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
    const T uyp_r = sm.ring[s_k].uy[ln1];
    T pn, xn, yn, cn;
    {
      const KG2<T> kg = sm.kgz[mk0 & (M_MAT | M_NODE)];  // (0, 0) in a pore
      const T g4 = sm.g4z[corner_index(mk0, mkp)];      // 0 in a pore
      T p_, x_, y_, c_;
      if constexpr (F32) {
        node_trial(sub_rn(ux0_r, ux0), sub_rn(uyp, uy0), exx0, eyy0, kg.k, kg.g2, rdX, rdY, third, p_, x_, y_);
        c_ = corner_trial(g4, sub_rn(uxp_r, ux0_r), sub_rn(uyp_r, uyp), exy0, rdX, rdY);
      } else {
        node_trial(sub_rn(ux0_r, ux0), sub_rn(uyp, uy0), kg.k, kg.g2, rdX, rdY, third, p_, x_, y_);
        c_ = corner_trial(g4, sub_rn(uxp_r, ux0_r), sub_rn(uyp_r, uyp), rdX, rdY);
      }
      if (INTERIOR) {
        pn = p_; xn = x_; yn = y_; cn = c_;
      } else {  // nodes and corners outside the grid: 0
        const bool node_ok = coln && r >= 0 && r < ny;
        pn = node_ok ? p_ : (T)0;
        xn = node_ok ? x_ : (T)0;
        yn = node_ok ? y_ : (T)0;
        const bool corner_ok = i >= 0 && i < nx - 1 && r >= 0 && r < ny - 1;
        cn = corner_ok ? c_ : (T)0;
      }
    }
    pa_ = pb; xa = xb; ya = yb;
    pb = pn; xb = xn; yb = yn;
    c0 = c1; c1 = c2; c2 = c3; c3 = cn;
    c2_l = shfl_up1(c2);
    // interior: pair sum of row r-1's corners (i-1, i); the previous step's is hs1
    const T hs0 = hs1;
    if (INTERIOR && PLASTIC) hs1 = add_rn(c2_l, c2);

    // ---- return of row j = r - 1
    const int j = r - 1;
    T tav_o = 0, j2_o = 0, j2xy_o = 0;
    T cq_l = 0;
    bool yld_n = false, yld_c = false;  // TRACK: node / corner (i, j) yields at this iteration
    if constexpr (STAGE >= 1) {
      T xr = xa, yr = ya, cr = c2;
      if (PLASTIC) {
        // node: tauXY averaged from the clamped 2x2 corner block (EffPlast2D.cu:109-135)
        T hsum;  // the four-corner sum; tauXY averaged onto the node is hsum / 4
        if (INTERIOR) {  // the block below-left: corners (i-1..i, j-1..j), rows j-1 and j
          hsum = add_rn(hs0, hs1);
        } else {
          const int a = min(max(i - 1, 0), nx - 3) - i;  // -2, -1 or 0 inside the grid
          const int bsel = min(max(j - 1, 0), ny - 3) - j;
          const T cr0 = (bsel == 0) ? c2 : (bsel == -1 ? c1 : c0);  // row j + bsel
          const T cr1 = (bsel == 0) ? c3 : (bsel == -1 ? c2 : c1);  // row j + bsel + 1
          const int sa = min(max(lane + a, 0), 31), sb = min(max(lane + a + 1, 0), 31);
          hsum = pair_sum4(shfl_idx(cr0, sa), shfl_idx(cr0, sb), shfl_idx(cr1, sa), shfl_idx(cr1, sb));
        }
        const T nJ2sq = node_j2sq_h(xa, ya, hsum);
        const bool node_in = INTERIOR || (coln && j >= 0 && j < ny);
        const T fn = node_in ? return_factor(nJ2sq, coh, coh2) : (T)1;
        // corner: node deviators (i..i+1, j..j+1) = rows a (j) and b (j+1), summed as
        // column pairs, column i+1's from the next lane
        const T vx_ = add_rn(xa, xb), vy_ = add_rn(ya, yb);
        const T sx = add_rn(vx_, shfl_dn(vx_));
        const T sy = add_rn(vy_, shfl_dn(vy_));
        const T cJ2sq16 = corner_j2sq16(sx, sy, c2);  // 16 J2^2
        const bool corner_in = INTERIOR || (i >= 0 && i < nx - 1 && j >= 0 && j < ny - 1);
        const T fc = corner_in ? return_factor(cJ2sq16, coh4, coh2x16) : (T)1;
        if (TRACK) {  // J2 > coh from the trial stresses (get_sigma_2D.m:126-138)
          yld_n = node_in && nJ2sq > coh2;
          yld_c = corner_in && cJ2sq16 > coh2x16;
        }
        if (REC_STRESS) {
          tav_o = node_in ? mul_rn(mul_rn((T)0.25, hsum), fn) : (T)0;
          j2_o = !node_in ? (T)0
                          : (fn != (T)1) ? sqrt_rn(node_j2sq(mul_rn(xa, fn), mul_rn(ya, fn), tav_o))
                                         : sqrt_rn(nJ2sq);
          j2xy_o = corner_in ? mul_rn((T)0.25, sqrt_rn(cJ2sq16)) : (T)0;
        }
        xr = mul_rn(xa, fn);
        yr = mul_rn(ya, fn);
        cr = mul_rn(c2, fc);
      }
      cq_l = cw_l;
      syq = syw; cq = cw;
      pw = pa_; xw = xr; yw = yr; cw = cr;
      sxw = sub_rn(xw, pw);
      syw = sub_rn(yw, pw);
      cw_l = shfl_up1(cw);
    }

    // ---- faces of row j (owned rows [jA, jB)); U and V of row j from the ring.  A face
    // the reference leaves alone gets its old velocity back, unchanged.
    if constexpr (STAGE == 2) {
      const T sxw_l = shfl_up1(sxw);
      const StreamRow<TU, TV>& rj = sm.ring[s_k2];
      const T uxm = rj.ux[lane], uym = rj.uy[lane];
      const T vxm = (T)rj.vx[lane], vym = (T)rj.vy[lane];
      const TV vxs = (TV)face_velocity_s(vxm, cX, sub_rn(sxw, sxw_l), dtrX, sub_rn(cw_l, cq_l), dtrY);
      const TV vys = (TV)face_velocity_s(vym, cY, sub_rn(syw, syq), dtrY, sub_rn(cq, cq_l), dtrX);
      // the displacement moves by the stored velocity
      const T vx = (INTERIOR || (i > 0 && j > 0 && j < ny - 1)) ? (T)vxs : vxm;
      const T vy = (INTERIOR || (i > 0 && i < nx - 1 && j > 0)) ? (T)vys : vym;
      const T uxn = advance(uxm, vx, dT), uyn = advance(uym, vy, dT);
      if (own) {
        const int q = j * pitch + i;
        if (TRACK) {  // mkm: the mask byte of node (i, j); only this lane writes it
          const int bits = (yld_n ? M_YN : 0) | (yld_c ? M_YC : 0);
          if (bits & ~mkm) mask_w[q] = (uint8_t)(mkm | bits);
        }
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
            const StreamRow<TU, TV>& rj1 = sm.ring[s_k1];
            uyo[ny * pitch + i] = rj1.uy[lane];
            if (RECORD) vmy = fmax(vmy, fabs((double)rj1.vy[lane]));
          }
        }
        if (RECORD) {
          vmx = fmax(vmx, fabs((double)vx));
          vmy = fmax(vmy, fabs((double)vy));
        }
        if (REC_STRESS) {
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

template <bool PLASTIC, bool RECORD, typename TU, typename TV, bool TRACK = false>
__device__ __forceinline__ void stream_segment(const Geo& g, const Fields& f, int src, int strip, int seg, int seg_h,
                                               StreamWarpSmem<TU, TV>& sm, double& vmx, double& vmy) {
  const int jA = seg * seg_h;
  const int jB = min(jA + seg_h, g.ny);
  if (stream_interior(g.nx, g.ny, strip, jA, jB))
    stream_task<PLASTIC, RECORD, true, TU, TV, TRACK>(g, f, src, strip, jA, jB, sm, vmx, vmy);
  else
    stream_task<PLASTIC, RECORD, false, TU, TV, TRACK>(g, f, src, strip, jA, jB, sm, vmx, vmy);
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
template <bool PLASTIC, bool RECORD, typename TU, typename TV, bool TRACK = false>
__global__ void __launch_bounds__(32 * STREAM_WARPS) k_iter_stream(Geo g, Fields f, int src, int nstrips, int nsegs,
                                                                   int seg_h) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  StreamWarpSmem<TU, TV>& sm = reinterpret_cast<StreamWarpSmem<TU, TV>*>(smem_raw)[threadIdx.x >> 5];
  // let the next iteration's grid be scheduled now: it waits for this grid's completion
  // before reading anything (griddepcontrol.wait in stream_task)
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
  const int task = blockIdx.x * STREAM_WARPS + (threadIdx.x >> 5);
  if (task >= nstrips * nsegs) return;  // whole warp
  double vmx = 0.0, vmy = 0.0;
  stream_segment<PLASTIC, RECORD, TU, TV, TRACK>(g, f, src, task % nstrips, task / nstrips, seg_h, sm, vmx, vmy);
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
  StreamWarpSmem<double, TV>& sm = reinterpret_cast<StreamWarpSmem<double, TV>*>(smem_raw)[threadIdx.x >> 5];
  const int n = *nunits;
  const int nw = gridDim.x * STREAM_WARPS;
  for (int t = blockIdx.x * STREAM_WARPS + (threadIdx.x >> 5); t < n; t += nw) {
    const int2 u = units[t];
    const BatchEntry& e = ents[u.x];
    const int src = e.src0 ^ parity;
    double vmx = 0.0, vmy = 0.0;
    if (e.plastic)
      stream_segment<true, RECORD, double, TV>(e.g, e.f, src, u.y & 0xffff, u.y >> 16, seg_h, sm, vmx, vmy);
    else
      stream_segment<false, RECORD, double, TV>(e.g, e.f, src, u.y & 0xffff, u.y >> 16, seg_h, sm, vmx, vmy);
    stream_fold_vmax<RECORD>(vmx, vmy, e.f.vmax);
  }
}

}  // namespace ep2d
