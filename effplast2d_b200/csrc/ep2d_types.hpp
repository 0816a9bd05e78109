// ep2d_types.hpp -- plain C++ types shared by the CUDA kernels (nvcc) and the host
// orchestration (g++), plus the kernel launch wrappers the host calls.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace ep2d {

// mask byte of node (i, j): M_MAT, M_NODE, M_CORNER as below (ep2d_device.cuh), and
// M_MAT_R = the M_MAT bit of node (i + 1, j) (0 on the last column), so that a corner's
// four material bits come from the two mask bytes of its column
// M_YN, M_YC: set by the plastic-zone tracking launches when the trial J2 of node (i, j)
// / corner (i, j) has exceeded coh at some iteration (get_sigma_2D.m's Plast, PlastXY)
enum : uint8_t { M_MAT = 1, M_NODE = 2, M_CORNER = 4, M_MAT_R = 8, M_YN = 16, M_YC = 32 };

// Per-RVE scalars, passed to kernels by value.
struct Geo {
  int nx, ny, pitch;
  double dX, dY, dT, rho, dampX, dampY, coh;
  double K0, G0, Kp, Gp;  // Kp = 0.01 * K0, Gp = 0.01 * G0 (EffPlast2D.cu:721-722)
  double rad, nPores;
  // host-computed factors of the iteration kernel: 1/dX, 1/dY, coh^2,
  // 1 - dT dampX, 1 - dT dampY, dT / rho
  double rdX, rdY, coh2, cX, cY, dtr;
  // 4 coh, 16 coh^2 (the corner return), dt/rho / dX, dt/rho / dY (the face updates)
  double coh4, coh2x16, dtrX, dtrY;
  // FP32 bulk only: strains of the affine field Ua its displacements are measured from:
  // exx0 = dUa_x/dx, eyy0 = dUa_y/dy, exy0 = dUa_x/dy + dUa_y/dx (= 2 Exy)
  double exx0, eyy0, exy0;
};

// Device pointers of one RVE.  Velocities are stored as double on the FP64 path and as
// float on the mixed path (the launch selects the type); everything else is double.
struct Fields {
  double* ux[2];
  double* uy[2];
  void* vx;
  void* vy;
  double *p, *txx, *tyy, *txy, *txyav, *j2, *j2xy;  // last recorded stress state
  const uint8_t* mask;
  unsigned long long* vmax;  // [2]: bit patterns of max|Vx|, max|Vy| (non-negative)
  // FP32 bulk only: the displacement perturbations u' = U - Ua (ping-pong), float
  float* ux32[2];
  float* uy32[2];
  // resident form: the grid barrier {64-bit arrival count, error flag, unused}, 8-byte aligned
  unsigned* gbar;
};

// One RVE of a batched launch.
struct BatchEntry {
  Geo g;
  Fields f;
  int src0;     // ping-pong buffer holding U at the start of the current graph
  int plastic;  // NL > 1
};

// Tile of the fused iteration kernel: 32 columns x TILE_Y rows; the tile height is a
// launch-time choice among TILE_Y_CHOICES (the batch autotuner picks it).
constexpr int TILE_X = 32;
constexpr int TILE_Y = 16;
constexpr int TILE_Y_CHOICES[3] = {8, 16, 32};

// The forms of the fused iteration kernel: FORM_TILE (CTA per tile, halos in shared
// memory; rows = tile height), FORM_STREAM (warp per 28-column strip segment; rows =
// segment height, SEG_MIN..SEG_MAX) and FORM_RESIDENT (the tile form's CTAs kept
// resident across the iterations between two checkpoints, one cooperative launch;
// rows = tile height; single launches, the recording ones among them, are tile-form
// launches).
enum IterForm { FORM_TILE = 0, FORM_STREAM = 1, FORM_RESIDENT = 2 };
constexpr int STREAM_COLS = 28;  // columns a warp of the stream form owns (32 lanes, 2-lane halos)
constexpr int SEG_MIN = 4, SEG_MAX = 1024;
constexpr int SEG_DEFAULT = 64;
constexpr int SEG_CHOICES[4] = {8, 16, 32, 64};  // the batch autotuner's stream-form candidates
struct IterShape {
  int form = FORM_STREAM;
  int rows = SEG_DEFAULT;
};
// true if `s` names a launchable kernel
inline bool shape_valid(const IterShape& s) {
  if (s.form == FORM_TILE || s.form == FORM_RESIDENT) return s.rows == 8 || s.rows == 16 || s.rows == 32;
  return s.form == FORM_STREAM && s.rows >= SEG_MIN && s.rows <= SEG_MAX;
}
// work units of one RVE: tiles or strip segments, as (x, y) counts
void shape_units(const IterShape& s, int nx, int ny, int* ux, int* uy);

// Number of sums produced by the averaging and boundary reductions.
constexpr int NAVG = 11;

// Launch wrappers (ep2d_kernels.cu).  All are asynchronous on `stream`.
cudaError_t prepare_kernels();  // per-device function attributes
cudaError_t launch_mask(const Geo& g, uint8_t* mask, cudaStream_t stream);
cudaError_t launch_preload(const Geo& g, const Fields& f, int src, double dUxdx, double dUydy, double dUxdy,
                           int zero_first, cudaStream_t stream);
// one iteration of one RVE; mixed: velocities stored as float; track: also mark the
// nodes and corners that yield (M_YN, M_YC; stream form and plastic iterations only)
cudaError_t launch_iter(const Geo& g, const Fields& f, int src, bool plastic, bool record, bool mixed,
                        const IterShape& shape, cudaStream_t stream, bool track = false);
// n_iter plain iterations of one RVE from buffer src in one cooperative launch (the
// resident form; tile height `rows`); each barrier wait gives up after timeout_ns,
// which leaves the error flag f.gbar[2] set (zero when the RVE is created; a set flag
// makes later launches return at once)
cudaError_t launch_iter_resident(const Geo& g, const Fields& f, int src, bool plastic, bool mixed, int rows,
                                 int64_t n_iter, unsigned long long timeout_ns, cudaStream_t stream);
constexpr unsigned long long RESIDENT_TIMEOUT_NS = 2000000000ull;  // 2 s per barrier wait
// the grid barrier alone on `blocks` co-resident CTAs, `missing` of which never arrive;
// out[0] = CTAs that passed all `rounds`; gbar (4 words) zeroed first
cudaError_t launch_grid_barrier_check(unsigned* gbar, int blocks, int missing, int rounds,
                                      unsigned long long timeout_ns, unsigned* out, cudaStream_t stream);
// clear the M_YN / M_YC bits of every node
cudaError_t launch_clear_track(const Geo& g, uint8_t* mask, cudaStream_t stream);
// one iteration of the FP32 bulk (stream form, segments of seg_h rows): u' and V in
// f.ux32/uy32 and f.vx/vy (float), affine strains in g.exx0/eyy0/exy0; a recording launch
// folds max|V| only
cudaError_t launch_iter_f32(const Geo& g, const Fields& f, int src, bool plastic, bool record, int seg_h,
                            cudaStream_t stream);
// the FP64 state U (buffer src) to the FP32 bulk's u' (both buffers), and back (u'
// buffer src to both U buffers), with the affine strains of g
cudaError_t launch_to_f32(const Geo& g, const Fields& f, int src, cudaStream_t stream);
cudaError_t launch_from_f32(const Geo& g, const Fields& f, int src, cudaStream_t stream);
// one iteration of every RVE in the work list {rve, x | y << 16} (tiles or strip
// segments of `shape`), by a persistent grid of `blocks` CTAs
cudaError_t launch_iter_batch(const BatchEntry* ents, const int2* units, const int* nunits, int parity, bool record,
                              bool mixed, const IterShape& shape, int blocks, cudaStream_t stream);
// CTAs of the batched kernel of `shape` resident per SM
int iter_blocks_per_sm(bool record, bool mixed, const IterShape& shape);
// averaging: writes NAVG sums to `sums` (device); `partials` holds avg_partials_len(g) doubles
size_t avg_partials_len(const Geo& g);
cudaError_t launch_average(const Geo& g, const Fields& f, int src, double nu0, int perOffsetX, int perOffsetY,
                           double* partials, double* sums, cudaStream_t stream);
cudaError_t launch_boundary(const Geo& g, const Fields& f, double* sums, cudaStream_t stream);
cudaError_t launch_gather(const Geo& g, const Fields& f, int src, const unsigned long long* idx, int n,
                          double* out, cudaStream_t stream);
cudaError_t launch_static_fields(const Geo& g, const Fields& f, int src, double* unu, double* j1, double* j2,
                                 cudaStream_t stream);
// accumulated: the zone from the M_YN / M_YC bits, else from the recorded J2, J2XY
cudaError_t launch_polar_fields(const Geo& g, const Fields& f, double sgn, double* snrr, double* snff, double* sarr,
                                double* saff, uint8_t* plast, bool accumulated, cudaStream_t stream);

// Scalars of the analytic static solution (SaveAnStatic2D, EffPlast2D.cu:1062-1078).
struct AnParams {
  double deltaP, tauInfty, Y, rad, G0, K0;
  double xi, kappa, c0, rx, ry, Rx, Ry, Rmin, Rmax, eps;
  int hydro;  // isHydroStatic (EffPlast2D.cu:1062-1064)
};

constexpr int ANALYTIC_BLOCKS = 592;  // 4 x 148 SMs; stats[ANALYTIC_BLOCKS][8]
cudaError_t launch_analytic(const Geo& g, const AnParams& a, const double* unu, const double* j1nu, const double* j2nu,
                            double* uan, double* eu, double* j1an, double* j2an, double* ej1, double* ej2,
                            double* stats, cudaStream_t stream);

}  // namespace ep2d
