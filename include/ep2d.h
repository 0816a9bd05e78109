/*
 * ep2d.h -- C ABI of the B200-native EffPlast2D solver (libep2d.so).
 *
 * The reference (beacon1143/EffPlast2D) has no FFI: its boundary is the C++ class
 * `EffPlast2D` (EffPlast2D.h:53-65) driven by `main.cu` and by the MATLAB script
 * eff_props_2D.m through a process boundary.  Every entry point below replaces one
 * piece of that class; the reference function it stands for is cited beside it.
 *
 * Conventions
 *  - plain C types only: pointers, sizes, doubles; no CUDA or torch types;
 *  - every function returns an int status (EP2D_OK == 0); nothing calls exit();
 *    ep2d_last_error() returns a thread-local message for the last failure;
 *  - fields cross the boundary in the reference's own layout: row-major, x (i)
 *    fastest, unpadded, FP64 (EffPlast2D.cu:785-799), whatever the device layout;
 *  - a handle owns one CUDA stream and its device buffers; handles are not
 *    thread-safe, distinct handles may be used from distinct threads;
 *  - a missed convergence is reported in the records (converged == 0), as the
 *    reference's warning (EffPlast2D.cu:423-426) -- it is not an error status.
 */
#ifndef EP2D_H
#define EP2D_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EP2D_NPARS 11   /* NPARS, EffPlast2D.h:21-23 */
#define EP2D_MAX_NL 3   /* ComputeEffModuli supports NL <= 3, EffPlast2D.cu:182-184 */
#define EP2D_MAX_STEPS 64  /* load steps a handle keeps records for: NL >= 4 is the damping
                              mode (ComputeEffDamping, EffPlast2D.cu:230-310) */

/* status codes */
enum {
  EP2D_OK = 0,
  EP2D_ERR_ARG = 1,      /* invalid argument (sizes, NL, null pointers) */
  EP2D_ERR_CUDA = 2,     /* a CUDA runtime call failed (reference: gpuErrchk, EffPlast2D.h:41-49) */
  EP2D_ERR_IO = 3,       /* cannot open/read pa.dat (reference: ReadParams, EffPlast2D.cu:700-707) */
  EP2D_ERR_STATE = 4,    /* call out of order (e.g. increment step before the preload) */
  EP2D_ERR_NOMEM = 5,    /* device allocation failed or admission budget exceeded */
  EP2D_ERR_RANGE = 6,    /* a value left the representable range of the chosen precision */
  EP2D_ERR_NODEV = 7     /* no CUDA device, or the library was built without the kernels */
};

/* arithmetic of the pseudo-transient stencil */
enum {
  EP2D_FP64 = 0,         /* plain path: every field and every operation in FP64 */
  EP2D_MIXED = 1,        /* velocities stored in FP32 (half their HBM traffic); displacements,
                            stencil arithmetic, residual, averages and moduli in FP64 */
  EP2D_F32_BULK = 2      /* FP32 stencil bulk: each time step starts in FP32 -- arithmetic,
                            velocities and the displacement perturbation u' = U - Ua about the
                            affine preload field Ua (three FP64 strains) -- and iterates there
                            while its checkpoint residual keeps falling by at least 1/0.7 per
                            interval; the state then goes back to FP64 displacements (EP2D_MIXED)
                            for the final decades.  Only FP64 checkpoints decide convergence;
                            averages, increments and moduli stay FP64.  Single-RVE handles only. */
};

/* form of the fused iteration kernel (both compute the same iteration, operation for
 * operation; they differ in how threads map onto the grid) */
enum {
  EP2D_KERNEL_AUTO = 0,   /* the library's choice (the stream form, segments of 4 to 64
                             rows by grid size; the tile form for grids too small to occupy
                             the GPU even with 4-row segments, the resident form for small
                             elastic ones; batches: timed) */
  EP2D_KERNEL_TILE = 1,   /* one CTA per 32-column x `rows`-row tile, stencil halos in
                             shared memory; rows 8, 16 or 32 */
  EP2D_KERNEL_STREAM = 2, /* one warp per 28-column strip segment of `rows` rows, marching
                             up its rows with a register window; neighbours by warp
                             shuffles; rows 4 to 1024 */
  EP2D_KERNEL_RESIDENT = 3 /* the tile form's CTAs kept resident for all the iterations
                             between two checkpoints: one cooperative launch, a grid-wide
                             barrier (bounded waits) after each iteration; rows 8, 16 or
                             32.  Single-RVE handles only (batches refuse it) */
};

/* pa.dat layout (get_sigma_2D.m:32, read at EffPlast2D.cu:700-707, used at :1563-1573) */
enum {
  EP2D_PA_DX = 0, EP2D_PA_DY = 1, EP2D_PA_DT = 2, EP2D_PA_K0 = 3, EP2D_PA_G0 = 4,
  EP2D_PA_RHO0 = 5, EP2D_PA_DAMPX = 6, EP2D_PA_DAMPY = 7, EP2D_PA_COH = 8,
  EP2D_PA_RAD = 9, EP2D_PA_NPORES = 10
};

/* field identifiers; sizes follow the reference arrays (EffPlast2D.cu:1577-1604) */
enum {
  EP2D_FIELD_P = 0,      /* nx   x ny     */
  EP2D_FIELD_TAUXX = 1,  /* nx   x ny     */
  EP2D_FIELD_TAUYY = 2,  /* nx   x ny     */
  EP2D_FIELD_TAUXY = 3,  /* nx-1 x ny-1   */
  EP2D_FIELD_TAUXYAV = 4,/* nx   x ny     */
  EP2D_FIELD_J2 = 5,     /* nx   x ny     */
  EP2D_FIELD_J2XY = 6,   /* nx-1 x ny-1   */
  EP2D_FIELD_UX = 7,     /* nx+1 x ny     */
  EP2D_FIELD_UY = 8,     /* nx   x ny+1   */
  EP2D_FIELD_VX = 9,     /* nx+1 x ny     */
  EP2D_FIELD_VY = 10,    /* nx   x ny+1   */
  EP2D_FIELD_K = 11,     /* nx   x ny     (materials, SetMaterials EffPlast2D.cu:708-728) */
  EP2D_FIELD_G = 12,     /* nx   x ny     */
  EP2D_NFIELDS = 13
};

/* Solver configuration: the reference's compile-time macros (EffPlast2D.h:17-39),
 * its launch geometry (EffPlast2D.cu:1544-1552) and pa.dat, as run-time values. */
typedef struct ep2d_params {
  int32_t nx, ny;          /* grid; the reference uses nX = nY = 32*NGRID */
  double pa[EP2D_NPARS];   /* dX,dY,dt,K0,G0,rho0,dampX,dampY,coh,rad,N */
  int32_t nl;              /* NL: 1 elastic, 2 + bulk increment, 3 + shear increment;
                              4..EP2D_MAX_STEPS: damping mode, NL-1 sinusoidal increments */
  int32_t check_every;     /* output_step (10'000, EffPlast2D.cu:1608) */
  int64_t niter;           /* NITER */
  double eiter;            /* EITER */
  int32_t precision;       /* EP2D_FP64, EP2D_MIXED or EP2D_F32_BULK */
  int32_t device;          /* DEVICE_IDX */
  int32_t kernel;          /* EP2D_KERNEL_*; 0 = library's choice (no reference counterpart) */
  int32_t rows;            /* rows per tile / strip segment; 0 = library's choice */
} ep2d_params;

/* One time step of one load step: the per-step quantities the reference keeps in
 * its member arrays (EffPlast2D.h:108-117) and prints (EffPlast2D.cu:311-698). */
typedef struct ep2d_step_record {
  int32_t step;            /* load step: 0 preload, 1 spherical increment, 2 deviatoric */
  int32_t time_step;       /* it, 0-based */
  int64_t iterations;      /* iterations run (iter + 1 at the break, EffPlast2D.cu:419) */
  int32_t converged;       /* 1 if error < EITER at a checkpoint */
  int32_t n_checks;        /* number of checkpoints evaluated */
  double error;            /* error at the last checkpoint (EffPlast2D.cu:411-412) */
  double macro_strain[3];  /* epsilon[step][it] == curEffStrain (EffPlast2D.cu:355-358) */
  double sigma[4];         /* sigma[step][it]    (EffPlast2D.cu:456-494) */
  double sigma_per[4];     /* sigmaPer[step][it] (EffPlast2D.cu:469-499) */
  double eps_per[3];       /* epsilonPer[step][it] (EffPlast2D.cu:480-503) */
  double delta_p;          /* getDeltaP_honest   (EffPlast2D.cu:825-853) */
  double delta_p_per;      /* getDeltaP_periodic (EffPlast2D.cu:854-882) */
  double tau_infty;        /* getTauInfty_honest (EffPlast2D.cu:925-942) */
  double hole_area_pi;     /* HoleAreaPi         (EffPlast2D.cu:549-607) */
  double internal_hole_area_pi;
  double phi0, phi, phi_per;         /* EffPlast2D.cu:610-616 */
  double dphi, dphi_per;             /* dPhi[step][it], dPhiPer[step][it] (:619-620) */
  /* analytic (Yarushina) values of this step, EffPlast2D.cu:643-696; NaN when the
   * reference does not compute them for this (NL, step) */
  double kphi_exact_elast, kd_exact_elast;
  double kphi_exact_plast, kd_exact_plast;
  double kphi_exact_plast_per, kd_exact_plast_per;
  double g_exact_elast, g_exact_plast, g_exact_plast_per;
} ep2d_step_record;

typedef struct ep2d_moduli { double kphi, kd, g; } ep2d_moduli;  /* EffModuli, EffPlast2D.h:120-134 */

/* Outcome of ComputeEffModuli (EffPlast2D.cu:179-229). */
typedef struct ep2d_result {
  ep2d_moduli an, an_per, num, num_per;   /* eff_moduli_an, _an_per, _num, _num_per */
  int32_t nl;
  int32_t n_time_steps;
  int64_t total_iterations;               /* over all load and time steps */
  int32_t all_converged;
  int32_t reserved;
} ep2d_result;

typedef struct ep2d_handle ep2d_handle;

/* ---- batches and serving (no counterpart in the reference, which solves one RVE per
 * process; each RVE below is what one run of the reference's binary computes) ------- */

/* One homogenisation request: the inputs of one reference run (pa.dat, NGRID, NL and
 * the CLI's load arguments, main.cu:12-14). */
typedef struct ep2d_rve_spec {
  int32_t nx, ny;
  double pa[EP2D_NPARS];
  int32_t nl;
  int32_t n_time_steps;
  double init_load_value;
  double load_type[3];
} ep2d_rve_spec;

/* Settings shared by every RVE of a batch. */
typedef struct ep2d_batch_config {
  int64_t niter;          /* NITER (a multiple of check_every) */
  double eiter;           /* EITER */
  int32_t check_every;    /* output_step */
  int32_t precision;      /* EP2D_FP64 or EP2D_MIXED (FP32 velocity storage) */
  int32_t device;
  int32_t rows;           /* rows per tile (tile form: 8, 16, 32) or strip segment (stream
                             form: 4..1024); 0 = pick form and rows by timing the first
                             launches of the batch */
  int32_t graph_len;      /* iterations per captured CUDA graph (even; 0 = 64) */
  int32_t kernel;         /* EP2D_KERNEL_*; with rows != 0, AUTO means the stream form */
} ep2d_batch_config;

typedef struct ep2d_batch_stats {
  double kernel_ms;       /* device time of the iteration launches (CUDA events) */
  double wall_ms;
  int64_t launches;       /* batched iteration launches */
  int64_t all_launches;   /* every kernel launched, post-processing included */
  int64_t cell_updates;   /* sum over RVEs of nx*ny per iteration */
  int32_t rows;           /* rows per tile / strip segment used */
  int32_t blocks;         /* persistent grid size (CTAs) */
  int32_t kernel;         /* EP2D_KERNEL_TILE or EP2D_KERNEL_STREAM: the form used */
  int32_t n_tuned;        /* candidates timed by the latest autotuning run */
  double tune_us[7];      /* measured us per launch in the latest autotuning run: tile form
                             rows 8, 16, 32, stream form rows 8, 16, 32, 64 (0 if untimed) */
  int32_t n_tunes;        /* autotuning runs: one when the batch starts, and one whenever
                             the set of active RVEs has changed at a checkpoint */
  int32_t solo_intervals; /* RVE checkpoint intervals run through the single-RVE path (its
                             own kernel shape, overlapped launches, its own graphs): RVEs
                             that fill the GPU alone, and a lone active RVE of any size */
} ep2d_batch_stats;

/* ---- library ---------------------------------------------------------------- */
const char* ep2d_version(void);
const char* ep2d_last_error(void);
/* number of CUDA devices visible (0 without a GPU); never fails */
int ep2d_device_count(void);

/* ---- parameters ------------------------------------------------------------- */
/* ReadParams (EffPlast2D.cu:700-707): read NPARS little-endian doubles from `path`. */
int ep2d_read_pa(const char* path, double pa_out[EP2D_NPARS]);
/* The pa.dat derivation of get_sigma_2D.m:3-32 (Lx, Ly, nx, ny, K0, G0, rho0, CFL, Y,
 * porosity, nPores -> pa), so that callers without MATLAB produce the same file. */
int ep2d_make_pa(double lx, double ly, int32_t nx, int32_t ny, double k0, double g0,
                 double rho0, double cfl, double yield, double porosity, double n_pores,
                 double pa_out[EP2D_NPARS]);
/* width/height of a field for an nx x ny grid */
int ep2d_field_dims(int32_t nx, int32_t ny, int32_t field, int32_t* width, int32_t* height);

/* ---- single RVE --------------------------------------------------------------- */
/* EffPlast2D::EffPlast2D (EffPlast2D.cu:1541-1612): allocate device state, build the
 * pore/material mask on the device (SetMaterials :708-769, kernel mask :77-97),
 * zero all fields (SetMatrixZero :785-794; P0 == 0, SetInitPressure :770-783). */
int ep2d_create(const ep2d_params* params, ep2d_handle** out);
/* EffPlast2D::~EffPlast2D (EffPlast2D.cu:1613-1658) */
int ep2d_destroy(ep2d_handle* h);
/* Return a handle to the state of a freshly constructed object (EffPlast2D.cu:1585-1604:
 * every field zero, no records) without reallocating.  The reference object keeps its
 * velocities across ComputeEffModuli calls; a new object starts from rest, as this does. */
int ep2d_reset(ep2d_handle* h);

/* Exactly n pseudo-time iterations of the reference's kernel sequence
 * ComputeStress -> [ComputeJ2 -> ComputePlasticity if nl > 1] -> ComputeDisp
 * (EffPlast2D.cu:389-399), with no convergence check.  Stress-type fields
 * (P, tau*, J2*) hold the last iteration's values afterwards.  Returns when the
 * iterations have completed; their device time is added to ep2d_get_stats' kernel_ms. */
int ep2d_iterate(ep2d_handle* h, int64_t n_iter);

/* SaveMatrix's device->host copy (EffPlast2D.cu:795-799) / the H2D copies of
 * EffPlast2D.cu:375,381.  Buffers are width*height doubles (ep2d_field_dims). */
int ep2d_get_field(ep2d_handle* h, int32_t field, double* host_out);
int ep2d_set_field(ep2d_handle* h, int32_t field, const double* host_in);

/* ComputeEffParams (EffPlast2D.cu:311-698): one load step of n_time_steps time steps
 * (affine preload, iterate to EITER with checks every check_every iterations,
 * averaging, boundary P/tau, hole area, dPhi, analytic moduli).  `out` receives
 * n_time_steps records (may be NULL). */
int ep2d_solve_step(ep2d_handle* h, int32_t step, double load_step_value,
                    const double load_type[3], int32_t n_time_steps, ep2d_step_record* out);
/* the record of (step, time_step) kept by the handle */
int ep2d_get_record(ep2d_handle* h, int32_t step, int32_t time_step, ep2d_step_record* out);
/* errors evaluated at the checkpoints of (step, time_step), the values the reference
 * prints as "Iteration k: Error is e" (EffPlast2D.cu:415-416) */
int ep2d_get_check_errors(ep2d_handle* h, int32_t step, int32_t time_step,
                          double* errors_out, int32_t max_n, int32_t* n_out);

/* ComputeEffModuli (EffPlast2D.cu:179-229) without the printing and file output:
 * step 0 preload, then the spherical (NL >= 2) and deviatoric (NL == 3) increments
 * of incPercent = 0.005 (EffPlast2D.h:105), then calc* (EffPlast2D.cu:1412-1539). */
int ep2d_compute_eff_moduli(ep2d_handle* h, double init_load_value, const double load_type[3],
                            int32_t n_time_steps, ep2d_result* out);

/* ComputeEffDamping (EffPlast2D.cu:230-310) without the printing: the handle's nl must be
 * >= 4 (EP2D_ERR_ARG otherwise, as the reference throws).  Step 0 preloads
 * init_load_value along load_type over n_time_steps; steps i = 1 .. nl-1 apply one
 * time step each of load_value * (sin(i 2 pi' / (nl-1)) - sin((i-1) 2 pi' / (nl-1)))
 * along load_type, pi' = 3.1415926 as the reference writes it.  The strain and stress
 * tensors the reference prints are the records (ep2d_get_record): epsilon, epsilonPer,
 * sigma, sigmaPer of (0, n_time_steps-1) and of (i, 0).  *total_iterations (may be
 * NULL): iterations over all steps. */
int ep2d_compute_eff_damping(ep2d_handle* h, double init_load_value, const double load_type[3],
                             int32_t n_time_steps, double load_value, int64_t* total_iterations);

/* SaveAnStatic2D's numerical fields (EffPlast2D.cu:1098-1134): |u| at nodes (nx*ny),
 * J1 and J2 at corners ((nx-1)*(ny-1)), from the state after the last load step with
 * displacements zeroed inside the pores (EffPlast2D.cu:514-547). */
int ep2d_static_fields(ep2d_handle* h, double* unu_abs, double* j1nu, double* j2nu);

/* SaveAnStatic2D's analytic part (EffPlast2D.cu:1060-1292): the Yarushina (2010)
 * displacement magnitude at nodes (nx*ny) and stress invariants J1, J2 at corners
 * ((nx-1)*(ny-1)) for the far-field pressure delta_p and shear tau_infty, the relative
 * error maps against the current numerical fields (cut to -0.5 above 0.5, as the
 * reference does), and stats = {Uabs max, avg, J1 max, avg, J2 max, avg}.  The
 * reference computes these only for one pore (nPores == 1); the load type of the last
 * ep2d_compute_eff_moduli call selects the hydrostatic branch. */
int ep2d_analytic_fields(ep2d_handle* h, double delta_p, double tau_infty, double* uan_abs,
                         double* error_uabs, double* j1an, double* j2an, double* error_j1,
                         double* error_j2, double stats[6]);

/* Plastic-zone tracking as the reference's CPU solver does it (get_sigma_2D.m:126-138):
 * on = 1 clears the zone and, from then on, every iteration marks each node and corner
 * whose trial J2 exceeds coh (Plast(iPlast) = 1, PlastXY(iPlastXY) = 1); the marks
 * accumulate over iterations, time steps and load steps until tracking is turned on
 * again (cleared) or off (kept).  While tracking, the handle launches the stream form of
 * the iteration kernel (tracking instantiation; results unchanged, both forms round
 * alike) and the FP32 phase of EP2D_F32_BULK marks nothing.  ep2d_polar_fields uses the
 * accumulated zone once tracking has been turned on.  No counterpart in the reference's
 * CUDA path. */
int ep2d_track_plastic_zone(ep2d_handle* h, int32_t on);

/* The plastic zone and the stresses in polar coordinates about the grid centre (the pore
 * of a single-pore RVE) that the reference's CPU solver computes after its solve
 * (get_sigma_2D.m:170-194), from the state the last iteration recorded.  Every output is
 * nx*ny, node (i, j) at j*nx + i:
 *   plastic: Plast + PlastXY of get_sigma_2D.m:170-173: 1 if the node yielded plus the
 *            number of yielded corners among the four around it.  With tracking on
 *            (ep2d_track_plastic_zone) "yielded" means at any tracked iteration, as the
 *            CPU solver counts it; without, in the final state (recorded J2 at coh,
 *            recorded trial J2XY > coh);
 *   snu_rr, snu_ff: tauXX - P, tauYY - P, tauXYav rotated to the polar axes, where
 *            plastic > 0;
 *   san_rr, san_ff: -P0 + sign(load_value) 2 coh (log(sqrt(r)) [+ 1]) / sqrt(2), P0 = 0,
 *            where plastic > 0;
 * all zero elsewhere and inside the pore (r < rad). */
int ep2d_polar_fields(ep2d_handle* h, double load_value, double* snu_rr, double* snu_ff, double* san_rr,
                      double* san_ff, uint8_t* plastic);

/* ---- batch ---------------------------------------------------------------------- */
/* Solve n RVEs together: every RVE runs ComputeEffModuli's chain (EffPlast2D.cu:179-229)
 * with the reference's convergence test and checkpoint cadence; all active RVEs advance
 * in lockstep through one persistent batched kernel per iteration, captured in a CUDA
 * graph; finished RVEs retire at their checkpoint.  results[k] is what the reference
 * binary would compute for specs[k].  Fails with EP2D_ERR_NOMEM if the RVEs do not fit
 * on the device at once (the server admits them progressively instead). */
int ep2d_batch_solve(const ep2d_batch_config* cfg, const ep2d_rve_spec* specs, int32_t n,
                     ep2d_result* results, ep2d_batch_stats* stats);
/* device bytes one RVE of this spec holds while it is being solved */
int64_t ep2d_rve_footprint(const ep2d_rve_spec* spec, int32_t precision);

/* ---- server (continuous batching) ------------------------------------------------- */
typedef struct ep2d_server ep2d_server;
/* A worker thread owns one batch engine on `cfg->device`.  Requests are admitted at
 * checkpoint boundaries while the summed footprint of the active RVEs stays within
 * mem_budget_bytes and their number within max_active; admitted RVEs stay resident
 * until they converge.  If a checkpoint interval fails (a CUDA error), every active and
 * queued request finishes with that status and the server accepts no more requests
 * (EP2D_ERR_STATE); destroy it and create a new one. */
int ep2d_server_create(const ep2d_batch_config* cfg, int64_t mem_budget_bytes, int32_t max_active,
                       ep2d_server** out);
int ep2d_server_submit(ep2d_server* s, const ep2d_rve_spec* spec, uint64_t* ticket_out);
/* Wait up to timeout_ms (negative: forever) for the request to finish.  *done = 1 and
 * *result / *latency_s (submit to completion, host clock) / *queue_s are filled when it
 * has, and the return value is the request's own status.  That wait releases the result:
 * a later wait on the same ticket, like one on a ticket this server never issued,
 * returns EP2D_ERR_ARG at once. */
int ep2d_server_wait(ep2d_server* s, uint64_t ticket, int32_t timeout_ms, int32_t* done,
                     ep2d_result* result, double* latency_s, double* queue_s);
/* requests submitted, admitted, finished; bytes of device memory in use */
int ep2d_server_stats(ep2d_server* s, int64_t* submitted, int64_t* admitted, int64_t* finished,
                      int64_t* bytes_in_use, ep2d_batch_stats* engine);
int ep2d_server_destroy(ep2d_server* s);

/* ---- scratch-free averaging ----------------------------------------------------- */
/* No counterpart in the reference (its averaging runs on the host after copying eight
 * fields back, EffPlast2D.cu:430-503).  For callers that cannot call cudaMalloc --
 * code whose device memory belongs to a host framework's allocator or to a fixed pool,
 * which a library must not grow, fragment or synchronise with cudaMalloc/cudaFree --
 * this computes the RVE averages of fields the caller already holds in device memory
 * and allocates nothing:
 *   inputs, in the reference's layout, on the current device: p, tau_xx, tau_yy
 *   (nx*ny), tau_xy ((nx-1)*(ny-1)), ux ((nx+1)*ny), uy (nx*(ny+1)); pa: pa.dat values;
 *   out_dev[11] (caller's device memory) = sigma[0..3], sigma_per[0..3], eps_per[0..2],
 *   divided as the reference divides them (the values ep2d_step_record holds).
 * The reduction's partial sums use a fixed device array of 2048 x 11 doubles (176 KiB,
 * held by every GPU that loads the library until the process exits), so ny may be at
 * most 8194; a larger ny returns EP2D_ERR_ARG without touching the GPU, as do dX or dY
 * not positive and N outside [1, 64].  A CUDA error left pending by earlier work is
 * reported (EP2D_ERR_CUDA) and nothing is launched.  The first call on a device looks
 * the array's address up (cudaGetSymbolAddress) with that device current, and again
 * after a cudaDeviceReset (the lookup is kept per device and context): make that first
 * call before any stream capture.  All calls share the array,
 * so calls that overlap on the GPU race: issue them on one stream.  The work is queued
 * on `stream` (a cudaStream_t; NULL: the default stream) and the call returns without
 * waiting for it. */
int ep2d_average_fields_noalloc(int32_t nx, int32_t ny, const double pa[EP2D_NPARS], const double* p,
                                const double* tau_xx, const double* tau_yy, const double* tau_xy,
                                const double* ux, const double* uy, double* out_dev, void* stream);

/* sizeof() of ep2d_params, ep2d_step_record, ep2d_moduli, ep2d_result, ep2d_rve_spec,
 * ep2d_batch_config and ep2d_batch_stats into out[0..n); returns the number of structs
 * (7).  Lets a binding check its layout. */
int ep2d_abi_sizes(int64_t* out, int32_t n);

/* Counters of this handle since creation: device time of the iteration loops measured
 * with CUDA events on the handle's stream (ms), launches of the fused iteration kernel,
 * cell updates (nx*ny per iteration), and all kernel launches (iteration kernel plus
 * preload, reductions and gathers).  Any pointer may be NULL. */
int ep2d_get_stats(ep2d_handle* h, double* kernel_ms, int64_t* iter_launches, int64_t* cell_updates,
                   int64_t* all_launches);
/* n_iter pseudo-time iterations of the FP32 form of EP2D_F32_BULK from the current state
 * (handles created with EP2D_F32_BULK only, else EP2D_ERR_STATE): the FP64 displacements
 * go to the FP32 perturbation about the affine field of the current macro strain, the
 * iterations run, and the state comes back to FP64.  No convergence check; the device time
 * is added to ep2d_get_stats' kernel_ms.  No counterpart in the reference (all FP64). */
int ep2d_iterate_f32(ep2d_handle* h, int64_t n_iter);
/* Iterations this handle has run in the FP32 form of EP2D_F32_BULK (0 for the other
 * precisions).  No counterpart in the reference (all FP64). */
int ep2d_get_f32_iterations(ep2d_handle* h, int64_t* f32_iterations);
/* The iteration kernel this handle launches: EP2D_KERNEL_TILE, EP2D_KERNEL_STREAM or
 * EP2D_KERNEL_RESIDENT and its rows per tile / strip segment (the parameters' choice, or
 * the library's).  No counterpart in the reference. */
int ep2d_get_kernel_shape(ep2d_handle* h, int32_t* kernel, int32_t* rows);
/* The resident form's grid barrier on its own, for checking its failure path without a
 * fault: one cooperative launch of `blocks` CTAs (all resident at once) on `device`
 * meets at the barrier `rounds` times (at most 1,000,000), except that `missing` of the
 * CTAs never arrive.
 * With missing == 0 every CTA passes every round (*passed = blocks, *flag = 0); with
 * missing > 0 the others' waits run out after timeout_ns (at most 10 s) and they return
 * with the error flag set (*passed = 0, *flag = 1), the context still usable.  A resident
 * launch whose barrier fails the same way makes the handle's next checkpoint (or the end
 * of ep2d_iterate / the time step) return EP2D_ERR_CUDA.  No counterpart in the
 * reference. */
int ep2d_check_grid_barrier(int32_t device, int32_t blocks, int32_t missing, int32_t rounds, int64_t timeout_ns,
                            int32_t* passed, int32_t* flag);

#ifdef __cplusplus
}
#endif
#endif /* EP2D_H */
