// ep2d_rve.hpp -- one RVE resident on a B200: device state, the load-step chain and
// its records.  Shared by the single-RVE C ABI, the batched solver and the server.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "ep2d.h"
#include "ep2d_types.hpp"

namespace ep2d {

// thread-local last-error text (ep2d_last_error)
void set_error(const std::string& msg);
const char* last_error();
int fail(int code, const std::string& msg);

// RAII: make `dev` current, restore the previous device on scope exit.
struct DeviceScope {
  int prev = -1;
  explicit DeviceScope(int dev);
  ~DeviceScope();
};

// Reference scalars derived from pa (EffPlast2D.cu:1563-1573, :1609-1611).
struct Derived {
  double dX, dY, dT, K0, G0, E0, nu0, rad, Y, nPores, porosity, lX, lY;
};
Derived derive(const ep2d_params& p);

// Host-side pore test of SetMaterials / ComputeEffParams (EffPlast2D.cu:719-720).
bool host_in_pore(const Derived& d, long nX, long nY, double x, double y);

// One hole-edge sample of EffPlast2D.cu:552-595.
struct HoleSample {
  unsigned long long code;  // bit 62: 0 = Ux, 1 = Uy; low bits: reference flat index
  bool zeroed;              // position inside a pore: the reference zeroes it (:514-547)
};
// The 20 samples per pore, in the reference's order (left, right, bottom, top).
int hole_samples(const Derived& d, long nX, long nY, std::vector<HoleSample>* out);

// Post-processing of one time step from the device sums (EffPlast2D.cu:491-696).
// avg[NAVG]: averaging sums; bnd[NAVG]: boundary sums; samples: hole-edge values.
void finish_record(const Derived& d, long nX, long nY, int nl, int step, const double* avg, const double* bnd,
                   const std::vector<HoleSample>& hs, const double* samples, ep2d_step_record* r,
                   ep2d_moduli* an, ep2d_moduli* an_per);

// calc* (EffPlast2D.cu:1412-1539) from the records of the three load steps.
void final_moduli(int nl, const ep2d_step_record& r0, const ep2d_step_record* r1, const ep2d_step_record* r2,
                  ep2d_moduli* num, ep2d_moduli* num_per);

// Validate an ep2d_params; returns EP2D_OK or an error status (with message).
int validate_params(const ep2d_params& p);
// The iteration kernel a handle uses: the form and rows the parameters name, or the
// library's choice where they are 0: the stream form, with the tallest segments (64,
// 32 or 16 rows) that still give every SM of the device 16 warps' worth of segments, or
// the tile form (16 rows) when 16-row segments would leave fewer than 6 warps per SM
// (sm_count <= 0: stream form, SEG_DEFAULT rows).
IterShape shape_of(const ep2d_params& p, int sm_count = 0);

// Device row pitch (elements) for an nx-wide grid.
int row_pitch(int nx);

// Per-device kernel attributes, once per device (the device must be current).
int prepare_device(int dev);

class Rve {
 public:
  Rve() = default;
  ~Rve();
  Rve(const Rve&) = delete;
  Rve& operator=(const Rve&) = delete;

  // allocate and initialise (constructor of the reference); stream may be null: own one
  int create(const ep2d_params& p, cudaStream_t stream = nullptr);
  void release();
  int reset();  // zero all fields and records (a freshly constructed object)

  // bytes of device memory one RVE with these parameters holds
  static size_t footprint(const ep2d_params& p);

  // ComputeEffParams (EffPlast2D.cu:311-698)
  int solve_step(int step, double load_step_value, const double load_type[3], int n_time_steps);
  // ComputeEffModuli without printing (EffPlast2D.cu:179-229)
  int compute_eff_moduli(double init_load_value, const double load_type[3], int n_time_steps,
                         ep2d_result* out);
  // ComputeEffDamping without printing (EffPlast2D.cu:230-310), nl >= 4
  int compute_eff_damping(double init_load_value, const double load_type[3], int n_time_steps, double load_value,
                          int64_t* total_iterations);
  // load value of increment `step` (1 .. nl-1) of the damping chain
  static double damping_step_value(int step, int nl, double load_value);

  // building blocks (used by solve_step, by the batch solver and by the tests)
  void begin_chain(const double load_type[3]);  // ComputeEffModuli's prologue
  // load value, load type and time steps of load step `step` of the chain
  static void step_load(int step, double init, const double lt[3], int nts, double* lsv, double lt_out[3],
                        int* nts_out);
  int begin_step(int step, int n_time_steps);   // ComputeEffParams' prologue
  void finish_chain(int n_time_steps, ep2d_result* out);  // calc* and the result
  int begin_time_step(int step, int it, double load_step_value, const double load_type[3], int n_time_steps);
  int iterate(int64_t n, bool record_last);  // n iterations; the last one records stresses
  int launch_one(bool record);                // one iteration kernel (no stats)
  int reset_vmax();
  int check_resident();  // the resident form's barrier error flag (sticky)
  int read_error(double* error);              // after a recording launch: D2H + error formula
  int finish_time_step(int step, int it);     // averaging etc. into the record
  double error_from_vmax(double vmx, double vmy) const;

  int get_field(int field, double* host) const;
  int set_field(int field, const double* host);
  int static_fields(double* unu, double* j1, double* j2);
  // get_sigma_2D.m:170-194's plastic zone and polar stresses from the recorded state
  int polar_fields(double load_value, double* snrr, double* snff, double* sarr, double* saff, uint8_t* plast);
  // SaveAnStatic2D's analytic fields and error statistics (EffPlast2D.cu:1060-1292)
  int analytic_fields(double delta_p, double tau_infty, double* uan, double* eu, double* j1an, double* j2an,
                      double* ej1, double* ej2, double stats[6]);

  // state
  ep2d_params prm{};
  Derived d{};
  Geo g{};
  Fields f{};
  IterShape shape{};  // form and rows of the iteration kernel (shape_of(prm))
  // velocities stored in FP32 (the mixed path, and both phases of the FP32 bulk)
  bool mixed() const { return prm.precision == EP2D_MIXED || prm.precision == EP2D_F32_BULK; }
  // FP32 bulk: true while the state is in its FP32 form (u' in f.ux32/uy32)
  bool f32 = false;
  int f32_rows = SEG_DEFAULT;        // segment height of the FP32 launches (stream form)
  double f32_drop = 0.7;             // stay in FP32 while error_k < f32_drop * error_(k-1)
  int64_t f32_iterations = 0;        // iterations run in FP32
  // plastic zone of get_sigma_2D.m (:126-138): with track on, every FP64 iteration marks
  // the nodes and corners whose trial J2 exceeds coh (mask bits M_YN, M_YC); turning it
  // on clears the marks; polar_fields then uses them (tracked)
  bool track = false, tracked = false;
  int track_plastic_zone(bool on);
  int enter_f32();                   // FP64 U -> u' (at the start of a time step)
  int leave_f32();                   // u' -> FP64 U
  int cur = 0;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;

  // records (EffPlast2D.h:108-117)
  // per load step (prm.nl of them): time steps, records, checkpoint errors
  std::vector<int> nts;
  std::vector<std::vector<ep2d_step_record>> rec;
  std::vector<std::vector<std::vector<double>>> checks;
  double ces[3] = {0.0, 0.0, 0.0};  // curEffStrain
  double load_type_[3] = {0.0, 0.0, 0.0};
  bool have_step0 = false;
  ep2d_moduli an{}, an_per{}, num{}, num_per{};

  // statistics
  double kernel_ms = 0.0;
  int64_t launches = 0;      // fused iteration kernel (a resident launch counts once)
  int64_t resident_launches = 0;  // of them, resident-form launches
  int64_t aux_launches = 0;  // preload, averaging, boundary, gather, mask
  int64_t cell_updates = 0;

  // device scratch
  void* dmem = nullptr;
  double* d_partials = nullptr;
  double* d_out = nullptr;  // [NAVG avg][NAVG boundary][samples]
  unsigned long long* d_idx = nullptr;
  double* h_pin = nullptr;  // pinned mirror of d_out plus 2 vmax words
  std::vector<HoleSample> holes;

 private:
  int run_plain(int64_t n);
  int capture(int parity);
  cudaGraphExec_t gexec_[2] = {nullptr, nullptr};
  cudaGraphExec_t gexec32_[2] = {nullptr, nullptr};  // FP32 bulk (hold the affine strains)
  static constexpr int kGraphLen = 64;  // iterations per captured graph (even)
  cudaEvent_t ev_[2] = {nullptr, nullptr};
};

}  // namespace ep2d
