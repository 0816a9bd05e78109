// ep2d_api.cpp -- the extern "C" boundary (include/ep2d.h).  No exception crosses it;
// every entry point returns a status and leaves a message for ep2d_last_error().
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <new>

#include "ep2d.h"
#include "ep2d_rve.hpp"

using ep2d::fail;

struct ep2d_handle {
  ep2d::Rve rve;
};

#define EP2D_GUARD(body)                                          \
  try {                                                           \
    body                                                          \
  } catch (const std::bad_alloc&) {                               \
    return fail(EP2D_ERR_NOMEM, "host allocation failed");        \
  } catch (const std::exception& ex) {                            \
    return fail(EP2D_ERR_STATE, std::string("exception: ") + ex.what()); \
  } catch (...) {                                                 \
    return fail(EP2D_ERR_STATE, "unknown exception");             \
  }

extern "C" {

const char* ep2d_version(void) { return "effplast2d_b200 0.1.0 (sm_100a)"; }

const char* ep2d_last_error(void) { return ep2d::last_error(); }

int ep2d_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

int ep2d_read_pa(const char* path, double pa_out[EP2D_NPARS]) {
  if (!path || !pa_out) return fail(EP2D_ERR_ARG, "null argument");
  std::FILE* fp = std::fopen(path, "rb");
  if (!fp) return fail(EP2D_ERR_IO, std::string("ERROR:  Cannot open file ") + path + "!");
  const size_t n = std::fread(pa_out, sizeof(double), EP2D_NPARS, fp);
  std::fclose(fp);
  if (n != EP2D_NPARS)
    return fail(EP2D_ERR_IO, std::string("short read of ") + path + ": " + std::to_string(n) + " of 11 values");
  return EP2D_OK;
}

// get_sigma_2D.m:3-32, operation by operation (MATLAB evaluates left to right).
int ep2d_make_pa(double lx, double ly, int32_t nx, int32_t ny, double k0, double g0, double rho0, double cfl,
                 double yield, double porosity, double n_pores, double pa_out[EP2D_NPARS]) {
  if (!pa_out) return fail(EP2D_ERR_ARG, "null output");
  if (nx < 2 || ny < 2) return fail(EP2D_ERR_ARG, "nx, ny must be >= 2");
  const double pi = 3.141592653589793;  // MATLAB pi
  const double coh = yield * std::sqrt(2.0);
  const double rad = std::sqrt(porosity * lx * ly / (pi * n_pores * n_pores));
  const double dX = lx / (nx - 1);
  const double dY = ly / (ny - 1);
  const double dt = cfl * std::min(dX, dY) / std::sqrt((k0 + 4 * g0 / 3) / rho0);
  const double dampX = 4.0 / dt / nx;
  const double dampY = 4.0 / dt / ny;
  const double pa[EP2D_NPARS] = {dX, dY, dt, k0, g0, rho0, dampX, dampY, coh, rad, n_pores};
  std::memcpy(pa_out, pa, sizeof(pa));
  return EP2D_OK;
}

int ep2d_field_dims(int32_t nx, int32_t ny, int32_t field, int32_t* width, int32_t* height) {
  if (!width || !height || field < 0 || field >= EP2D_NFIELDS) return fail(EP2D_ERR_ARG, "bad field");
  switch (field) {
    case EP2D_FIELD_TAUXY: case EP2D_FIELD_J2XY: *width = nx - 1; *height = ny - 1; break;
    case EP2D_FIELD_UX: case EP2D_FIELD_VX: *width = nx + 1; *height = ny; break;
    case EP2D_FIELD_UY: case EP2D_FIELD_VY: *width = nx; *height = ny + 1; break;
    default: *width = nx; *height = ny;
  }
  return EP2D_OK;
}

int ep2d_create(const ep2d_params* params, ep2d_handle** out) {
  if (!params || !out) return fail(EP2D_ERR_ARG, "null argument");
  *out = nullptr;
  EP2D_GUARD({
    ep2d_handle* h = new ep2d_handle();
    int rc = h->rve.create(*params);
    if (rc) {
      delete h;
      return rc;
    }
    *out = h;
    return EP2D_OK;
  })
}

int ep2d_destroy(ep2d_handle* h) {
  if (!h) return EP2D_OK;
  EP2D_GUARD({
    delete h;
    return EP2D_OK;
  })
}

int ep2d_reset(ep2d_handle* h) {
  if (!h) return fail(EP2D_ERR_ARG, "null handle");
  EP2D_GUARD({ return h->rve.reset(); })
}

int ep2d_iterate(ep2d_handle* h, int64_t n_iter) {
  if (!h || n_iter < 0) return fail(EP2D_ERR_ARG, "bad handle or count");
  EP2D_GUARD({
    int rc = h->rve.iterate(n_iter, true);
    if (rc) return rc;
    ep2d::DeviceScope ds(h->rve.device);
    cudaError_t e = cudaStreamSynchronize(h->rve.stream);
    if (e != cudaSuccess) return fail(EP2D_ERR_CUDA, std::string("iterate: ") + cudaGetErrorString(e));
    return EP2D_OK;
  })
}

int ep2d_get_field(ep2d_handle* h, int32_t field, double* host_out) {
  if (!h) return fail(EP2D_ERR_ARG, "null handle");
  EP2D_GUARD({ return h->rve.get_field(field, host_out); })
}

int ep2d_set_field(ep2d_handle* h, int32_t field, const double* host_in) {
  if (!h) return fail(EP2D_ERR_ARG, "null handle");
  EP2D_GUARD({ return h->rve.set_field(field, host_in); })
}

int ep2d_solve_step(ep2d_handle* h, int32_t step, double load_step_value, const double load_type[3],
                    int32_t n_time_steps, ep2d_step_record* out) {
  if (!h) return fail(EP2D_ERR_ARG, "null handle");
  EP2D_GUARD({
    int rc = h->rve.solve_step(step, load_step_value, load_type, n_time_steps);
    if (rc) return rc;
    if (out)
      for (int t = 0; t < n_time_steps; t++) out[t] = h->rve.rec[step][t];
    return EP2D_OK;
  })
}

int ep2d_get_record(ep2d_handle* h, int32_t step, int32_t time_step, ep2d_step_record* out) {
  if (!h || !out) return fail(EP2D_ERR_ARG, "null argument");
  if (step < 0 || step >= (int)h->rve.nts.size() || time_step < 0 || time_step >= h->rve.nts[step])
    return fail(EP2D_ERR_ARG, "no record for this (step, time_step)");
  *out = h->rve.rec[step][time_step];
  return EP2D_OK;
}

int ep2d_get_check_errors(ep2d_handle* h, int32_t step, int32_t time_step, double* errors_out, int32_t max_n,
                          int32_t* n_out) {
  if (!h) return fail(EP2D_ERR_ARG, "null handle");
  if (step < 0 || step >= (int)h->rve.nts.size() || time_step < 0 || time_step >= h->rve.nts[step])
    return fail(EP2D_ERR_ARG, "no record for this (step, time_step)");
  const std::vector<double>& c = h->rve.checks[step][time_step];
  if (n_out) *n_out = (int32_t)c.size();
  for (int32_t k = 0; errors_out && k < max_n && k < (int32_t)c.size(); k++) errors_out[k] = c[k];
  return EP2D_OK;
}

int ep2d_compute_eff_moduli(ep2d_handle* h, double init_load_value, const double load_type[3],
                            int32_t n_time_steps, ep2d_result* out) {
  if (!h) return fail(EP2D_ERR_ARG, "null handle");
  EP2D_GUARD({ return h->rve.compute_eff_moduli(init_load_value, load_type, n_time_steps, out); })
}

int ep2d_compute_eff_damping(ep2d_handle* h, double init_load_value, const double load_type[3],
                             int32_t n_time_steps, double load_value, int64_t* total_iterations) {
  if (!h) return fail(EP2D_ERR_ARG, "null handle");
  EP2D_GUARD({
    return h->rve.compute_eff_damping(init_load_value, load_type, n_time_steps, load_value, total_iterations);
  })
}

int ep2d_static_fields(ep2d_handle* h, double* unu_abs, double* j1nu, double* j2nu) {
  if (!h) return fail(EP2D_ERR_ARG, "null handle");
  EP2D_GUARD({ return h->rve.static_fields(unu_abs, j1nu, j2nu); })
}

int ep2d_analytic_fields(ep2d_handle* h, double delta_p, double tau_infty, double* uan_abs, double* error_uabs,
                         double* j1an, double* j2an, double* error_j1, double* error_j2, double stats[6]) {
  if (!h) return fail(EP2D_ERR_ARG, "null handle");
  EP2D_GUARD({
    return h->rve.analytic_fields(delta_p, tau_infty, uan_abs, error_uabs, j1an, j2an, error_j1, error_j2, stats);
  })
}

int ep2d_get_stats(ep2d_handle* h, double* kernel_ms, int64_t* launches, int64_t* cell_updates,
                   int64_t* all_launches) {
  if (!h) return fail(EP2D_ERR_ARG, "null handle");
  if (kernel_ms) *kernel_ms = h->rve.kernel_ms;
  if (launches) *launches = h->rve.launches;
  if (all_launches) *all_launches = h->rve.launches + h->rve.aux_launches;
  if (cell_updates) *cell_updates = h->rve.cell_updates;
  return EP2D_OK;
}

int ep2d_track_plastic_zone(ep2d_handle* h, int32_t on) {
  if (!h) return fail(EP2D_ERR_ARG, "null handle");
  EP2D_GUARD({ return h->rve.track_plastic_zone(on != 0); })
}

int ep2d_iterate_f32(ep2d_handle* h, int64_t n_iter) {
  if (!h) return fail(EP2D_ERR_ARG, "null handle");
  if (n_iter < 0) return fail(EP2D_ERR_ARG, "n_iter must be >= 0");
  if (h->rve.prm.precision != EP2D_F32_BULK)
    return fail(EP2D_ERR_STATE, "ep2d_iterate_f32 needs a handle created with EP2D_F32_BULK");
  EP2D_GUARD({
    int rc = h->rve.enter_f32();
    if (rc) return rc;
    rc = h->rve.iterate(n_iter, false);
    const int rc2 = h->rve.leave_f32();
    if (rc) return rc;
    h->rve.f32_iterations += n_iter;
    return rc2;
  })
}

int ep2d_get_f32_iterations(ep2d_handle* h, int64_t* f32_iterations) {
  if (!h || !f32_iterations) return fail(EP2D_ERR_ARG, "null argument");
  *f32_iterations = h->rve.f32_iterations;
  return EP2D_OK;
}

int ep2d_polar_fields(ep2d_handle* h, double load_value, double* snu_rr, double* snu_ff, double* san_rr,
                      double* san_ff, uint8_t* plastic) {
  if (!h) return fail(EP2D_ERR_ARG, "null handle");
  EP2D_GUARD({ return h->rve.polar_fields(load_value, snu_rr, snu_ff, san_rr, san_ff, plastic); })
}

int ep2d_get_kernel_shape(ep2d_handle* h, int32_t* kernel, int32_t* rows) {
  if (!h) return fail(EP2D_ERR_ARG, "null handle");
  if (kernel)
    *kernel = h->rve.shape.form == ep2d::FORM_TILE       ? EP2D_KERNEL_TILE
              : h->rve.shape.form == ep2d::FORM_RESIDENT ? EP2D_KERNEL_RESIDENT
                                                         : EP2D_KERNEL_STREAM;
  if (rows) *rows = h->rve.shape.rows;
  return EP2D_OK;
}

int ep2d_check_grid_barrier(int32_t device, int32_t blocks, int32_t missing, int32_t rounds, int64_t timeout_ns,
                            int32_t* passed, int32_t* flag) {
  if (!passed || !flag) return fail(EP2D_ERR_ARG, "null argument");
  if (blocks < 1 || missing < 0 || missing > blocks || rounds < 0 || timeout_ns < 0)
    return fail(EP2D_ERR_ARG, "need 1 <= blocks, 0 <= missing <= blocks, rounds >= 0, timeout_ns >= 0");
  if (timeout_ns > 10000000000LL) return fail(EP2D_ERR_ARG, "timeout_ns above 10 s");
  if (rounds > 1000000) return fail(EP2D_ERR_ARG, "rounds above 1,000,000");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(EP2D_ERR_NODEV, "no CUDA device");
  if (device < 0 || device >= ndev) return fail(EP2D_ERR_ARG, "device index out of range");
  ep2d::DeviceScope ds(device);
  unsigned* d = nullptr;
  cudaError_t e = cudaMalloc(&d, 8 * sizeof(unsigned));
  if (e != cudaSuccess) return fail(EP2D_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  unsigned hv[3] = {};
  e = ep2d::launch_grid_barrier_check(d, blocks, missing, rounds, (unsigned long long)timeout_ns, d + 4, nullptr);
  if (e == cudaSuccess) e = cudaMemcpy(hv, d + 2, sizeof(hv), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return fail(EP2D_ERR_CUDA, std::string("grid barrier check: ") + cudaGetErrorString(e));
  *flag = (int32_t)hv[0];    // gbar[2]
  *passed = (int32_t)hv[2];  // out[0]
  return EP2D_OK;
}

// sizeof() of every ABI struct, for the binding's layout check
int ep2d_abi_sizes(int64_t* out, int32_t n) {
  const int64_t s[7] = {(int64_t)sizeof(ep2d_params),      (int64_t)sizeof(ep2d_step_record),
                        (int64_t)sizeof(ep2d_moduli),      (int64_t)sizeof(ep2d_result),
                        (int64_t)sizeof(ep2d_rve_spec),    (int64_t)sizeof(ep2d_batch_config),
                        (int64_t)sizeof(ep2d_batch_stats)};
  for (int32_t k = 0; k < n && k < 7; k++) out[k] = s[k];
  return 7;
}

}  // extern "C"
