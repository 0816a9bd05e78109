// ep2d_rve.cpp -- host orchestration of one RVE (compiled by the host C++ compiler with
// -ffp-contract=off, so every host-side expression below rounds exactly like the
// reference's host code, which nvcc hands to the same compiler with default flags).
#include "ep2d_rve.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <mutex>
#include <set>

namespace ep2d {

// ---- errors ---------------------------------------------------------------------
namespace {
thread_local std::string t_last_error;
}
void set_error(const std::string& msg) { t_last_error = msg; }
const char* last_error() { return t_last_error.c_str(); }
int fail(int code, const std::string& msg) {
  t_last_error = msg;
  return code;
}

#define EP2D_CK(call)                                                                       \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess) return fail(EP2D_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

DeviceScope::DeviceScope(int dev) {
  if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  if (prev != dev) cudaSetDevice(dev);
}
DeviceScope::~DeviceScope() {
  int now = -1;
  if (prev >= 0 && cudaGetDevice(&now) == cudaSuccess && now != prev) cudaSetDevice(prev);
}

// ---- parameters -------------------------------------------------------------------
Derived derive(const ep2d_params& p) {
  Derived d{};
  d.dX = p.pa[0];
  d.dY = p.pa[1];
  d.dT = p.pa[2];
  d.K0 = p.pa[3];
  d.G0 = p.pa[4];
  d.E0 = 9.0 * d.K0 * d.G0 / (3.0 * d.K0 + d.G0);
  d.nu0 = (1.5 * d.K0 - d.G0) / (3.0 * d.K0 + d.G0);
  d.rad = p.pa[9];
  d.Y = p.pa[8] / std::sqrt(2.0);
  d.nPores = p.pa[10];
  const long nX = p.nx, nY = p.ny;
  d.lX = (nX - 1) * d.dX;
  d.lY = (nY - 1) * d.dY;
  d.porosity = 3.1415926 * d.rad * d.rad * d.nPores * d.nPores / (d.lX * d.lY);
  return d;
}

int row_pitch(int nx) { return ((nx + 1 + 31) / 32) * 32; }

int validate_params(const ep2d_params& p) {
  if (p.nx < 8 || p.ny < 8) return fail(EP2D_ERR_ARG, "grid must be at least 8 x 8");
  if (p.nx > (1 << 16) || p.ny > (1 << 16)) return fail(EP2D_ERR_ARG, "grid larger than 65536 per side");
  if ((int64_t)row_pitch(p.nx) * (p.ny + 1) >= ((int64_t)1 << 31))
    return fail(EP2D_ERR_ARG, "grid too large: a field would exceed 2^31 elements");
  if (p.nl < 1 || p.nl > EP2D_MAX_STEPS) return fail(EP2D_ERR_ARG, "nl (NL) must be in [1, 64]");
  if (p.check_every < 1) return fail(EP2D_ERR_ARG, "check_every must be >= 1");
  if (p.niter < 0) return fail(EP2D_ERR_ARG, "niter must be >= 0");
  if (p.precision != EP2D_FP64 && p.precision != EP2D_MIXED && p.precision != EP2D_F32_BULK)
    return fail(EP2D_ERR_ARG, "unknown precision");
  for (int k = 0; k < EP2D_NPARS; k++)
    if (!std::isfinite(p.pa[k])) return fail(EP2D_ERR_ARG, "pa[" + std::to_string(k) + "] is not finite");
  if (!(p.pa[0] > 0.0) || !(p.pa[1] > 0.0) || !(p.pa[2] > 0.0))
    return fail(EP2D_ERR_ARG, "dX, dY and dt must be positive");
  if (!(p.pa[5] > 0.0)) return fail(EP2D_ERR_ARG, "rho0 must be positive");
  if (!(p.pa[10] >= 1.0) || p.pa[10] > 64.0) return fail(EP2D_ERR_ARG, "N (pores per side) must be in [1, 64]");
  if (!(p.pa[9] >= 0.0)) return fail(EP2D_ERR_ARG, "rad must be >= 0");
  if (p.kernel < EP2D_KERNEL_AUTO || p.kernel > EP2D_KERNEL_RESIDENT) return fail(EP2D_ERR_ARG, "unknown kernel form");
  if (p.rows != 0 && !shape_valid(shape_of(p)))
    return fail(EP2D_ERR_ARG,
                "rows must be 8, 16 or 32 for the tile and resident forms and 4..1024 for the stream form");
  return EP2D_OK;
}

IterShape shape_of(const ep2d_params& p, int sm_count) {
  IterShape s;
  s.form = p.kernel == EP2D_KERNEL_TILE       ? FORM_TILE
           : p.kernel == EP2D_KERNEL_RESIDENT ? FORM_RESIDENT
                                              : FORM_STREAM;
  s.rows = p.rows ? p.rows : (s.form == FORM_STREAM ? SEG_DEFAULT : TILE_Y);
  if (p.rows == 0 && s.form == FORM_STREAM && sm_count > 0) {
    const int64_t strips = (p.nx + STREAM_COLS - 1) / STREAM_COLS, sms = sm_count;
    auto warps = [&](int rows) { return strips * ((p.ny + rows - 1) / rows); };  // one per segment
    // Segment height: the tallest power of two from 64 down that gives 16 warps of
    // segments per SM; below 16 rows the march's three extra rows per segment weigh more
    // (75 % at 4 rows), so 8 rows stay while they give 9 warps per SM.  Measured, us per
    // iteration, NL=3: 1024^2 16 rows 16.3 (8: 18.2); 768^2 8 rows 14.3 (16: 16.1);
    // 640^2 8 rows 9.6 (4: 10.7); 576^2 8 rows 9.6 (4: 9.9); 512^2 4 rows 8.8 (8: 9.5).
    s.rows = 64;
    while (s.rows > SEG_MIN && warps(s.rows) < (s.rows > 8 ? 16 : 9) * sms) s.rows /= 2;
    // Too few 4-row segments to keep the SMs busy: a warp's march latency then sets the
    // iteration time, and the tile form, one thread per cell, is faster.  With the
    // return map (NL > 1) below 5.5 warps per SM (256^2: tile 5.8 vs 4-row stream 6.1 us;
    // 320^2: 6.5 vs 6.1), elastic RVEs below 12 (384^2: 5.6 vs 6.0; 512^2: 6.9 vs 6.2).
    // Both forms round alike.  Tiles of 8 rows where 16-row tiles would give fewer than
    // two per SM (128^2 4.4 vs 5.2 us, 256^2 5.8 vs 7.2 us).  On elastic RVEs with at
    // most two 8-row tiles per SM (up to ~256^2) the resident form, all iterations of a
    // checkpoint interval in one launch, is faster still (128^2: 4.03 vs 4.39 us, 256^2:
    // 4.55 vs 4.90 us; 320^2: 5.12 vs 4.97); with the return map it is slower at every
    // size (256^2: 6.36 vs 5.77 us).
    if (p.kernel == EP2D_KERNEL_AUTO && 2 * warps(SEG_MIN) < (p.nl == 1 ? 24 : 11) * sms) {
      s.form = FORM_TILE;
      const int64_t tx = (p.nx + TILE_X - 1) / TILE_X;
      const int64_t tiles16 = tx * ((p.ny + TILE_Y - 1) / TILE_Y), tiles8 = tx * ((p.ny + 7) / 8);
      s.rows = tiles16 < 2 * sms ? 8 : TILE_Y;
      if (p.nl == 1 && s.rows == 8 && tiles8 <= 2 * sms) s.form = FORM_RESIDENT;
    }
  }
  return s;
}

bool host_in_pore(const Derived& d, long nX, long nY, double x, double y) {
  const double Lx = d.dX * (nX - 1);
  const double Ly = d.dY * (nY - 1);
  const double nPores = d.nPores, rad = d.rad;
  for (int k = 0; k < nPores; k++) {
    for (int l = 0; l < nPores; l++) {
      if (std::sqrt((x - 0.5 * Lx * (1.0 - 1.0 / nPores) + (Lx / nPores) * k) * (x - 0.5 * Lx * (1.0 - 1.0 / nPores) + (Lx / nPores) * k) +
                    (y - 0.5 * Ly * (1.0 - 1.0 / nPores) + (Ly / nPores) * l) * (y - 0.5 * Ly * (1.0 - 1.0 / nPores) + (Ly / nPores) * l)) < rad)
        return true;
    }
  }
  return false;
}

// EffPlast2D.cu:552-595, index arithmetic in size_t as the reference does it
int hole_samples(const Derived& d, long nX, long nY, std::vector<HoleSample>* out) {
  out->clear();
  const double nPores = d.nPores, rad = d.rad, dX = d.dX, dY = d.dY;
  const unsigned long long nux = (unsigned long long)(nX + 1) * nY, nuy = (unsigned long long)nX * (nY + 1);
  auto push_ux = [&](size_t fl) -> bool {
    if (fl >= nux) return false;
    const long i = (long)(fl % (size_t)(nX + 1)), j = (long)(fl / (size_t)(nX + 1));
    out->push_back({fl, host_in_pore(d, nX, nY, -0.5 * dX * nX + dX * i, -0.5 * dY * (nY - 1) + dY * j)});
    return true;
  };
  auto push_uy = [&](size_t fl) -> bool {
    if (fl >= nuy) return false;
    const long i = (long)(fl % (size_t)nX), j = (long)(fl / (size_t)nX);
    out->push_back({(1ull << 62) | fl, host_in_pore(d, nX, nY, -0.5 * dX * (nX - 1) + dX * i, -0.5 * dY * nY + dY * j)});
    return true;
  };
  for (int k = 0; k < nPores; k++) {
    for (int l = 0; l < nPores; l++) {
      const double cxdX = 0.5 * (nX - 1) * (1.0 - 1.0 / nPores) - (static_cast<double>(nX - 1) / nPores) * k;
      const double cydY = 0.5 * (nY - 1) * (1.0 - 1.0 / nPores) - (static_cast<double>(nY - 1) / nPores) * l;
      const double vals[4] = {cxdX - rad / dX + 0.5 * nX, cxdX + rad / dX + 0.5 * nX, cydY - rad / dY + 0.5 * nY,
                              cydY + rad / dY + 0.5 * nY};
      const double cyv = cydY + 0.5 * (nY - 1), cxv = cxdX + 0.5 * (nX - 1);
      // the windows start at index - 1 (left, bottom) and index - 2 (right, top)
      const double lo[4] = {1.0, 2.0, 1.0, 2.0};
      for (int a = 0; a < 4; a++)
        if (!(vals[a] >= lo[a]) || !(vals[a] < 1e18)) return fail(EP2D_ERR_ARG, "pore edge window outside the grid");
      if (!(cyv >= 0.0) || !(cxv >= 0.0)) return fail(EP2D_ERR_ARG, "pore centre outside the grid");
      const size_t cyIdx = static_cast<size_t>(cyv);
      size_t rxIdx = static_cast<size_t>(vals[0]);
      for (int q = 0; q < 5; q++)
        if (!push_ux(cyIdx * (nX + 1) + rxIdx - 1 + q)) return fail(EP2D_ERR_ARG, "pore edge window outside the grid");
      rxIdx = static_cast<size_t>(vals[1]);
      for (int q = 0; q < 5; q++)
        if (!push_ux(cyIdx * (nX + 1) + rxIdx - 2 + q)) return fail(EP2D_ERR_ARG, "pore edge window outside the grid");
      const size_t cxIdx = static_cast<size_t>(cxv);
      size_t ryIdx = static_cast<size_t>(vals[2]);
      for (int q = 0; q < 5; q++)
        if (!push_uy((ryIdx - 1 + q) * nX + cxIdx)) return fail(EP2D_ERR_ARG, "pore edge window outside the grid");
      ryIdx = static_cast<size_t>(vals[3]);
      for (int q = 0; q < 5; q++)
        if (!push_uy((ryIdx - 2 + q) * nX + cxIdx)) return fail(EP2D_ERR_ARG, "pore edge window outside the grid");
    }
  }
  return EP2D_OK;
}

// FindMaxAbs(const std::vector<double>&), EffPlast2D.cu:814-822: signed value of the
// element with the largest magnitude
static double find_max_abs_signed(const double* v, int n) {
  double m = 0.0;
  for (int i = 0; i < n; i++)
    if (std::abs(v[i]) > std::abs(m)) m = v[i];
  return m;
}

void finish_record(const Derived& d, long nX, long nY, int nl, int step, const double* avg, const double* bnd,
                   const std::vector<HoleSample>& hs, const double* samples, ep2d_step_record* r,
                   ep2d_moduli* an, ep2d_moduli* an_per) {
  const double dX = d.dX, dY = d.dY;
  // EffPlast2D.cu:453-503
  const int perOffsetX = static_cast<int>(nX / d.nPores);
  const int perOffsetY = static_cast<int>(nY / d.nPores);
  r->sigma[0] = avg[0] / (nX * nY);
  r->sigma[1] = avg[1] / (nX * nY);
  r->sigma[2] = avg[2] / ((nX - 1) * (nY - 1));
  r->sigma[3] = 0.0 / (nX * nY);
  const long inner = (nX - 2 * perOffsetX) * (nY - 2 * perOffsetY);
  for (int a = 0; a < 4; a++) r->sigma_per[a] = avg[4 + a] / inner;
  for (int a = 0; a < 3; a++) r->eps_per[a] = avg[8 + a] / inner;
  // getDeltaP_honest / _periodic / getTauInfty_honest
  r->delta_p = -0.125 * (bnd[0] / (nX - 2) + bnd[1] / (nY - 2));
  if (d.nPores <= 2) {
    r->delta_p_per = 0.0;
  } else {
    const int nP = static_cast<int>(d.nPores);
    r->delta_p_per = -0.125 * (bnd[2] / (nX * (nP - 2) / nP) + bnd[3] / (nY * (nP - 2) / nP));
  }
  r->tau_infty = -0.125 * (bnd[4] / (nX - 2) + bnd[5] / (nY - 2));
  // hole area, EffPlast2D.cu:549-607
  const double nPores = d.nPores, rad = d.rad;
  double HoleAreaPi = 0.0, InternalHoleAreaPi = 0.0;
  size_t q = 0;
  for (int k = 0; k < nPores; k++) {
    for (int l = 0; l < nPores; l++) {
      double w[4][5];
      for (int a = 0; a < 4; a++)
        for (int b = 0; b < 5; b++, q++) w[a][b] = hs[q].zeroed ? 0.0 : samples[q];
      const double dRx = -0.5 * (find_max_abs_signed(w[0], 5) - find_max_abs_signed(w[1], 5));
      const double dRy = -0.5 * (find_max_abs_signed(w[2], 5) - find_max_abs_signed(w[3], 5));
      HoleAreaPi += (rad + dRx) * (rad + dRy);
      if (k > 0 && l > 0 && k < nPores - 1 && l < nPores - 1) InternalHoleAreaPi += (rad + dRx) * (rad + dRy);
    }
  }
  const double Phi0 = 3.1415926 * rad * rad * nPores * nPores / (dX * (nX - 1) * dY * (nY - 1));
  const double Phi = 3.1415926 * HoleAreaPi / (dX * (nX - 1) * dY * (nY - 1));
  const double PhiPer = nPores > 2 ?
      3.1415926 * InternalHoleAreaPi / (dX * (nX - 1) * dY * (nY - 1) * (nPores - 2) * (nPores - 2) / nPores / nPores) :
      0.0;
  r->hole_area_pi = HoleAreaPi;
  r->internal_hole_area_pi = InternalHoleAreaPi;
  r->phi0 = Phi0;
  r->phi = Phi;
  r->phi_per = PhiPer;
  r->dphi = 3.1415926 * std::abs(HoleAreaPi - rad * rad * nPores * nPores) / (dX * (nX - 1) * dY * (nY - 1));
  r->dphi_per = std::abs(PhiPer - Phi0);
  // analytic moduli, EffPlast2D.cu:643-696
  const double G0 = d.G0, K0 = d.K0, Y = d.Y;
  const double phi = 3.1415926 * rad * rad / (dX * (nX - 1) * dY * (nY - 1));
  r->kphi_exact_elast = r->kd_exact_elast = NAN;
  r->kphi_exact_plast = r->kd_exact_plast = r->kphi_exact_plast_per = r->kd_exact_plast_per = NAN;
  r->g_exact_elast = r->g_exact_plast = r->g_exact_plast_per = NAN;
  if (nl <= 1) {
    const double KphiExactElast = G0 / Phi0;
    r->kphi_exact_elast = KphiExactElast;
    an->kphi = G0 / Phi0;
    r->kd_exact_elast = (1.0 - phi) / (1.0 / K0 + 1.0 / KphiExactElast);
    an->kd = G0 / Phi0;
  } else if (step == 0) {
    const double KphiExactPlast = G0 / Phi / std::exp(std::abs(r->delta_p) / Y - 1.0) /
                                  (1.0 + r->tau_infty * r->tau_infty / Y / Y);
    r->kphi_exact_plast = KphiExactPlast;
    an->kphi = KphiExactPlast;
    r->kd_exact_plast = (1.0 - phi) / (1.0 / K0 + 1.0 / KphiExactPlast);
    an->kd = r->kd_exact_plast;
    const double KphiExactPlastPer = G0 / Phi0 / std::exp(std::abs(r->delta_p_per) / Y - 1.0) /
                                     (1.0 + r->tau_infty * r->tau_infty / Y / Y);
    r->kphi_exact_plast_per = KphiExactPlastPer;
    an_per->kphi = KphiExactPlastPer;
    r->kd_exact_plast_per = (1.0 - phi) / (1.0 / K0 + 1.0 / KphiExactPlastPer);
    an_per->kd = r->kd_exact_plast_per;
  }
  if (nl == 3 && step == 0) {
    r->g_exact_elast = G0 / (1.0 + Phi0);
    r->g_exact_plast = G0 / (1.0 + Phi * std::exp(std::abs(r->delta_p) / Y - 1.0));
    an->g = r->g_exact_plast;
    r->g_exact_plast_per = G0 / (1.0 + Phi0 * std::exp(std::abs(r->delta_p_per) / Y - 1.0));
    an_per->g = r->g_exact_plast_per;
  }
}

void final_moduli(int nl, const ep2d_step_record& r0, const ep2d_step_record* r1, const ep2d_step_record* r2,
                  ep2d_moduli* num, ep2d_moduli* num_per) {
  if (nl == 1) {  // calcBulkModuli_PureElast, EffPlast2D.cu:1412-1428, :1456-1481
    num->kphi = r0.delta_p / r0.dphi;
    num_per->kphi = r0.delta_p_per / r0.dphi_per;
    const double pInc = -0.33333333 * (r0.sigma[0] + r0.sigma[1] + r0.sigma[2]);
    const double epsInc = r0.macro_strain[0] + r0.macro_strain[1];
    num->kd = -pInc / epsInc;
    const double pIncPer = -0.33333333 * (r0.sigma_per[0] + r0.sigma_per[1] + r0.sigma_per[2]);
    const double epsIncPer = r0.eps_per[0] + r0.eps_per[1];
    num_per->kd = -pIncPer / epsIncPer;
  } else if (r1) {  // calcBulkModuli_ElastPlast, EffPlast2D.cu:1429-1445, :1483-1514
    num->kphi = (r1->delta_p - r0.delta_p) / (r1->dphi - r0.dphi);
    num_per->kphi = (r1->delta_p_per - r0.delta_p_per) / (r1->dphi_per - r0.dphi_per);
    const double pInc = -0.33333333 * (r1->sigma[0] + r1->sigma[1] + r1->sigma[2] - r0.sigma[0] - r0.sigma[1] - r0.sigma[2]);
    const double epsInc = r1->macro_strain[0] + r1->macro_strain[1] - r0.macro_strain[0] - r0.macro_strain[1];
    num->kd = -pInc / epsInc;
    const double pIncPer = -0.33333333 * (r1->sigma_per[0] + r1->sigma_per[1] + r1->sigma_per[2] - r0.sigma_per[0] -
                                          r0.sigma_per[1] - r0.sigma_per[2]);
    const double epsIncPer = r1->eps_per[0] + r1->eps_per[1] - r0.eps_per[0] - r0.eps_per[1];
    num_per->kd = -pIncPer / epsIncPer;
  }
  if (nl == 3 && r1 && r2) {  // getG / getGper, EffPlast2D.cu:1516-1539
    num->g = 0.5 * (r2->sigma[0] - r1->sigma[0] - r2->sigma[1] + r1->sigma[1]) /
             (r2->macro_strain[0] - r1->macro_strain[0] - r2->macro_strain[1] + r1->macro_strain[1]);
    num_per->g = 0.5 * (r2->sigma_per[0] - r1->sigma_per[0] - r2->sigma_per[1] + r1->sigma_per[1]) /
                 (r2->eps_per[0] - r1->eps_per[0] - r2->eps_per[1] + r1->eps_per[1]);
  }
}

// ---- Rve ----------------------------------------------------------------------------
namespace {
constexpr int kFieldArrays = 13;  // ux0 ux1 uy0 uy1 vx vy p txx tyy txy txyav j2 j2xy
size_t field_elems(const ep2d_params& p) { return (size_t)row_pitch(p.nx) * (size_t)(p.ny + 1); }
size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }
size_t partial_elems(const ep2d_params& p) { return (size_t)((p.ny - 2 + 3) / 4 + 1) * NAVG; }
size_t n_samples(const ep2d_params& p) {
  const double n = p.pa[10];
  const long k = (long)std::ceil(n);
  return (size_t)(k * k * 20);
}

std::mutex g_prep_mu;
std::set<int> g_prepared;
}  // namespace

int prepare_device(int dev) {
  std::lock_guard<std::mutex> lk(g_prep_mu);
  if (g_prepared.count(dev)) return EP2D_OK;
  cudaError_t e = prepare_kernels();
  if (e != cudaSuccess) return fail(EP2D_ERR_CUDA, std::string("prepare_kernels: ") + cudaGetErrorString(e));
  g_prepared.insert(dev);
  return EP2D_OK;
}

size_t Rve::footprint(const ep2d_params& p) {
  const size_t fe = field_elems(p);
  size_t b = kFieldArrays * align256(fe * sizeof(double));
  if (p.precision == EP2D_F32_BULK) b += 4 * align256(fe * sizeof(float));  // u' (ping-pong)
  b += align256(fe);                                     // mask
  b += align256(partial_elems(p) * sizeof(double));      // averaging partials
  b += align256((2 * NAVG + n_samples(p) + 4) * sizeof(double));  // sums, samples, vmax, barrier
  b += align256(n_samples(p) * sizeof(unsigned long long));
  return b;
}

Rve::~Rve() { release(); }

void Rve::release() {
  if (device >= 0 && (dmem || stream || h_pin)) {
    DeviceScope ds(device);
    for (auto& ge : gexec_)
      if (ge) {
        cudaGraphExecDestroy(ge);
        ge = nullptr;
      }
    for (auto& ge : gexec32_)
      if (ge) {
        cudaGraphExecDestroy(ge);
        ge = nullptr;
      }
    for (auto& ev : ev_)
      if (ev) {
        cudaEventDestroy(ev);
        ev = nullptr;
      }
    if (stream) cudaStreamSynchronize(stream);
    if (dmem) cudaFree(dmem);
    if (h_pin) cudaFreeHost(h_pin);
    if (own_stream && stream) cudaStreamDestroy(stream);
  }
  dmem = nullptr;
  h_pin = nullptr;
  stream = nullptr;
}

int Rve::create(const ep2d_params& p, cudaStream_t s) {
  int rc = validate_params(p);
  if (rc) return rc;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(EP2D_ERR_NODEV, "no CUDA device");
  if (p.device < 0 || p.device >= ndev) return fail(EP2D_ERR_ARG, "device index out of range");
  prm = p;
  device = p.device;
  DeviceScope ds(device);
  rc = prepare_device(device);
  if (rc) return rc;
  int sms = 0;
  EP2D_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  shape = shape_of(p, sms);
  {
    // the FP32 bulk always runs the stream form: the parameters' segment height when they
    // pin the stream form, else the library's choice for the grid
    ep2d_params ps = p;
    if (ps.kernel != EP2D_KERNEL_STREAM) ps.rows = 0;
    ps.kernel = EP2D_KERNEL_STREAM;
    f32_rows = shape_of(ps, sms).rows;
  }
  d = derive(p);
  rc = hole_samples(d, p.nx, p.ny, &holes);
  if (rc) return rc;

  g.nx = p.nx;
  g.ny = p.ny;
  g.pitch = row_pitch(p.nx);
  g.dX = p.pa[0];
  g.dY = p.pa[1];
  g.dT = p.pa[2];
  g.rho = p.pa[5];
  g.dampX = p.pa[6];
  g.dampY = p.pa[7];
  g.coh = p.pa[8];
  g.K0 = p.pa[3];
  g.G0 = p.pa[4];
  g.Kp = 0.01 * g.K0;
  g.Gp = 0.01 * g.G0;
  g.rad = p.pa[9];
  g.nPores = p.pa[10];
  g.rdX = 1.0 / g.dX;
  g.rdY = 1.0 / g.dY;
  g.coh2 = g.coh * g.coh;
  g.cX = 1.0 - g.dT * g.dampX;
  g.cY = 1.0 - g.dT * g.dampY;
  g.dtr = g.dT / g.rho;
  g.coh4 = 4.0 * g.coh;
  g.coh2x16 = g.coh4 * g.coh4;
  g.dtrX = g.dtr * g.rdX;
  g.dtrY = g.dtr * g.rdY;

  if (s) {
    stream = s;
    own_stream = false;
  } else {
    EP2D_CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    own_stream = true;
  }
  const size_t bytes = footprint(p);
  cudaError_t e = cudaMalloc(&dmem, bytes);
  if (e != cudaSuccess) {
    dmem = nullptr;
    cudaGetLastError();
    return fail(EP2D_ERR_NOMEM, "cudaMalloc of " + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(e));
  }
  EP2D_CK(cudaMemsetAsync(dmem, 0, bytes, stream));
  const size_t fe = field_elems(p);
  char* cp = static_cast<char*>(dmem);
  double* arr[kFieldArrays];
  for (int a = 0; a < kFieldArrays; a++) {
    arr[a] = reinterpret_cast<double*>(cp);
    cp += align256(fe * sizeof(double));
  }
  f.ux[0] = arr[0];
  f.ux[1] = arr[1];
  f.uy[0] = arr[2];
  f.uy[1] = arr[3];
  f.vx = arr[4];
  f.vy = arr[5];
  f.p = arr[6];
  f.txx = arr[7];
  f.tyy = arr[8];
  f.txy = arr[9];
  f.txyav = arr[10];
  f.j2 = arr[11];
  f.j2xy = arr[12];
  f.ux32[0] = f.ux32[1] = f.uy32[0] = f.uy32[1] = nullptr;
  if (p.precision == EP2D_F32_BULK) {  // contiguous with the fields: reset() zeroes them too
    float** a32[4] = {&f.ux32[0], &f.ux32[1], &f.uy32[0], &f.uy32[1]};
    for (int a = 0; a < 4; a++) {
      *a32[a] = reinterpret_cast<float*>(cp);
      cp += align256(fe * sizeof(float));
    }
  }
  uint8_t* mask = reinterpret_cast<uint8_t*>(cp);
  f.mask = mask;
  cp += align256(fe);
  d_partials = reinterpret_cast<double*>(cp);
  cp += align256(partial_elems(p) * sizeof(double));
  d_out = reinterpret_cast<double*>(cp);
  f.vmax = reinterpret_cast<unsigned long long*>(d_out + 2 * NAVG + holes.size());
  f.gbar = reinterpret_cast<unsigned*>(d_out + 2 * NAVG + holes.size() + 2);  // zeroed above, never reset
  cp += align256((2 * NAVG + n_samples(p) + 4) * sizeof(double));
  d_idx = reinterpret_cast<unsigned long long*>(cp);

  EP2D_CK(cudaMallocHost(&h_pin, (2 * NAVG + holes.size() + 2) * sizeof(double) + 64));
  std::vector<unsigned long long> codes(holes.size());
  for (size_t k = 0; k < holes.size(); k++) codes[k] = holes[k].code;
  if (!codes.empty())
    EP2D_CK(cudaMemcpyAsync(d_idx, codes.data(), codes.size() * sizeof(unsigned long long), cudaMemcpyHostToDevice,
                            stream));
  EP2D_CK(launch_mask(g, mask, stream));
  aux_launches += 1;
  EP2D_CK(cudaEventCreate(&ev_[0]));
  EP2D_CK(cudaEventCreate(&ev_[1]));
  EP2D_CK(cudaStreamSynchronize(stream));
  cur = 0;
  nts.assign(prm.nl, 0);
  rec.assign(prm.nl, {});
  checks.assign(prm.nl, {});
  return EP2D_OK;
}

int Rve::reset() {
  if (!dmem) return fail(EP2D_ERR_STATE, "handle is not initialised");
  DeviceScope ds(device);
  // the 13 field arrays are contiguous at the start of the allocation
  const size_t bytes = reinterpret_cast<char*>(const_cast<uint8_t*>(f.mask)) - static_cast<char*>(dmem);
  EP2D_CK(cudaMemsetAsync(dmem, 0, bytes, stream));
  EP2D_CK(cudaStreamSynchronize(stream));
  cur = 0;
  nts.assign(prm.nl, 0);
  rec.assign(prm.nl, {});
  checks.assign(prm.nl, {});
  ces[0] = ces[1] = ces[2] = 0.0;
  load_type_[0] = load_type_[1] = load_type_[2] = 0.0;
  have_step0 = false;
  an = an_per = num = num_per = ep2d_moduli{0.0, 0.0, 0.0};
  return EP2D_OK;
}

int Rve::launch_one(bool record) {
  if (f32) EP2D_CK(launch_iter_f32(g, f, cur, prm.nl > 1, record, f32_rows, stream));
  else EP2D_CK(launch_iter(g, f, cur, prm.nl > 1, record, mixed(), shape, stream, track));
  cur ^= 1;
  return EP2D_OK;
}

int Rve::track_plastic_zone(bool on) {
  DeviceScope ds(device);
  if (on == track) {
    if (on) {  // restart the accumulation
      EP2D_CK(launch_clear_track(g, const_cast<uint8_t*>(f.mask), stream));
      aux_launches += 1;
    }
    return EP2D_OK;
  }
  for (auto& ge : gexec_)  // captured with the other kernel
    if (ge) {
      cudaGraphExecDestroy(ge);
      ge = nullptr;
    }
  if (on) {
    // the tracking launches are stream-form launches; the RVE keeps that shape while
    // tracking (both forms round alike)
    if (shape.form != FORM_STREAM) {
      shape.form = FORM_STREAM;
      shape.rows = f32_rows;
    }
    EP2D_CK(launch_clear_track(g, const_cast<uint8_t*>(f.mask), stream));
    aux_launches += 1;
    tracked = true;
  } else {
    int sms = 0;
    EP2D_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    shape = shape_of(prm, sms);
  }
  track = on;
  return EP2D_OK;
}

int Rve::enter_f32() {
  // the affine field of the preloads so far: its strains are the macro strain
  g.exx0 = ces[0];
  g.eyy0 = ces[1];
  g.exy0 = 2.0 * ces[2];
  for (auto& ge : gexec32_)  // captured with the previous strains
    if (ge) {
      cudaGraphExecDestroy(ge);
      ge = nullptr;
    }
  EP2D_CK(launch_to_f32(g, f, cur, stream));
  aux_launches += 1;
  f32 = true;
  return EP2D_OK;
}

int Rve::leave_f32() {
  EP2D_CK(launch_from_f32(g, f, cur, stream));
  aux_launches += 1;
  f32 = false;
  return EP2D_OK;
}

int Rve::capture(int parity) {
  cudaGraph_t graph = nullptr;
  EP2D_CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
  const int saved = cur;
  cur = parity;
  cudaError_t le = cudaSuccess;
  for (int k = 0; k < kGraphLen && le == cudaSuccess; k++) {
    le = f32 ? launch_iter_f32(g, f, cur, prm.nl > 1, false, f32_rows, stream)
             : launch_iter(g, f, cur, prm.nl > 1, false, mixed(), shape, stream, track);
    cur ^= 1;
  }
  cur = saved;
  cudaError_t ee = cudaStreamEndCapture(stream, &graph);
  if (le != cudaSuccess || ee != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    return fail(EP2D_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(le != cudaSuccess ? le : ee));
  }
  cudaError_t ie = cudaGraphInstantiate(f32 ? &gexec32_[parity] : &gexec_[parity], graph, 0);
  cudaGraphDestroy(graph);
  if (ie != cudaSuccess) return fail(EP2D_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ie));
  return EP2D_OK;
}

int Rve::run_plain(int64_t n) {
  if (shape.form == FORM_RESIDENT && !f32 && !track) {
    // one cooperative launch for all n iterations (n == 1: an ordinary tile launch)
    if (n > 1) {
      EP2D_CK(launch_iter_resident(g, f, cur, prm.nl > 1, mixed(), shape.rows, n, RESIDENT_TIMEOUT_NS, stream));
      cur ^= (int)(n & 1);
      launches++;
      resident_launches++;
      return EP2D_OK;
    }
  }
  if (n >= kGraphLen) {
    cudaGraphExec_t* ge = f32 ? gexec32_ : gexec_;
    if (!ge[cur]) {
      int rc = capture(cur);
      if (rc) return rc;
    }
    while (n >= kGraphLen) {
      EP2D_CK(cudaGraphLaunch(ge[cur], stream));  // even length: parity unchanged
      n -= kGraphLen;
      launches += kGraphLen;
    }
  }
  for (; n > 0; n--) {
    int rc = launch_one(false);
    if (rc) return rc;
    launches++;
  }
  return EP2D_OK;
}

int Rve::reset_vmax() {
  EP2D_CK(cudaMemsetAsync(f.vmax, 0, 2 * sizeof(unsigned long long), stream));
  return EP2D_OK;
}

int Rve::iterate(int64_t n, bool record_last) {
  if (n <= 0) return EP2D_OK;
  DeviceScope ds(device);
  EP2D_CK(cudaEventRecord(ev_[0], stream));
  int rc = run_plain(record_last ? n - 1 : n);
  if (rc) return rc;
  if (record_last) {
    rc = reset_vmax();
    if (rc) return rc;
    rc = launch_one(true);
    if (rc) return rc;
    launches++;
  }
  EP2D_CK(cudaEventRecord(ev_[1], stream));
  EP2D_CK(cudaEventSynchronize(ev_[1]));
  float ms = 0.0f;
  EP2D_CK(cudaEventElapsedTime(&ms, ev_[0], ev_[1]));
  kernel_ms += ms;
  cell_updates += n * (int64_t)prm.nx * prm.ny;
  return check_resident();
}

double Rve::error_from_vmax(double vmx, double vmy) const {
  // EffPlast2D.cu:411-412 (std::max kept: max(|e0|, max(e1, e2)))
  const double a = std::abs(ces[0]);
  const double b = std::max(ces[1], ces[2]);
  return (vmx / (d.dX * (prm.nx - 1)) + vmy / (d.dY * (prm.ny - 1))) * d.dT / std::max(a, b);
}

// The resident form's barrier error flag (sticky), read back; EP2D_OK if the RVE never
// ran that form.
int Rve::check_resident() {
  if (!resident_launches) return EP2D_OK;
  unsigned* hf = reinterpret_cast<unsigned*>(h_pin + 2 * NAVG + holes.size() + 2);
  EP2D_CK(cudaMemcpyAsync(hf, f.gbar + 2, sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
  EP2D_CK(cudaStreamSynchronize(stream));
  if (*hf)
    return fail(EP2D_ERR_CUDA,
                "resident form: a grid barrier wait ran out (a CTA did not arrive); the RVE's state is invalid");
  return EP2D_OK;
}

int Rve::read_error(double* error) {
  unsigned long long* hv = reinterpret_cast<unsigned long long*>(h_pin + 2 * NAVG + holes.size());
  EP2D_CK(cudaMemcpyAsync(hv, f.vmax, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream));
  EP2D_CK(cudaStreamSynchronize(stream));
  {
    const int rc = check_resident();
    if (rc) return rc;
  }
  double vmx, vmy;
  std::memcpy(&vmx, &hv[0], sizeof(double));
  std::memcpy(&vmy, &hv[1], sizeof(double));
  *error = error_from_vmax(vmx, vmy);
  return EP2D_OK;
}

int Rve::begin_time_step(int step, int it, double lsv, const double lt[3], int n_time_steps) {
  DeviceScope ds(device);
  ep2d_step_record& r = rec[step][it];
  std::memset(&r, 0, sizeof(r));
  r.step = step;
  r.time_step = it;
  // EffPlast2D.cu:349-358
  const double dUxdx = lsv * lt[0] / static_cast<double>(n_time_steps);
  const double dUydy = lsv * lt[1] / static_cast<double>(n_time_steps);
  const double dUxdy = lsv * lt[2] / static_cast<double>(n_time_steps);
  ces[0] += dUxdx;
  ces[1] += dUydy;
  ces[2] += dUxdy;
  std::memcpy(r.macro_strain, ces, sizeof(ces));
  const int zero_first = (step == 0 && it == 0) ? 1 : 0;
  EP2D_CK(launch_preload(g, f, cur, dUxdx, dUydy, dUxdy, zero_first, stream));
  aux_launches += 1;
  return EP2D_OK;
}

int Rve::finish_time_step(int step, int it) {
  DeviceScope ds(device);
  ep2d_step_record& r = rec[step][it];
  const int perOffsetX = static_cast<int>(prm.nx / d.nPores);
  const int perOffsetY = static_cast<int>(prm.ny / d.nPores);
  EP2D_CK(launch_average(g, f, cur, d.nu0, perOffsetX, perOffsetY, d_partials, d_out, stream));
  EP2D_CK(launch_boundary(g, f, d_out + NAVG, stream));
  EP2D_CK(launch_gather(g, f, cur, d_idx, (int)holes.size(), d_out + 2 * NAVG, stream));
  aux_launches += holes.empty() ? 3 : 4;
  EP2D_CK(cudaMemcpyAsync(h_pin, d_out, (2 * NAVG + holes.size()) * sizeof(double), cudaMemcpyDeviceToHost, stream));
  EP2D_CK(cudaStreamSynchronize(stream));
  finish_record(d, prm.nx, prm.ny, prm.nl, step, h_pin, h_pin + NAVG, holes, h_pin + 2 * NAVG, &r, &an, &an_per);
  return EP2D_OK;
}

int Rve::begin_step(int step, int n_time_steps) {
  if (step < 0 || step >= prm.nl) return fail(EP2D_ERR_ARG, "step must be in [0, nl)");
  if (n_time_steps < 1) return fail(EP2D_ERR_ARG, "n_time_steps must be >= 1");
  if (step > 0 && !have_step0) return fail(EP2D_ERR_STATE, "increment step before the preload (step 0)");
  nts[step] = n_time_steps;
  rec[step].assign(n_time_steps, ep2d_step_record{});
  checks[step].assign(n_time_steps, std::vector<double>{});
  if (step == 0) {
    ces[0] = ces[1] = ces[2] = 0.0;
    have_step0 = true;
  }
  return EP2D_OK;
}

void Rve::begin_chain(const double lt[3]) {
  std::memcpy(load_type_, lt, sizeof(load_type_));
  an = an_per = num = num_per = ep2d_moduli{0.0, 0.0, 0.0};
}

// ComputeEffModuli's three load steps (EffPlast2D.cu:188-205): the preload, then the
// spherical and deviatoric increments of incPercent = 0.005 (EffPlast2D.h:105)
void Rve::step_load(int step, double init, const double lt[3], int nts, double* lsv, double lt_out[3], int* nts_out) {
  const double incPercent = 0.005;
  const double sph[3] = {0.5 * (lt[0] + lt[1]), 0.5 * (lt[0] + lt[1]), 0.0};
  const double dev[3] = {lt[0] - sph[0], lt[1] - sph[1], lt[2]};
  if (step == 0) {
    *lsv = init;
    std::memcpy(lt_out, lt, 3 * sizeof(double));
    *nts_out = nts;
  } else {
    *lsv = init * incPercent;
    std::memcpy(lt_out, step == 1 ? sph : dev, 3 * sizeof(double));
    *nts_out = 1;
  }
}

void Rve::finish_chain(int n_time_steps, ep2d_result* out) {
  const ep2d_step_record& r0 = rec[0][n_time_steps - 1];
  final_moduli(prm.nl, r0, prm.nl > 1 ? &rec[1][0] : nullptr, prm.nl == 3 ? &rec[2][0] : nullptr, &num, &num_per);
  if (!out) return;
  std::memset(out, 0, sizeof(*out));
  out->an = an;
  out->an_per = an_per;
  out->num = num;
  out->num_per = num_per;
  out->nl = prm.nl;
  out->n_time_steps = n_time_steps;
  int allc = 1;
  int64_t tot = 0;
  for (int a = 0; a < prm.nl; a++)
    for (int t = 0; t < nts[a]; t++) {
      tot += rec[a][t].iterations;
      allc &= rec[a][t].converged;
    }
  out->total_iterations = tot;
  out->all_converged = allc;
}

int Rve::solve_step(int step, double lsv, const double lt[3], int n_time_steps) {
  if (!lt) return fail(EP2D_ERR_ARG, "load_type is null");
  DeviceScope ds(device);
  int rc0 = begin_step(step, n_time_steps);
  if (rc0) return rc0;
  const int64_t ce = prm.check_every;
  for (int it = 0; it < n_time_steps; it++) {
    int rc = begin_time_step(step, it, lsv, lt, n_time_steps);
    if (rc) return rc;
    ep2d_step_record& r = rec[step][it];
    // FP32 bulk: the time step starts in the FP32 form (below)
    if (prm.precision == EP2D_F32_BULK) {
      rc = enter_f32();
      if (rc) return rc;
    }
    double f32_prev = std::numeric_limits<double>::infinity();
    // iteration loop, EffPlast2D.cu:386-428
    double error = 0.0;
    int64_t iter = 0, iters = prm.niter;
    int converged = 0;
    EP2D_CK(cudaEventRecord(ev_[0], stream));
    while (iter < prm.niter) {
      const int64_t block_end = std::min<int64_t>(prm.niter, (iter / ce + 1) * ce);
      // the last interval, and with it the stresses the step records, is always FP64
      if (f32 && block_end == prm.niter) {
        rc = leave_f32();
        if (rc) return rc;
      }
      const bool in_f32 = f32;
      rc = run_plain(block_end - iter - 1);
      if (rc) return rc;
      rc = reset_vmax();
      if (rc) return rc;
      rc = launch_one(true);
      if (rc) return rc;
      launches++;
      if (in_f32) f32_iterations += block_end - iter;
      iter = block_end;
      if (iter % ce == 0) {
        rc = read_error(&error);
        if (rc) return rc;
        checks[step][it].push_back(error);
        r.n_checks++;
        if (in_f32) {
          // An FP32 checkpoint never decides convergence.  The FP32 form continues
          // while its residual falls by more than f32_drop per interval; once it stalls
          // (its rounding floor, or the slow late decay of the plastic zone) or passes
          // EITER, the state returns to FP64 and FP64 checkpoints take over.
          if (!(error < f32_drop * f32_prev) || error < prm.eiter) {
            rc = leave_f32();
            if (rc) return rc;
          }
          f32_prev = error;
          continue;
        }
        if (error < prm.eiter) {
          converged = 1;
          iters = iter;
          break;
        }
      }
    }
    if (f32) {  // niter not a multiple of check_every: still FP32 at the end
      rc = leave_f32();
      if (rc) return rc;
    }
    EP2D_CK(cudaEventRecord(ev_[1], stream));
    EP2D_CK(cudaEventSynchronize(ev_[1]));
    float ms = 0.0f;
    EP2D_CK(cudaEventElapsedTime(&ms, ev_[0], ev_[1]));
    kernel_ms += ms;
    cell_updates += iters * (int64_t)prm.nx * prm.ny;
    rc = check_resident();  // the last interval may end without a checkpoint
    if (rc) return rc;
    r.iterations = iters;
    r.converged = converged;
    r.error = error;
    rc = finish_time_step(step, it);
    if (rc) return rc;
  }
  return EP2D_OK;
}

int Rve::compute_eff_moduli(double init, const double lt[3], int n_time_steps, ep2d_result* out) {
  if (!lt) return fail(EP2D_ERR_ARG, "load_type is null");
  if (n_time_steps < 1) return fail(EP2D_ERR_ARG, "n_time_steps must be >= 1");
  // EffPlast2D.cu:182-184
  if (prm.nl > EP2D_MAX_NL) return fail(EP2D_ERR_ARG, "Wrong number of loads in ComputeEffModuli(): nl > 3");
  begin_chain(lt);
  for (int step = 0; step < prm.nl; step++) {
    double lsv, lts[3];
    int ns;
    step_load(step, init, lt, n_time_steps, &lsv, lts, &ns);
    const int rc = solve_step(step, lsv, lts, ns);
    if (rc) return rc;
  }
  finish_chain(n_time_steps, out);
  return EP2D_OK;
}

// The increments of ComputeEffDamping (EffPlast2D.cu:240-243): load_value times the
// difference of sin(i 2 pi' / (NL-1)) between consecutive steps, pi' = 3.1415926.
double Rve::damping_step_value(int step, int nl, double load_value) {
  return load_value * (std::sin(step * 2.0 * 3.1415926 / (nl - 1)) - std::sin((step - 1) * 2.0 * 3.1415926 / (nl - 1)));
}

int Rve::compute_eff_damping(double init, const double lt[3], int n_time_steps, double load_value,
                             int64_t* total_iterations) {
  if (!lt) return fail(EP2D_ERR_ARG, "load_type is null");
  if (n_time_steps < 1) return fail(EP2D_ERR_ARG, "n_time_steps must be >= 1");
  // EffPlast2D.cu:233-235
  if (prm.nl < 4) return fail(EP2D_ERR_ARG, "Wrong number of loads in ComputeEffDamping(): nl < 4");
  begin_chain(lt);
  int rc = solve_step(0, init, lt, n_time_steps);
  if (rc) return rc;
  for (int step = 1; step < prm.nl; step++) {
    rc = solve_step(step, damping_step_value(step, prm.nl, load_value), lt, 1);
    if (rc) return rc;
  }
  if (total_iterations) {
    int64_t tot = 0;
    for (int a = 0; a < prm.nl; a++)
      for (int t = 0; t < nts[a]; t++) tot += rec[a][t].iterations;
    *total_iterations = tot;
  }
  return EP2D_OK;
}

namespace {
void dims(int nx, int ny, int field, int* w, int* h) {
  switch (field) {
    case EP2D_FIELD_TAUXY: case EP2D_FIELD_J2XY: *w = nx - 1; *h = ny - 1; break;
    case EP2D_FIELD_UX: case EP2D_FIELD_VX: *w = nx + 1; *h = ny; break;
    case EP2D_FIELD_UY: case EP2D_FIELD_VY: *w = nx; *h = ny + 1; break;
    default: *w = nx; *h = ny;
  }
}
}  // namespace

int Rve::get_field(int field, double* host) const {
  if (!host || field < 0 || field >= EP2D_NFIELDS) return fail(EP2D_ERR_ARG, "bad field or null buffer");
  DeviceScope ds(device);
  int w, h;
  dims(prm.nx, prm.ny, field, &w, &h);
  const size_t pb = (size_t)g.pitch * sizeof(double);
  if (field == EP2D_FIELD_K || field == EP2D_FIELD_G) {
    std::vector<uint8_t> m((size_t)g.pitch * h);
    EP2D_CK(cudaMemcpyAsync(m.data(), f.mask, m.size(), cudaMemcpyDeviceToHost, stream));
    EP2D_CK(cudaStreamSynchronize(stream));
    const double base = field == EP2D_FIELD_K ? g.K0 : g.G0;
    const double pore = field == EP2D_FIELD_K ? g.Kp : g.Gp;
    for (int j = 0; j < h; j++)
      for (int i = 0; i < w; i++) host[(size_t)j * w + i] = (m[(size_t)j * g.pitch + i] & M_MAT) ? pore : base;
    return EP2D_OK;
  }
  const double* src = nullptr;
  switch (field) {
    case EP2D_FIELD_P: src = f.p; break;
    case EP2D_FIELD_TAUXX: src = f.txx; break;
    case EP2D_FIELD_TAUYY: src = f.tyy; break;
    case EP2D_FIELD_TAUXY: src = f.txy; break;
    case EP2D_FIELD_TAUXYAV: src = f.txyav; break;
    case EP2D_FIELD_J2: src = f.j2; break;
    case EP2D_FIELD_J2XY: src = f.j2xy; break;
    case EP2D_FIELD_UX: src = f.ux[cur]; break;
    case EP2D_FIELD_UY: src = f.uy[cur]; break;
    case EP2D_FIELD_VX: src = static_cast<const double*>(f.vx); break;
    case EP2D_FIELD_VY: src = static_cast<const double*>(f.vy); break;
  }
  if (mixed() && (field == EP2D_FIELD_VX || field == EP2D_FIELD_VY)) {  // float storage
    std::vector<float> tmp((size_t)w * h);
    EP2D_CK(cudaMemcpy2DAsync(tmp.data(), (size_t)w * sizeof(float), field == EP2D_FIELD_VX ? f.vx : f.vy,
                              (size_t)g.pitch * sizeof(float), (size_t)w * sizeof(float), h, cudaMemcpyDeviceToHost,
                              stream));
    EP2D_CK(cudaStreamSynchronize(stream));
    for (size_t k = 0; k < tmp.size(); k++) host[k] = tmp[k];
    return EP2D_OK;
  }
  EP2D_CK(cudaMemcpy2DAsync(host, (size_t)w * sizeof(double), src, pb, (size_t)w * sizeof(double), h,
                            cudaMemcpyDeviceToHost, stream));
  EP2D_CK(cudaStreamSynchronize(stream));
  return EP2D_OK;
}

int Rve::set_field(int field, const double* host) {
  if (!host || field < 0 || field >= EP2D_NFIELDS) return fail(EP2D_ERR_ARG, "bad field or null buffer");
  if (field == EP2D_FIELD_K || field == EP2D_FIELD_G)
    return fail(EP2D_ERR_ARG, "K and G follow from the pore geometry and cannot be set");
  DeviceScope ds(device);
  int w, h;
  dims(prm.nx, prm.ny, field, &w, &h);
  const size_t pb = (size_t)g.pitch * sizeof(double);
  double* dst[2] = {nullptr, nullptr};
  switch (field) {
    case EP2D_FIELD_P: dst[0] = f.p; break;
    case EP2D_FIELD_TAUXX: dst[0] = f.txx; break;
    case EP2D_FIELD_TAUYY: dst[0] = f.tyy; break;
    case EP2D_FIELD_TAUXY: dst[0] = f.txy; break;
    case EP2D_FIELD_TAUXYAV: dst[0] = f.txyav; break;
    case EP2D_FIELD_J2: dst[0] = f.j2; break;
    case EP2D_FIELD_J2XY: dst[0] = f.j2xy; break;
    case EP2D_FIELD_UX: dst[0] = f.ux[0]; dst[1] = f.ux[1]; break;
    case EP2D_FIELD_UY: dst[0] = f.uy[0]; dst[1] = f.uy[1]; break;
    case EP2D_FIELD_VX: dst[0] = static_cast<double*>(f.vx); break;
    case EP2D_FIELD_VY: dst[0] = static_cast<double*>(f.vy); break;
  }
  if (mixed() && (field == EP2D_FIELD_VX || field == EP2D_FIELD_VY)) {  // float storage
    std::vector<float> tmp((size_t)w * h);
    for (size_t k = 0; k < tmp.size(); k++) tmp[k] = (float)host[k];
    EP2D_CK(cudaMemcpy2DAsync(field == EP2D_FIELD_VX ? f.vx : f.vy, (size_t)g.pitch * sizeof(float), tmp.data(),
                              (size_t)w * sizeof(float), (size_t)w * sizeof(float), h, cudaMemcpyHostToDevice, stream));
    EP2D_CK(cudaStreamSynchronize(stream));
    return EP2D_OK;
  }
  for (double* dp : dst)
    if (dp)
      EP2D_CK(cudaMemcpy2DAsync(dp, pb, host, (size_t)w * sizeof(double), (size_t)w * sizeof(double), h,
                                cudaMemcpyHostToDevice, stream));
  EP2D_CK(cudaStreamSynchronize(stream));
  return EP2D_OK;
}

int Rve::static_fields(double* unu, double* j1, double* j2) {
  if (!unu || !j1 || !j2) return fail(EP2D_ERR_ARG, "null output buffer");
  DeviceScope ds(device);
  const size_t nn = (size_t)prm.nx * prm.ny, nc = (size_t)(prm.nx - 1) * (prm.ny - 1);
  double* tmp = nullptr;
  EP2D_CK(cudaMallocAsync(&tmp, (nn + 2 * nc) * sizeof(double), stream));
  cudaError_t e = launch_static_fields(g, f, cur, tmp, tmp + nn, tmp + nn + nc, stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(unu, tmp, nn * sizeof(double), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(j1, tmp + nn, nc * sizeof(double), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(j2, tmp + nn + nc, nc * sizeof(double), cudaMemcpyDeviceToHost, stream);
  cudaFreeAsync(tmp, stream);
  cudaError_t se = cudaStreamSynchronize(stream);
  if (e != cudaSuccess || se != cudaSuccess)
    return fail(EP2D_ERR_CUDA, std::string("static fields: ") + cudaGetErrorString(e != cudaSuccess ? e : se));
  return EP2D_OK;
}

int Rve::polar_fields(double load_value, double* snrr, double* snff, double* sarr, double* saff, uint8_t* plast) {
  if (!snrr || !snff || !sarr || !saff || !plast) return fail(EP2D_ERR_ARG, "null output buffer");
  DeviceScope ds(device);
  const size_t nn = (size_t)prm.nx * prm.ny;
  // sign(loadValue), get_sigma_2D.m:175 (MATLAB sign: 0 for 0)
  const double sgn = load_value > 0.0 ? 1.0 : (load_value < 0.0 ? -1.0 : 0.0);
  double* tmp = nullptr;
  EP2D_CK(cudaMallocAsync(&tmp, 4 * nn * sizeof(double) + nn, stream));
  uint8_t* pl = reinterpret_cast<uint8_t*>(tmp + 4 * nn);
  cudaError_t e = launch_polar_fields(g, f, sgn, tmp, tmp + nn, tmp + 2 * nn, tmp + 3 * nn, pl, tracked, stream);
  double* outs[4] = {snrr, snff, sarr, saff};
  for (int k = 0; k < 4 && e == cudaSuccess; k++)
    e = cudaMemcpyAsync(outs[k], tmp + k * nn, nn * sizeof(double), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(plast, pl, nn, cudaMemcpyDeviceToHost, stream);
  cudaFreeAsync(tmp, stream);
  cudaError_t se = cudaStreamSynchronize(stream);
  if (e != cudaSuccess || se != cudaSuccess)
    return fail(EP2D_ERR_CUDA, std::string("polar fields: ") + cudaGetErrorString(e != cudaSuccess ? e : se));
  aux_launches += 1;
  return EP2D_OK;
}

int Rve::analytic_fields(double deltaP, double tauInfty, double* uan, double* eu, double* j1an, double* j2an,
                         double* ej1, double* ej2, double stats[6]) {
  if (!uan || !eu || !j1an || !j2an || !ej1 || !ej2 || !stats) return fail(EP2D_ERR_ARG, "null output buffer");
  DeviceScope ds(device);
  // scalars, EffPlast2D.cu:1062-1078, in host arithmetic
  AnParams a{};
  a.deltaP = deltaP;
  a.tauInfty = tauInfty;
  a.Y = d.Y;
  a.rad = d.rad;
  a.G0 = d.G0;
  a.K0 = d.K0;
  a.hydro = (std::abs(load_type_[0] - load_type_[1]) < std::numeric_limits<double>::epsilon()) &&
            std::abs(load_type_[2]) < std::numeric_limits<double>::epsilon();
  a.Rmin = d.rad;
  a.Rmax = 0.5 * d.dX * (prm.nx - 1) - d.dX * 20.0;
  a.eps = 1.0e-18;
  a.xi = (deltaP > 0.0) ? 1.0 : -1.0;
  a.kappa = tauInfty / d.Y * a.xi;
  a.c0 = d.rad * std::exp(std::abs(deltaP) / 2.0 / d.Y - 0.5);
  a.rx = d.rad + (-0.5 * d.Y * d.rad * d.rad * std::exp((deltaP - d.Y) / d.Y) / (d.G0 * d.rad));
  a.ry = a.rx;
  a.Rx = a.c0 * (1.0 - a.kappa);
  a.Ry = a.c0 * (1.0 + a.kappa);
  const size_t nn = (size_t)prm.nx * prm.ny, nc = (size_t)(prm.nx - 1) * (prm.ny - 1);
  const size_t nst = (size_t)ANALYTIC_BLOCKS * 8;
  double* tmp = nullptr;
  EP2D_CK(cudaMallocAsync(&tmp, (3 * nn + 6 * nc + nst) * sizeof(double), stream));
  double* unu = tmp;
  double* j1nu = unu + nn;
  double* j2nu = j1nu + nc;
  double* d_uan = j2nu + nc;
  double* d_eu = d_uan + nn;
  double* d_j1 = d_eu + nn;
  double* d_j2 = d_j1 + nc;
  double* d_e1 = d_j2 + nc;
  double* d_e2 = d_e1 + nc;
  double* d_st = d_e2 + nc;
  std::vector<double> st(nst);
  cudaError_t e = launch_static_fields(g, f, cur, unu, j1nu, j2nu, stream);
  if (e == cudaSuccess) e = launch_analytic(g, a, unu, j1nu, j2nu, d_uan, d_eu, d_j1, d_j2, d_e1, d_e2, d_st, stream);
  struct {
    double* h;
    const double* dd;
    size_t n;
  } cp[] = {{uan, d_uan, nn}, {eu, d_eu, nn}, {j1an, d_j1, nc}, {j2an, d_j2, nc}, {ej1, d_e1, nc}, {ej2, d_e2, nc},
            {st.data(), d_st, nst}};
  for (auto& c : cp)
    if (e == cudaSuccess) e = cudaMemcpyAsync(c.h, c.dd, c.n * sizeof(double), cudaMemcpyDeviceToHost, stream);
  cudaFreeAsync(tmp, stream);
  cudaError_t se = cudaStreamSynchronize(stream);
  if (e != cudaSuccess || se != cudaSuccess)
    return fail(EP2D_ERR_CUDA, std::string("analytic fields: ") + cudaGetErrorString(e != cudaSuccess ? e : se));
  double umax = 0, usum = 0, un = 0, j1max = 0, j1sum = 0, j2max = 0, j2sum = 0, jn = 0;
  for (int b = 0; b < ANALYTIC_BLOCKS; b++) {
    const double* v = &st[(size_t)b * 8];
    umax = std::max(umax, v[0]);
    usum += v[1];
    un += v[2];
    j1max = std::max(j1max, v[3]);
    j1sum += v[4];
    j2max = std::max(j2max, v[5]);
    j2sum += v[6];
    jn += v[7];
  }
  stats[0] = umax;
  stats[1] = usum / un;
  stats[2] = j1max;
  stats[3] = j1sum / jn;
  stats[4] = j2max;
  stats[5] = j2sum / jn;
  return EP2D_OK;
}

}  // namespace ep2d
