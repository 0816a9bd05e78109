// EffPlast2D.cu -- drop-in implementation of the reference's EffPlast2D class on top of
// the libep2d C ABI.  Control flow, messages and output files follow the reference's
// EffPlast2D.cu (constructor :1541-1612, ComputeEffModuli :179-229, ComputeEffDamping
// :230-310, ComputeEffParams
// printing :311-698, SaveAnStatic2D output :1060-1292, print* :1295-1409, calc* logging
// :1412-1454); the numerics run in libep2d on the GPU.
//
// Build (link): nvcc -gencode arch=compute_100a,code=sm_100a -D... -I<repo>/include
//               EffPlast2D.cu main.cu -L<repo>/effplast2d_b200 -lep2d
// Build (self-contained, the reference's own command line plus -DEP2D_UNITY):
//               nvcc -O3 -gencode arch=compute_100a,code=sm_100a -DEP2D_UNITY -D...
//               -I<repo>/include -I<repo>/effplast2d_b200/csrc EffPlast2D.cu main.cu
#include "EffPlast2D.h"

#include <chrono>
#include <cstdlib>
#include <limits>

#if defined(EP2D_UNITY)
#include "ep2d_kernels.cu"
#include "ep2d_rve.cpp"
#include "ep2d_api.cpp"
#endif

namespace {
template <class... T>
void to_both(std::ostream& a, std::ostream& b, const T&... v) {
  (a << ... << v);
  (b << ... << v);
}
}  // namespace

void EffPlast2D::both(const std::string& s) { to_both(std::cout, log_file, s); }

void EffPlast2D::Check(int status, int line) {
  if (status == EP2D_OK) return;
  const std::string msg = ep2d_last_error();
  if (status == EP2D_ERR_CUDA || status == EP2D_ERR_NODEV || status == EP2D_ERR_NOMEM) {
    // gpuErrchk: print and exit(-1) (EffPlast2D.h:41-49)
    std::cout << "[" + std::string(__FILE__) + ":" + std::to_string(line) + "] " + "CUDA error: " + msg;
    std::exit(-1);
  }
  if (status == EP2D_ERR_IO) throw std::runtime_error(msg + "\n");
  throw std::invalid_argument("ERROR:  " + msg + "\n");
}

EffPlast2D::EffPlast2D(const unsigned int nTimeSteps) : nTimeSteps_(nTimeSteps) {
  nX = 32 * NGRID;  // block 32 x grid NGRID (EffPlast2D.cu:1544-1552)
  nY = 32 * NGRID;
  prm_.nx = static_cast<int32_t>(nX);
  prm_.ny = static_cast<int32_t>(nY);
  prm_.nl = NL;
  prm_.niter = NITER;
  prm_.eiter = EITER;
  prm_.check_every = 10'000;  // output_step (EffPlast2D.cu:1608)
  prm_.precision = EP2D_FP64;
  prm_.device = DEVICE_IDX;
  Check(ep2d_read_pa("data/pa.dat", prm_.pa), __LINE__);
  const double dX = prm_.pa[0], dY = prm_.pa[1];
  const double rad = prm_.pa[9];
  Y = prm_.pa[8] / std::sqrt(2.0);
  nPores = prm_.pa[10];
  Check(ep2d_create(&prm_, &h_), __LINE__);
  log_file.open("EffPlast2D.log", std::ios_base::app);
  const double lX = (nX - 1) * dX;
  const double lY = (nY - 1) * dY;
  porosity = 3.1415926 * rad * rad * nPores * nPores / (lX * lY);
}

EffPlast2D::~EffPlast2D() {
  if (h_) ep2d_destroy(h_);
  log_file.close();
}

double EffPlast2D::ComputeEffModuli(const double initLoadValue, const std::array<double, 3>& loadType,
                                    const double /*loadValue: unused, as in the reference*/) {
  if (NL > 3) throw std::invalid_argument("ERROR:  Wrong number of loads in ComputeEffModuli()!\n");
  const auto start = std::chrono::system_clock::now();
  loadType_ = loadType;
  printCalculationType();
  Check(ep2d_compute_eff_moduli(h_, initLoadValue, loadType_.data(), static_cast<int32_t>(nTimeSteps_), &res_),
        __LINE__);
  // the reference interleaves these lines with the solves; their content and order
  // in stdout and EffPlast2D.log are the same
  ComputeEffParams(0, nTimeSteps_);
  if (NL == 1) {  // calcBulkModuli_PureElast (EffPlast2D.cu:1412-1428)
    log_file << "    ==============\n" << "    Kphi = " << res_.num.kphi << std::endl;
    log_file << "    KphiPer = " << res_.num_per.kphi << "\n";
    log_file << "    Kd = " << res_.num.kd << "\n";
    log_file << "    KdPer = " << res_.num_per.kd << "\n";
  } else {
    ComputeEffParams(1, 1);
    // calcBulkModuli_ElastPlast (EffPlast2D.cu:1429-1445)
    log_file << "==============\n" << "    Kphi = " << res_.num.kphi << std::endl;
    log_file << "    KphiPer = " << res_.num_per.kphi << "\n";
    log_file << "    Kd = " << res_.num.kd << "\n";
    log_file << "    KdPer = " << res_.num_per.kd << "\n";
  }
  if (NL == 3) {
    ComputeEffParams(2, 1);
    // calcShearModulus (EffPlast2D.cu:1446-1454)
    log_file << "==============\n" << "    G = " << res_.num.g << "\n";
    log_file << "    Gper = " << res_.num_per.g << "\n";
  }
  printEffectiveModuli();
  printWarnings();
  if (NL > 1 && nTimeSteps_) {
    ep2d_step_record r{};
    Check(ep2d_get_record(h_, 0, nTimeSteps_ - 1, &r), __LINE__);
    SaveAnStatic2D(r.delta_p, r.tau_infty);
  }
  SaveField(EP2D_FIELD_P, "data/Pc_" + std::to_string(32 * NGRID) + "_.dat");
  SaveField(EP2D_FIELD_TAUXX, "data/tauXXc_" + std::to_string(32 * NGRID) + "_.dat");
  const auto end = std::chrono::system_clock::now();
  const int elapsed_sec = static_cast<int>(std::chrono::duration_cast<std::chrono::seconds>(end - start).count());
  printDuration(elapsed_sec);
  return 0.0;
}

// ComputeEffDamping (EffPlast2D.cu:230-310): the preload, NL-1 sinusoidal increments of
// loadValue along loadType, the strain and stress tensors of every step on stdout, the
// static fields.  The reference never assigns loadType_ on this path, so its
// SaveAnStatic2D there reads an uninitialised array to choose the analytic branch
// (EffPlast2D.h:81, EffPlast2D.cu:1062-1064); here the load type of the call decides.
// With nPores > 1 (no analytic fields) the outputs do not depend on that choice.
double EffPlast2D::ComputeEffDamping(const double initLoadValue, const std::array<double, 3>& loadType,
                                     const double loadValue) {
  if (NL < 4) throw std::invalid_argument("ERROR:  Wrong number of loads in ComputeEffModuli()!\n");
  const auto start = std::chrono::system_clock::now();
  printCalculationType();
  int64_t total = 0;
  Check(ep2d_compute_eff_damping(h_, initLoadValue, loadType.data(), static_cast<int32_t>(nTimeSteps_), loadValue,
                                 &total),
        __LINE__);
  ComputeEffParams(0, nTimeSteps_);
  for (size_t i = 1; i < NL; i++) ComputeEffParams(i, 1);
  // the record of step i's tensor: (0, nTimeSteps-1) for the preload, (i, 0) after it
  auto rec = [this](size_t i) {
    ep2d_step_record r{};
    Check(ep2d_get_record(h_, static_cast<int32_t>(i), i == 0 ? static_cast<int32_t>(nTimeSteps_) - 1 : 0, &r),
          __LINE__);
    return r;
  };
  auto table = [&](const char* title, int n, auto get) {
    std::cout << title;
    for (size_t i = 0; i < NL; i++) {
      std::cout << i << ") ";
      const ep2d_step_record r = rec(i);
      for (int j = 0; j < n; j++) std::cout << get(r)[j] << " ";
      std::cout << "\n";
    }
  };
  table("\nStrain tensors:\n", 3, [](const ep2d_step_record& r) { return r.macro_strain; });
  table("\nStrain tensors periodic:\n", 3, [](const ep2d_step_record& r) { return r.eps_per; });
  table("\nStress tensors:\n", 4, [](const ep2d_step_record& r) { return r.sigma; });
  table("\nStress tensors periodic:\n", 4, [](const ep2d_step_record& r) { return r.sigma_per; });
  if (nTimeSteps_ > 0) {
    const ep2d_step_record r0 = rec(0);
    SaveAnStatic2D(r0.delta_p, r0.tau_infty);
  }
  const auto end = std::chrono::system_clock::now();
  const int elapsed_sec = static_cast<int>(std::chrono::duration_cast<std::chrono::seconds>(end - start).count());
  printDuration(elapsed_sec);
  return 0.0;
}

// The printing of ComputeEffParams (EffPlast2D.cu:311-698) from the step's records.
void EffPlast2D::ComputeEffParams(const size_t step, const size_t nTimeSteps) {
  printStepInfo(step);
  for (size_t it = 0; it < nTimeSteps; it++) {
    ep2d_step_record r{};
    Check(ep2d_get_record(h_, static_cast<int32_t>(step), static_cast<int32_t>(it), &r), __LINE__);
    to_both(std::cout, log_file, "Time step ", it + 1, " from ", nTimeSteps, "\n");
    to_both(std::cout, log_file, "Macro strain: (", r.macro_strain[0], ", ", r.macro_strain[1], ", ",
            r.macro_strain[2], ")\n");
    std::vector<double> errs(r.n_checks > 0 ? r.n_checks : 1);
    int32_t n = 0;
    Check(ep2d_get_check_errors(h_, static_cast<int32_t>(step), static_cast<int32_t>(it), errs.data(),
                                static_cast<int32_t>(errs.size()), &n),
          __LINE__);
    for (int32_t k = 0; k < n; k++) {
      const long iter1 = static_cast<long>(k + 1) * prm_.check_every;
      std::cout << "    Iteration " << iter1 << ": Error is " << errs[k] << std::endl;
      log_file << "    Iteration " << iter1 << ": Error is " << errs[k] << std::endl;
      if (k == n - 1) {
        if (r.converged) {
          to_both(std::cout, log_file, "Number of iterations is ", iter1, "\n\n");
        } else if (iter1 >= prm_.niter) {
          to_both(std::cout, log_file, "WARNING: Maximum number of iterations reached!\nError is ", errs[k], "\n\n");
        }
      }
    }
    log_file << "    dPhi = " << r.dphi << '\n';
    if (nPores > 2) log_file << "    dPhiPer = " << r.dphi_per << '\n';
    to_both(std::cout, log_file, "    P / Y = ", r.delta_p / Y, '\n');
    if (nPores > 2) to_both(std::cout, log_file, "    Pper / Y = ", r.delta_p_per / Y, '\n');
    to_both(std::cout, log_file, "    tau / Y = ", r.tau_infty / Y, '\n');
    if (NL <= 1) {
      log_file << "    KphiExactElast = " << r.kphi_exact_elast << '\n';
      log_file << "    KdExactElast = " << r.kd_exact_elast << '\n';
    } else if (step == 0) {
      log_file << "    KphiExactPlast = " << r.kphi_exact_plast << '\n';
      log_file << "    KdExactPlast = " << r.kd_exact_plast << '\n';
      log_file << "    KphiExactPlastPer = " << r.kphi_exact_plast_per << '\n';
      log_file << "    KdExactPlastPer = " << r.kd_exact_plast_per << '\n';
    }
    if (NL == 3 && step == 0) {
      log_file << "    GexactElast = " << r.g_exact_elast << '\n';
      log_file << "    GexactPlast = " << r.g_exact_plast << '\n';
      log_file << "    GexactPlastPer = " << r.g_exact_plast_per << '\n';
    }
  }
}

void EffPlast2D::SaveField(int field, const std::string& filename) {
  int32_t w = 0, h = 0;
  Check(ep2d_field_dims(prm_.nx, prm_.ny, field, &w, &h), __LINE__);
  std::vector<double> buf(static_cast<size_t>(w) * h);
  Check(ep2d_get_field(h_, field, buf.data()), __LINE__);
  std::ofstream f(filename, std::ios_base::binary);
  f.write(reinterpret_cast<const char*>(buf.data()), sizeof(double) * buf.size());
}

// SaveAnStatic2D (EffPlast2D.cu:1060-1292): numerical fields always, analytic fields,
// error maps and error statistics for a single pore.
void EffPlast2D::SaveAnStatic2D(const double deltaP, const double tauInfty) {
  const size_t nn = static_cast<size_t>(nX) * nY, nc = static_cast<size_t>(nX - 1) * (nY - 1);
  const std::string sfx = "_" + std::to_string(32 * NGRID) + "_.dat";
  auto save = [](const std::vector<double>& v, const std::string& name) {
    std::ofstream f(name, std::ios_base::binary);
    f.write(reinterpret_cast<const char*>(v.data()), sizeof(double) * v.size());
  };
  if (nPores == 1) {
    std::vector<double> uan(nn), eu(nn), j1(nc), j2(nc), e1(nc), e2(nc);
    double st[6];
    Check(ep2d_analytic_fields(h_, deltaP, tauInfty, uan.data(), eu.data(), j1.data(), j2.data(), e1.data(), e2.data(),
                               st),
          __LINE__);
    std::cout << "\n"
              << "Uabs max error  = " << st[0] << ", avg = " << st[1] << '\n'
              << "J1 max error = " << st[2] << ", avg = " << st[3] << '\n'
              << "J2 max error = " << st[4] << ", avg = " << st[5] << std::endl;
    log_file << "\n"
             << "Uabs max error  = " << st[0] << ", avg = " << st[1] << '\n'
             << "J1 max error = " << st[2] << ", avg = " << st[3] << '\n'
             << "J2 max error = " << st[4] << ", avg = " << st[5] << std::endl;
    save(uan, "data/UanAbs" + sfx);
    save(eu, "data/errorUabs" + sfx);
    save(j1, "data/J1an" + sfx);
    save(j2, "data/J2an" + sfx);
    save(e1, "data/errorJ1" + sfx);
    save(e2, "data/errorJ2" + sfx);
  }
  std::vector<double> unu(nn), j1nu(nc), j2nu(nc);
  Check(ep2d_static_fields(h_, unu.data(), j1nu.data(), j2nu.data()), __LINE__);
  save(unu, "data/UnuAbs" + sfx);
  save(j1nu, "data/J1nu" + sfx);
  save(j2nu, "data/J2nu" + sfx);
}

// ---- console and log output, EffPlast2D.cu:1295-1409 --------------------------------
void EffPlast2D::printStepInfo(const size_t step) {
  to_both(std::cout, log_file, "\nLOAD STEP ", step + 1, " FROM ", NL, ": ");
  if (NL <= 3) {
    switch (step) {
      case 0: both("PRELOADING\n"); break;
      case 1: both("SMALL HYDROSTATIC INCREMENT\n"); break;
      case 2: both("SMALL DEVIATORIC INCREMENT\n"); break;
      default: throw std::invalid_argument("ERROR:  Wrong step index!\n");
    }
  }
  to_both(std::cout, log_file, "Porosity is ", porosity * 100, "%\n");
  to_both(std::cout, log_file, "Grid resolution is ", nX, "x", nY, "\n\n");
}

void EffPlast2D::printCalculationType() {
  switch (NL) {
    case 1: both("\nPURE ELASTIC CALCULATION\nESTIMATION OF THE EFFECTIVE BULK MODULI\n"); break;
    case 2: both("\nELASTOPLASTIC CALCULATION\nESTIMATION OF THE EFFECTIVE BULK MODULI\n"); break;
    case 3:
      both("\nELASTOPLASTIC CALCULATION\nESTIMATION OF THE EFFECTIVE BULK MODULI AND THE EFFECTIVE SHEAR MODULUS\n");
      break;
    default: both("\nELASTOPLASTIC CALCULATION\nESTIMATION OF THE EFFECTIVE DAMPING\n");
  }
}

void EffPlast2D::printEffectiveModuli() {
  auto output = [this](const ep2d_moduli& m) {  // EffModuli::output, EffPlast2D.h:124-133
    to_both(std::cout, log_file, "        Kphi = ", m.kphi, "\n");
    to_both(std::cout, log_file, "        Kd = ", m.kd, "\n");
    if (NL > 2) to_both(std::cout, log_file, "        G = ", m.g, "\n");
  };
  both("\nEFFECTIVE MODULI ESTIMATED\nNON-PERIODIC\n    Analytical:\n");
  output(res_.an);
  both("    Numerical:\n");
  output(res_.num);
  if (nPores > 2) {
    both("PERIODIC\n    Analytical:\n");
    output(res_.an_per);
    both("    Numerical:\n");
    output(res_.num_per);
  }
}

void EffPlast2D::printWarnings() {
  if (NL > 1) {
    ep2d_step_record r{};
    Check(ep2d_get_record(h_, 0, nTimeSteps_ - 1, &r), __LINE__);
    if (std::abs(r.delta_p) / Y < 1.0 || std::abs(r.delta_p) / Y > 5.0 || std::abs(r.tau_infty) / Y > 0.42) {
      both("\nWARNING:  Analytical solution is not applicable for this load!\n");
      both("TODO: Set the load so that 1 < |P|/Y < 5 and 0 < |tau|/Y < 0.42\n");
    }
    if (std::abs(loadType_[0] - loadType_[1]) > 0.05 * std::max(std::abs(loadType_[0]), std::abs(loadType_[1])) ||
        std::abs(loadType_[2]) > 0.01 * std::max(std::abs(loadType_[0]), std::abs(loadType_[1]))) {
      both("\nWARNING:  The numerical effective Kphi is not calculated quite accurately for non-hydrostatic load!\n");
    }
  }
}

void EffPlast2D::printDuration(int elapsed_sec) {
  if (elapsed_sec < 60) {
    std::cout << "\nCalculation time is " << elapsed_sec << " sec\n";
    log_file << "\nCalculation time is " << elapsed_sec << " sec\n\n\n";
    return;
  }
  int elapsed_min = elapsed_sec / 60;
  elapsed_sec = elapsed_sec % 60;
  if (elapsed_min < 60) {
    std::cout << "\nCalculation time is " << elapsed_min << " min " << elapsed_sec << " sec\n";
    log_file << "\nCalculation time is " << elapsed_min << " min " << elapsed_sec << " sec\n\n\n";
    return;
  }
  int elapsed_hour = elapsed_min / 60;
  elapsed_min = elapsed_min % 60;
  if (elapsed_hour < 24) {
    std::cout << "\nCalculation time is " << elapsed_hour << " hours " << elapsed_min << " min " << elapsed_sec << " sec\n";
    log_file << "\nCalculation time is " << elapsed_hour << " hours " << elapsed_min << " min " << elapsed_sec
             << " sec\n\n\n";
    return;
  }
  const int elapsed_day = elapsed_hour / 24;
  elapsed_hour = elapsed_hour % 24;
  if (elapsed_day < 7) {
    std::cout << "\nCalculation time is " << elapsed_day << " days " << elapsed_hour << " hours " << elapsed_min
              << " min " << elapsed_sec << " sec\n";
    log_file << "\nCalculation time is " << elapsed_day << " days " << elapsed_hour << " hours " << elapsed_min
             << " min " << elapsed_sec << " sec\n\n\n";
  } else {
    std::cout << "\nCalculation time is " << elapsed_day / 7 << " weeks " << elapsed_day % 7 << " days "
              << elapsed_hour << " hours " << elapsed_min << " min " << elapsed_sec << " sec\n";
    log_file << "\nCalculation time is " << elapsed_day / 7 << " weeks " << elapsed_day % 7 << " days "
             << elapsed_hour << " hours " << elapsed_min << " min " << elapsed_sec << " sec\n\n\n";
  }
}
