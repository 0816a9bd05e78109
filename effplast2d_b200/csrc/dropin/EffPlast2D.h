// EffPlast2D.h -- drop-in replacement for the reference's class header.
//
// Same public interface as beacon1143/EffPlast2D's EffPlast2D.h:53-65 and the same
// compile-time macros (EffPlast2D.h:17-39), so the reference's main.cu and the
// eff_props_2D.m build line keep working.  The work is done by libep2d (include/ep2d.h):
// B200 kernels behind a C ABI.  Outputs (stdout, EffPlast2D.log, data/*.dat) follow the
// reference line by line.
#ifndef EP2D_DROPIN_EFFPLAST2D_H
#define EP2D_DROPIN_EFFPLAST2D_H

#include <array>
#include <cmath>
#include <fstream>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "ep2d.h"

#if !defined(NGRID)
#define NGRID 32
#endif

#if !defined(NPARS)
#define NPARS 11
#endif

#if !defined(NL)
#define NL 3
#endif

#if !defined(NITER)
#define NITER 100'000
#endif

#if !defined(EITER)
#define EITER 1.0e-10
#endif

#if !defined(DEVICE_IDX)
#define DEVICE_IDX 0
#endif

class EffPlast2D {
 public:
  double ComputeEffModuli(double initLoadValue, const std::array<double, 3>& loadType, double loadValue = 0.0);
  double ComputeEffDamping(double initLoadValue, const std::array<double, 3>& loadType, double loadValue = 0.0);

  EffPlast2D(const unsigned int nTimeSteps = 1);
  ~EffPlast2D();

 private:
  void Check(int status, int line);  // gpuErrchk's role (EffPlast2D.h:41-49)
  void ComputeEffParams(size_t step, size_t nTimeSteps);
  void SaveAnStatic2D(double deltaP, double tauInfty);
  void SaveField(int field, const std::string& filename);

  void printStepInfo(size_t step);
  void printCalculationType();
  void printEffectiveModuli();
  void printWarnings();
  void printDuration(int elapsed_sec);
  void both(const std::string& s);  // to std::cout and the log file

  ep2d_handle* h_ = nullptr;
  ep2d_params prm_{};
  unsigned int nTimeSteps_;
  std::array<double, 3> loadType_{};
  long nX, nY;
  double Y, porosity, nPores;
  std::ofstream log_file;
  ep2d_result res_{};
};

#endif
