// ref_harness.cu -- TEST INFRASTRUCTURE: a driver for the UNMODIFIED reference.
//
// Linked (relocatable device code, as the reference's CMakeLists.txt:12 asks) with the
// reference's own EffPlast2D.cu, compiled from where it lies; nothing of the reference
// is copied here.  It makes the reference's internal state observable at full
// precision so that the CPU oracle can be pinned against it:
//
//   kernels <in_dir> <out_dir> <nx> <ny> <nl> <iters>
//       Loads pa.bin (11 doubles) and K,G,Ux,Uy,Vx,Vy .bin fields (reference layout)
//       from in_dir, runs `iters` iterations of the reference's kernel sequence
//       ComputeStress -> [ComputeJ2 -> ComputePlasticity] -> ComputeDisp exactly as
//       EffPlast2D.cu:389-399 launches it (grid nx/32 x ny/32, block 32x32, a device
//       synchronisation after each launch) and writes every field to out_dir.
//   moduli <out_dir> <initLoad> <lt.x> <lt.y> <lt.xy> <nTimeSteps> <loadValue>
//       Runs EffPlast2D(nTimeSteps).ComputeEffModuli(...) (ComputeEffDamping(...) when the
//       build's NL > 3, as the reference's main.cu:32-37 chooses) in the current directory
//       (which must hold data/pa.dat), then writes the per-step records and the
//       effective moduli at 17 significant digits (records.txt) and every device
//       field (*.bin) to out_dir.
//
// The class's members are private; they are read through a `private` -> `public`
// macro applied only to the reference header, after every standard header has been
// included.  All data members of EffPlast2D sit in one access section, so the object
// layout is unchanged.
#include <array>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <limits>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include <device_launch_parameters.h>

#define private public
#include "EffPlast2D.h"
#undef private

__global__ void ComputeDisp(double* Ux, double* Uy, double* Vx, double* Vy, const double* const P,
                            const double* const tauXX, const double* const tauYY, const double* const tauXY,
                            const double* const pa, const long int nX, const long int nY);
__global__ void ComputeStress(const double* const Ux, const double* const Uy, const double* const K,
                              const double* const G, const double* const P0, double* P, double* tauXX,
                              double* tauYY, double* tauXY, const double* const pa, const long int nX,
                              const long int nY);
__global__ void ComputeJ2(double* tauXX, double* tauYY, double* tauXY, double* const tauXYav, double* const J2,
                          double* const J2XY, const long int nX, const long int nY);
__global__ void ComputePlasticity(double* tauXX, double* tauYY, double* tauXY, double* const tauXYav,
                                  double* const J2, double* const J2XY, const double* const pa, const long int nX,
                                  const long int nY);

static void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    std::fprintf(stderr, "CUDA error at %s: %s\n", what, cudaGetErrorString(e));
    std::exit(2);
  }
}

static std::vector<double> read_bin(const std::string& path, size_t n) {
  std::vector<double> v(n, 0.0);
  std::ifstream f(path, std::ios::binary);
  if (!f) {
    std::fprintf(stderr, "cannot open %s\n", path.c_str());
    std::exit(3);
  }
  f.read(reinterpret_cast<char*>(v.data()), sizeof(double) * n);
  if (static_cast<size_t>(f.gcount()) != sizeof(double) * n) {
    std::fprintf(stderr, "short read %s\n", path.c_str());
    std::exit(3);
  }
  return v;
}

static void write_bin(const std::string& path, const double* p, size_t n) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(p), sizeof(double) * n);
}

static void dump_dev(const std::string& path, const double* d, size_t n) {
  std::vector<double> h(n);
  check(cudaMemcpy(h.data(), d, sizeof(double) * n, cudaMemcpyDeviceToHost), path.c_str());
  write_bin(path, h.data(), n);
}

static int run_kernels(int argc, char** argv) {
  if (argc < 8) return 1;
  const std::string in = argv[2], out = argv[3];
  const long nX = std::atol(argv[4]), nY = std::atol(argv[5]);
  const int nl = std::atoi(argv[6]);
  const long iters = std::atol(argv[7]);
  if (nX % 32 || nY % 32 || nX < 32 || nY < 32) {
    std::fprintf(stderr, "nx, ny must be multiples of 32 (the reference has no bounds guard)\n");
    return 1;
  }
  const size_t nn = nX * nY, nc = (nX - 1) * (nY - 1), nux = (nX + 1) * nY, nuy = nX * (nY + 1);
  std::vector<double> pa = read_bin(in + "/pa.bin", 11);
  struct F { const char* name; size_t n; bool load; double* d; } f[] = {
      {"P", nn, false, nullptr},    {"tauXX", nn, false, nullptr}, {"tauYY", nn, false, nullptr},
      {"tauXY", nc, false, nullptr}, {"tauXYav", nn, false, nullptr}, {"J2", nn, false, nullptr},
      {"J2XY", nc, false, nullptr},  {"Ux", nux, true, nullptr},     {"Uy", nuy, true, nullptr},
      {"Vx", nux, true, nullptr},    {"Vy", nuy, true, nullptr},     {"K", nn, true, nullptr},
      {"G", nn, true, nullptr},      {"P0", nn, false, nullptr}};
  for (auto& x : f) {
    check(cudaMalloc(&x.d, sizeof(double) * x.n), "malloc");
    check(cudaMemset(x.d, 0, sizeof(double) * x.n), "memset");
    if (x.load) {
      std::vector<double> h = read_bin(in + "/" + x.name + ".bin", x.n);
      check(cudaMemcpy(x.d, h.data(), sizeof(double) * x.n, cudaMemcpyHostToDevice), "h2d");
    }
  }
  double* pa_d = nullptr;
  check(cudaMalloc(&pa_d, sizeof(double) * 11), "malloc pa");
  check(cudaMemcpy(pa_d, pa.data(), sizeof(double) * 11, cudaMemcpyHostToDevice), "h2d pa");
  double *P = f[0].d, *tXX = f[1].d, *tYY = f[2].d, *tXY = f[3].d, *tXYav = f[4].d, *J2 = f[5].d, *J2XY = f[6].d;
  double *Ux = f[7].d, *Uy = f[8].d, *Vx = f[9].d, *Vy = f[10].d, *K = f[11].d, *G = f[12].d, *P0 = f[13].d;
  const dim3 grid(nX / 32, nY / 32), block(32, 32);
  for (long it = 0; it < iters; it++) {
    ComputeStress<<<grid, block>>>(Ux, Uy, K, G, P0, P, tXX, tYY, tXY, pa_d, nX, nY);
    check(cudaDeviceSynchronize(), "stress");
    if (nl > 1) {
      ComputeJ2<<<grid, block>>>(tXX, tYY, tXY, tXYav, J2, J2XY, nX, nY);
      check(cudaDeviceSynchronize(), "j2");
      ComputePlasticity<<<grid, block>>>(tXX, tYY, tXY, tXYav, J2, J2XY, pa_d, nX, nY);
      check(cudaDeviceSynchronize(), "plast");
    }
    ComputeDisp<<<grid, block>>>(Ux, Uy, Vx, Vy, P, tXX, tYY, tXY, pa_d, nX, nY);
    check(cudaDeviceSynchronize(), "disp");
  }
  for (auto& x : f) dump_dev(out + "/" + x.name + ".bin", x.d, x.n);
  for (auto& x : f) cudaFree(x.d);
  cudaFree(pa_d);
  return 0;
}

static void put(std::FILE* fp, const char* key, int step, int it, const double* v, int n) {
  std::fprintf(fp, "%s %d %d", key, step, it);
  for (int a = 0; a < n; a++) std::fprintf(fp, " %.17g", v[a]);
  std::fprintf(fp, "\n");
}

static int run_moduli(int argc, char** argv) {
  if (argc < 9) return 1;
  const std::string out = argv[2];
  const double init = std::stod(argv[3]);
  const std::array<double, 3> lt = {std::stod(argv[4]), std::stod(argv[5]), std::stod(argv[6])};
  const unsigned nts = static_cast<unsigned>(std::stod(argv[7]));
  const double lv = std::stod(argv[8]);
  EffPlast2D e(nts);
  if (NL > 3) e.ComputeEffDamping(init, lt, lv);
  else e.ComputeEffModuli(init, lt, lv);
  std::FILE* fp = std::fopen((out + "/records.txt").c_str(), "w");
  if (!fp) return 3;
  std::fprintf(fp, "nX %ld\nnY %ld\nNL %d\nNITER %ld\nnTimeSteps %u\n", e.nX, e.nY, (int)NL, (long)NITER, nts);
  for (int s = 0; s < NL; s++) {
    for (size_t it = 0; it < e.deltaP[s].size(); it++) {
      put(fp, "deltaP", s, (int)it, &e.deltaP[s][it], 1);
      put(fp, "deltaPper", s, (int)it, &e.deltaPper[s][it], 1);
      put(fp, "tauInfty", s, (int)it, &e.tauInfty[s][it], 1);
      put(fp, "dPhi", s, (int)it, &e.dPhi[s][it], 1);
      put(fp, "dPhiPer", s, (int)it, &e.dPhiPer[s][it], 1);
      put(fp, "epsilon", s, (int)it, e.epsilon[s][it].data(), 3);
      put(fp, "epsilonPer", s, (int)it, e.epsilonPer[s][it].data(), 3);
      put(fp, "sigma", s, (int)it, e.sigma[s][it].data(), 4);
      put(fp, "sigmaPer", s, (int)it, e.sigmaPer[s][it].data(), 4);
    }
  }
  const double an[3] = {e.eff_moduli_an.Kphi, e.eff_moduli_an.Kd, e.eff_moduli_an.G};
  const double anp[3] = {e.eff_moduli_an_per.Kphi, e.eff_moduli_an_per.Kd, e.eff_moduli_an_per.G};
  const double nu[3] = {e.eff_moduli_num.Kphi, e.eff_moduli_num.Kd, e.eff_moduli_num.G};
  const double nup[3] = {e.eff_moduli_num_per.Kphi, e.eff_moduli_num_per.Kd, e.eff_moduli_num_per.G};
  put(fp, "moduli_an", -1, -1, an, 3);
  put(fp, "moduli_an_per", -1, -1, anp, 3);
  put(fp, "moduli_num", -1, -1, nu, 3);
  put(fp, "moduli_num_per", -1, -1, nup, 3);
  std::fclose(fp);
  const long nX = e.nX, nY = e.nY;
  const size_t nn = nX * nY, nc = (nX - 1) * (nY - 1), nux = (nX + 1) * nY, nuy = nX * (nY + 1);
  dump_dev(out + "/P.bin", e.P_cuda, nn);
  dump_dev(out + "/tauXX.bin", e.tauXX_cuda, nn);
  dump_dev(out + "/tauYY.bin", e.tauYY_cuda, nn);
  dump_dev(out + "/tauXY.bin", e.tauXY_cuda, nc);
  dump_dev(out + "/tauXYav.bin", e.tauXYav_cuda, nn);
  dump_dev(out + "/J2.bin", e.J2_cuda, nn);
  dump_dev(out + "/J2XY.bin", e.J2XY_cuda, nc);
  dump_dev(out + "/Ux.bin", e.Ux_cuda, nux);
  dump_dev(out + "/Uy.bin", e.Uy_cuda, nuy);
  dump_dev(out + "/Vx.bin", e.Vx_cuda, nux);
  dump_dev(out + "/Vy.bin", e.Vy_cuda, nuy);
  dump_dev(out + "/K.bin", e.K_cuda, nn);
  dump_dev(out + "/G.bin", e.G_cuda, nn);
  return 0;
}

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: %s kernels|moduli ...\n", argv[0]);
    return 1;
  }
  const std::string mode = argv[1];
  int rc = 1;
  if (mode == "kernels") rc = run_kernels(argc, argv);
  else if (mode == "moduli") rc = run_moduli(argc, argv);
  if (rc == 1) std::fprintf(stderr, "bad arguments\n");
  return rc;
}
