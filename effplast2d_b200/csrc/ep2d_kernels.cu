// ep2d_kernels.cu -- launch wrappers for the sm_100a kernels of ep2d_device.cuh.
#include "ep2d_device.cuh"
#include "ep2d_iter_f64.cuh"

namespace ep2d {

namespace {
constexpr int kIterThreadsX = 32, kIterThreadsY = 8;

template <bool PLASTIC, bool RECORD>
cudaError_t set_iter_attr() {
  return cudaFuncSetAttribute(k_iter_f64<TILE_X, TILE_Y, PLASTIC, RECORD>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)sizeof(TileSmem<TILE_X, TILE_Y>));
}
}  // namespace

cudaError_t prepare_kernels() {
  cudaError_t e;
  if ((e = set_iter_attr<false, false>()) != cudaSuccess) return e;
  if ((e = set_iter_attr<false, true>()) != cudaSuccess) return e;
  if ((e = set_iter_attr<true, false>()) != cudaSuccess) return e;
  return set_iter_attr<true, true>();
}

cudaError_t launch_mask(const Geo& g, uint8_t* mask, cudaStream_t stream) {
  const dim3 block(32, 8);
  const dim3 grid((g.nx + 31) / 32, (g.ny + 7) / 8);
  k_mask<<<grid, block, 0, stream>>>(g, mask);
  return cudaGetLastError();
}

cudaError_t launch_preload(const Geo& g, const F64Fields& f, int src, double dUxdx, double dUydy, double dUxdy,
                           int zero_first, cudaStream_t stream) {
  const dim3 block(32, 8);
  const dim3 grid((g.nx + 1 + 31) / 32, (g.ny + 1 + 7) / 8);
  k_preload<<<grid, block, 0, stream>>>(g, f.ux[0], f.ux[1], f.uy[0], f.uy[1], src, dUxdx, dUydy, dUxdy,
                                        zero_first);
  return cudaGetLastError();
}

cudaError_t launch_iter_f64(const Geo& g, const F64Fields& f, int src, bool plastic, bool record,
                            cudaStream_t stream) {
  const dim3 block(kIterThreadsX, kIterThreadsY);
  const dim3 grid((g.nx + TILE_X - 1) / TILE_X, (g.ny + TILE_Y - 1) / TILE_Y);
  const size_t sm = sizeof(TileSmem<TILE_X, TILE_Y>);
  if (plastic) {
    if (record) k_iter_f64<TILE_X, TILE_Y, true, true><<<grid, block, sm, stream>>>(g, f, src);
    else k_iter_f64<TILE_X, TILE_Y, true, false><<<grid, block, sm, stream>>>(g, f, src);
  } else {
    if (record) k_iter_f64<TILE_X, TILE_Y, false, true><<<grid, block, sm, stream>>>(g, f, src);
    else k_iter_f64<TILE_X, TILE_Y, false, false><<<grid, block, sm, stream>>>(g, f, src);
  }
  return cudaGetLastError();
}

namespace {
constexpr int kAvgRowsPerBlock = 4;
int avg_blocks(const Geo& g) {
  const int rows = g.ny - 2;
  return rows > 0 ? (rows + kAvgRowsPerBlock - 1) / kAvgRowsPerBlock : 1;
}
}  // namespace

size_t avg_partials_len(const Geo& g) { return (size_t)avg_blocks(g) * NAVG; }

cudaError_t launch_average(const Geo& g, const F64Fields& f, int src, double nu0, int perOffsetX, int perOffsetY,
                           double* partials, double* sums, cudaStream_t stream) {
  const int nb = avg_blocks(g);
  k_average<<<nb, 256, 0, stream>>>(g, f.p, f.txx, f.tyy, f.txy, src ? f.ux[1] : f.ux[0], src ? f.uy[1] : f.uy[0], nu0, perOffsetX,
                                    perOffsetY, kAvgRowsPerBlock, partials);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_sum_partials<<<1, 32, 0, stream>>>(partials, nb, NAVG, sums);
  return cudaGetLastError();
}

cudaError_t launch_boundary(const Geo& g, const F64Fields& f, double* sums, cudaStream_t stream) {
  k_boundary<<<1, 256, 0, stream>>>(g, f.p, f.txx, f.tyy, sums);
  return cudaGetLastError();
}

cudaError_t launch_gather(const Geo& g, const F64Fields& f, int src, const unsigned long long* idx, int n,
                          double* out, cudaStream_t stream) {
  if (n <= 0) return cudaSuccess;
  k_gather<<<(n + 127) / 128, 128, 0, stream>>>(g, src ? f.ux[1] : f.ux[0], src ? f.uy[1] : f.uy[0], idx, n, out);
  return cudaGetLastError();
}

cudaError_t launch_static_fields(const Geo& g, const F64Fields& f, int src, double* unu, double* j1, double* j2,
                                 cudaStream_t stream) {
  const dim3 block(32, 8);
  const dim3 grid((g.nx + 31) / 32, (g.ny + 7) / 8);
  k_static_fields<<<grid, block, 0, stream>>>(g, src ? f.ux[1] : f.ux[0], src ? f.uy[1] : f.uy[0], f.p, f.txx, f.tyy, f.txy, unu, j1, j2);
  return cudaGetLastError();
}

cudaError_t launch_analytic(const Geo& g, const AnParams& a, const double* unu, const double* j1nu, const double* j2nu,
                            double* uan, double* eu, double* j1an, double* j2an, double* ej1, double* ej2,
                            double* stats, cudaStream_t stream) {
  k_analytic<<<ANALYTIC_BLOCKS, 256, 0, stream>>>(g, a, unu, j1nu, j2nu, uan, eu, j1an, j2an, ej1, ej2, stats);
  return cudaGetLastError();
}

}  // namespace ep2d
