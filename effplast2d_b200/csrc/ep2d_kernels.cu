// ep2d_kernels.cu -- launch wrappers for the sm_100a kernels of ep2d_device.cuh,
// ep2d_iter_f64.cuh (tile form) and ep2d_iter_stream.cuh (stream form).
#include <algorithm>
#include <type_traits>

#include "ep2d_device.cuh"
#include "ep2d_iter_f64.cuh"
#include "ep2d_iter_stream.cuh"

namespace ep2d {

namespace {
constexpr int kIterThreadsX = 32, kIterThreadsY = 8;

template <int TY>
constexpr size_t smem_bytes() {
  return sizeof(TileSmem<TILE_X, TY>);
}

template <int TY, bool PLASTIC, bool RECORD, typename TV>
cudaError_t set_one_attr() {
  return cudaFuncSetAttribute(k_iter<TILE_X, TY, PLASTIC, RECORD, TV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)smem_bytes<TY>());
}

template <int TY, bool RECORD, typename TV>
cudaError_t set_batch_attr() {
  return cudaFuncSetAttribute(k_iter_batch<TILE_X, TY, RECORD, TV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)smem_bytes<TY>());
}

template <int TY, bool PLASTIC, typename TV>
cudaError_t set_resident_attr() {
  return cudaFuncSetAttribute(k_iter_resident<TILE_X, TY, PLASTIC, TV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)smem_bytes<TY>());
}

template <int TY, typename TV>
cudaError_t set_attrs_ty() {
  cudaError_t e;
  if ((e = set_resident_attr<TY, false, TV>()) != cudaSuccess) return e;
  if ((e = set_resident_attr<TY, true, TV>()) != cudaSuccess) return e;
  if ((e = set_one_attr<TY, false, false, TV>()) != cudaSuccess) return e;
  if ((e = set_one_attr<TY, false, true, TV>()) != cudaSuccess) return e;
  if ((e = set_one_attr<TY, true, false, TV>()) != cudaSuccess) return e;
  if ((e = set_one_attr<TY, true, true, TV>()) != cudaSuccess) return e;
  if ((e = set_batch_attr<TY, false, TV>()) != cudaSuccess) return e;
  return set_batch_attr<TY, true, TV>();
}

template <int TY, typename TV>
cudaError_t launch_iter_ty(const Geo& g, const Fields& f, int src, bool plastic, bool record, cudaStream_t stream) {
  const dim3 block(kIterThreadsX, kIterThreadsY);
  const dim3 grid((g.nx + TILE_X - 1) / TILE_X, (g.ny + TY - 1) / TY);
  const size_t sm = smem_bytes<TY>();
  if (plastic) {
    if (record) k_iter<TILE_X, TY, true, true, TV><<<grid, block, sm, stream>>>(g, f, src);
    else k_iter<TILE_X, TY, true, false, TV><<<grid, block, sm, stream>>>(g, f, src);
  } else {
    if (record) k_iter<TILE_X, TY, false, true, TV><<<grid, block, sm, stream>>>(g, f, src);
    else k_iter<TILE_X, TY, false, false, TV><<<grid, block, sm, stream>>>(g, f, src);
  }
  return cudaGetLastError();
}

template <int TY, typename TV>
cudaError_t launch_batch_ty(const BatchEntry* ents, const int2* tiles, const int* ntiles, int parity, bool record,
                            int blocks, cudaStream_t stream) {
  const dim3 block(kIterThreadsX, kIterThreadsY);
  const size_t sm = smem_bytes<TY>();
  if (record) k_iter_batch<TILE_X, TY, true, TV><<<blocks, block, sm, stream>>>(ents, tiles, ntiles, parity);
  else k_iter_batch<TILE_X, TY, false, TV><<<blocks, block, sm, stream>>>(ents, tiles, ntiles, parity);
  return cudaGetLastError();
}

// One cooperative launch of the resident form: as many CTAs as there are tiles, at most
// as many as fit on the GPU at once (the barrier needs all of them resident).
template <int TY, bool PLASTIC, typename TV>
cudaError_t launch_resident_ty(const Geo& g, const Fields& f, int src, int n_iter, unsigned long long timeout_ns,
                               cudaStream_t stream) {
  auto kern = k_iter_resident<TILE_X, TY, PLASTIC, TV>;
  const size_t sm = smem_bytes<TY>();
  int dev = 0, sms = 0, per_sm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, sm);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorCooperativeLaunchTooLarge;
  const int64_t ntiles = (int64_t)((g.nx + TILE_X - 1) / TILE_X) * ((g.ny + TY - 1) / TY);
  const int blocks = (int)std::min<int64_t>(ntiles, (int64_t)per_sm * sms);
  // the arrival count starts at zero; the error flag (gbar[2]) is left as it is
  if ((e = cudaMemsetAsync(f.gbar, 0, 2 * sizeof(unsigned), stream)) != cudaSuccess) return e;
  Geo ga = g;
  Fields fa = f;
  int srca = src, na = n_iter;
  unsigned long long to = timeout_ns;
  void* args[] = {&ga, &fa, &srca, &na, &to};
  return cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(kern), dim3(blocks), dim3(kIterThreadsX, kIterThreadsY),
                                     args, sm, stream);
}

template <int TY, typename TV>
cudaError_t launch_resident_tv(const Geo& g, const Fields& f, int src, bool plastic, int n_iter,
                               unsigned long long timeout_ns, cudaStream_t stream) {
  return plastic ? launch_resident_ty<TY, true, TV>(g, f, src, n_iter, timeout_ns, stream)
                 : launch_resident_ty<TY, false, TV>(g, f, src, n_iter, timeout_ns, stream);
}

template <int TY, typename TV>
int occupancy_ty(bool record) {
  int n = 0;
  const cudaError_t e =
      record ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_iter_batch<TILE_X, TY, true, TV>, 256,
                                                             smem_bytes<TY>())
             : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_iter_batch<TILE_X, TY, false, TV>, 256,
                                                             smem_bytes<TY>());
  return e == cudaSuccess && n > 0 ? n : 1;
}

cudaError_t prepare_kernels_impl() {
  cudaError_t e;
  if ((e = set_attrs_ty<8, double>()) != cudaSuccess) return e;
  if ((e = set_attrs_ty<16, double>()) != cudaSuccess) return e;
  if ((e = set_attrs_ty<32, double>()) != cudaSuccess) return e;
  if ((e = set_attrs_ty<8, float>()) != cudaSuccess) return e;
  if ((e = set_attrs_ty<16, float>()) != cudaSuccess) return e;
  return set_attrs_ty<32, float>();
}

// A launch that may begin while the previous kernel on the stream is still running
// (programmatic stream serialization): the stream-form kernels wait for that kernel's
// completion (griddepcontrol.wait) before they touch global memory, so only their
// start-up overlaps the previous iteration's tail.
template <typename... KArgs, typename... Args>
cudaError_t launch_overlapped(void (*kernel)(KArgs...), int blocks, int threads, size_t smem, cudaStream_t stream,
                              Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

template <typename TU, typename TV>
cudaError_t launch_stream_tv(const Geo& g, const Fields& f, int src, bool plastic, bool record, int seg_h,
                             cudaStream_t stream, bool track = false) {
  const int nstrips = (g.nx + STREAM_COLS - 1) / STREAM_COLS;
  const int nsegs = (g.ny + seg_h - 1) / seg_h;
  const int blocks = (nstrips * nsegs + STREAM_WARPS - 1) / STREAM_WARPS;
  const int threads = 32 * STREAM_WARPS;
  const size_t sm = stream_smem_bytes<TU, TV>();
  if constexpr (std::is_same<TU, double>::value) {
    if (track && plastic) {
      if (record)
        return launch_overlapped(k_iter_stream<true, true, TU, TV, true>, blocks, threads, sm, stream, g, f, src, nstrips, nsegs, seg_h);
      return launch_overlapped(k_iter_stream<true, false, TU, TV, true>, blocks, threads, sm, stream, g, f, src, nstrips, nsegs, seg_h);
    }
  }
  if (plastic) {
    if (record) return launch_overlapped(k_iter_stream<true, true, TU, TV>, blocks, threads, sm, stream, g, f, src, nstrips, nsegs, seg_h);
    return launch_overlapped(k_iter_stream<true, false, TU, TV>, blocks, threads, sm, stream, g, f, src, nstrips, nsegs, seg_h);
  }
  if (record) return launch_overlapped(k_iter_stream<false, true, TU, TV>, blocks, threads, sm, stream, g, f, src, nstrips, nsegs, seg_h);
  return launch_overlapped(k_iter_stream<false, false, TU, TV>, blocks, threads, sm, stream, g, f, src, nstrips, nsegs, seg_h);
}

template <typename TV>
cudaError_t launch_stream_batch_tv(const BatchEntry* ents, const int2* units, const int* nunits, int parity,
                                   bool record, int seg_h, int blocks, cudaStream_t stream) {
  const int threads = 32 * STREAM_WARPS;
  const size_t sm = stream_smem_bytes<double, TV>();
  // plain launches: the persistent batched grid measured 1.5-3 % slower overlapped
  if (record) k_iter_stream_batch<true, TV><<<blocks, threads, sm, stream>>>(ents, units, nunits, parity, seg_h);
  else k_iter_stream_batch<false, TV><<<blocks, threads, sm, stream>>>(ents, units, nunits, parity, seg_h);
  return cudaGetLastError();
}

template <typename TV>
int stream_occupancy(bool record) {
  int n = 0;
  const cudaError_t e =
      record ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_iter_stream_batch<true, TV>, 32 * STREAM_WARPS,
                                                             stream_smem_bytes<double, TV>())
             : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_iter_stream_batch<false, TV>, 32 * STREAM_WARPS,
                                                             stream_smem_bytes<double, TV>());
  return e == cudaSuccess && n > 0 ? n : 1;
}
}  // namespace

cudaError_t prepare_kernels() { return prepare_kernels_impl(); }

void shape_units(const IterShape& s, int nx, int ny, int* ux, int* uy) {
  const int cols = s.form == FORM_TILE ? TILE_X : STREAM_COLS;
  *ux = (nx + cols - 1) / cols;
  *uy = (ny + s.rows - 1) / s.rows;
}

cudaError_t launch_iter(const Geo& g, const Fields& f, int src, bool plastic, bool record, bool mixed,
                        const IterShape& shape, cudaStream_t stream, bool track) {
  if (shape.form == FORM_STREAM) {
    if (shape.rows < SEG_MIN || shape.rows > SEG_MAX) return cudaErrorInvalidValue;
    return mixed ? launch_stream_tv<double, float>(g, f, src, plastic, record, shape.rows, stream, track)
                 : launch_stream_tv<double, double>(g, f, src, plastic, record, shape.rows, stream, track);
  }
  if (track) return cudaErrorInvalidValue;  // the plastic-zone tracking runs the stream form
  const int tile_y = shape.rows;
  if (mixed) {
    if (tile_y == 8) return launch_iter_ty<8, float>(g, f, src, plastic, record, stream);
    if (tile_y == 32) return launch_iter_ty<32, float>(g, f, src, plastic, record, stream);
    return launch_iter_ty<16, float>(g, f, src, plastic, record, stream);
  }
  if (tile_y == 8) return launch_iter_ty<8, double>(g, f, src, plastic, record, stream);
  if (tile_y == 32) return launch_iter_ty<32, double>(g, f, src, plastic, record, stream);
  return launch_iter_ty<16, double>(g, f, src, plastic, record, stream);
}

cudaError_t launch_iter_resident(const Geo& g, const Fields& f, int src, bool plastic, bool mixed, int rows,
                                 int64_t n_iter, unsigned long long timeout_ns, cudaStream_t stream) {
  if (rows != 8 && rows != 16 && rows != 32) return cudaErrorInvalidValue;
  if (!f.gbar) return cudaErrorInvalidValue;
  // in chunks of an even number of iterations below 2^31 (a chunk keeps the parity)
  constexpr int64_t kChunk = (int64_t)1 << 30;
  while (n_iter > 0) {
    const int n = (int)std::min(n_iter, kChunk);
    cudaError_t e;
    if (mixed) {
      e = rows == 8    ? launch_resident_tv<8, float>(g, f, src, plastic, n, timeout_ns, stream)
          : rows == 32 ? launch_resident_tv<32, float>(g, f, src, plastic, n, timeout_ns, stream)
                       : launch_resident_tv<16, float>(g, f, src, plastic, n, timeout_ns, stream);
    } else {
      e = rows == 8    ? launch_resident_tv<8, double>(g, f, src, plastic, n, timeout_ns, stream)
          : rows == 32 ? launch_resident_tv<32, double>(g, f, src, plastic, n, timeout_ns, stream)
                       : launch_resident_tv<16, double>(g, f, src, plastic, n, timeout_ns, stream);
    }
    if (e != cudaSuccess) return e;
    n_iter -= n;
  }
  return cudaSuccess;
}

cudaError_t launch_grid_barrier_check(unsigned* gbar, int blocks, int missing, int rounds,
                                      unsigned long long timeout_ns, unsigned* out, cudaStream_t stream) {
  if (blocks < 1 || missing < 0 || missing > blocks || rounds < 0) return cudaErrorInvalidValue;
  int dev = 0, sms = 0, per_sm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_grid_barrier_check, 32, 0);
  if (e != cudaSuccess) return e;
  if ((int64_t)blocks > (int64_t)per_sm * sms) return cudaErrorCooperativeLaunchTooLarge;
  if ((e = cudaMemsetAsync(gbar, 0, 4 * sizeof(unsigned), stream)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(out, 0, sizeof(unsigned), stream)) != cudaSuccess) return e;
  void* args[] = {&gbar, &missing, &rounds, &timeout_ns, &out};
  return cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(k_grid_barrier_check), dim3(blocks), dim3(32), args,
                                     0, stream);
}

cudaError_t launch_iter_f32(const Geo& g, const Fields& f, int src, bool plastic, bool record, int seg_h,
                            cudaStream_t stream) {
  if (seg_h < SEG_MIN || seg_h > SEG_MAX) return cudaErrorInvalidValue;
  return launch_stream_tv<float, float>(g, f, src, plastic, record, seg_h, stream);
}

cudaError_t launch_iter_batch(const BatchEntry* ents, const int2* units, const int* nunits, int parity, bool record,
                              bool mixed, const IterShape& shape, int blocks, cudaStream_t stream) {
  if (shape.form == FORM_STREAM) {
    if (shape.rows < SEG_MIN || shape.rows > SEG_MAX) return cudaErrorInvalidValue;
    return mixed ? launch_stream_batch_tv<float>(ents, units, nunits, parity, record, shape.rows, blocks, stream)
                 : launch_stream_batch_tv<double>(ents, units, nunits, parity, record, shape.rows, blocks, stream);
  }
  const int tile_y = shape.rows;
  if (mixed) {
    if (tile_y == 8) return launch_batch_ty<8, float>(ents, units, nunits, parity, record, blocks, stream);
    if (tile_y == 32) return launch_batch_ty<32, float>(ents, units, nunits, parity, record, blocks, stream);
    return launch_batch_ty<16, float>(ents, units, nunits, parity, record, blocks, stream);
  }
  if (tile_y == 8) return launch_batch_ty<8, double>(ents, units, nunits, parity, record, blocks, stream);
  if (tile_y == 32) return launch_batch_ty<32, double>(ents, units, nunits, parity, record, blocks, stream);
  return launch_batch_ty<16, double>(ents, units, nunits, parity, record, blocks, stream);
}

int iter_blocks_per_sm(bool record, bool mixed, const IterShape& shape) {
  if (shape.form == FORM_STREAM) return mixed ? stream_occupancy<float>(record) : stream_occupancy<double>(record);
  const int tile_y = shape.rows;
  if (mixed) {
    if (tile_y == 8) return occupancy_ty<8, float>(record);
    if (tile_y == 32) return occupancy_ty<32, float>(record);
    return occupancy_ty<16, float>(record);
  }
  if (tile_y == 8) return occupancy_ty<8, double>(record);
  if (tile_y == 32) return occupancy_ty<32, double>(record);
  return occupancy_ty<16, double>(record);
}

cudaError_t launch_mask(const Geo& g, uint8_t* mask, cudaStream_t stream) {
  const dim3 block(32, 8);
  const dim3 grid((g.nx + 31) / 32, (g.ny + 7) / 8);
  k_mask<<<grid, block, 0, stream>>>(g, mask);
  return cudaGetLastError();
}

cudaError_t launch_preload(const Geo& g, const Fields& f, int src, double dUxdx, double dUydy, double dUxdy,
                           int zero_first, cudaStream_t stream) {
  const dim3 block(32, 8);
  const dim3 grid((g.nx + 1 + 31) / 32, (g.ny + 1 + 7) / 8);
  k_preload<<<grid, block, 0, stream>>>(g, f.ux[0], f.ux[1], f.uy[0], f.uy[1], src, dUxdx, dUydy, dUxdy,
                                        zero_first);
  return cudaGetLastError();
}

cudaError_t launch_to_f32(const Geo& g, const Fields& f, int src, cudaStream_t stream) {
  const dim3 block(32, 8);
  const dim3 grid((g.nx + 1 + 31) / 32, (g.ny + 1 + 7) / 8);
  k_to_f32<<<grid, block, 0, stream>>>(g, f.ux[src], f.uy[src], f.ux32[0], f.ux32[1], f.uy32[0], f.uy32[1], g.exx0,
                                       g.eyy0, 0.5 * g.exy0);
  return cudaGetLastError();
}

cudaError_t launch_from_f32(const Geo& g, const Fields& f, int src, cudaStream_t stream) {
  const dim3 block(32, 8);
  const dim3 grid((g.nx + 1 + 31) / 32, (g.ny + 1 + 7) / 8);
  k_from_f32<<<grid, block, 0, stream>>>(g, f.ux32[src], f.uy32[src], f.ux[0], f.ux[1], f.uy[0], f.uy[1], g.exx0,
                                         g.eyy0, 0.5 * g.exy0);
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

cudaError_t launch_average(const Geo& g, const Fields& f, int src, double nu0, int perOffsetX, int perOffsetY,
                           double* partials, double* sums, cudaStream_t stream) {
  const int nb = avg_blocks(g);
  k_average<<<nb, 256, 0, stream>>>(g, f.p, f.txx, f.tyy, f.txy, src ? f.ux[1] : f.ux[0], src ? f.uy[1] : f.uy[0],
                                    nu0, perOffsetX, perOffsetY, kAvgRowsPerBlock, partials);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_sum_partials<<<1, 32, 0, stream>>>(partials, nb, NAVG, sums);
  return cudaGetLastError();
}

cudaError_t launch_boundary(const Geo& g, const Fields& f, double* sums, cudaStream_t stream) {
  k_boundary<<<1, 256, 0, stream>>>(g, f.p, f.txx, f.tyy, sums);
  return cudaGetLastError();
}

cudaError_t launch_gather(const Geo& g, const Fields& f, int src, const unsigned long long* idx, int n,
                          double* out, cudaStream_t stream) {
  if (n <= 0) return cudaSuccess;
  k_gather<<<(n + 127) / 128, 128, 0, stream>>>(g, src ? f.ux[1] : f.ux[0], src ? f.uy[1] : f.uy[0], idx, n, out);
  return cudaGetLastError();
}

cudaError_t launch_static_fields(const Geo& g, const Fields& f, int src, double* unu, double* j1, double* j2,
                                 cudaStream_t stream) {
  const dim3 block(32, 8);
  const dim3 grid((g.nx + 31) / 32, (g.ny + 7) / 8);
  k_static_fields<<<grid, block, 0, stream>>>(g, src ? f.ux[1] : f.ux[0], src ? f.uy[1] : f.uy[0], f.p, f.txx, f.tyy,
                                              f.txy, unu, j1, j2);
  return cudaGetLastError();
}

cudaError_t launch_polar_fields(const Geo& g, const Fields& f, double sgn, double* snrr, double* snff, double* sarr,
                                double* saff, uint8_t* plast, bool accumulated, cudaStream_t stream) {
  const dim3 block(32, 8);
  const dim3 grid((g.nx + 31) / 32, (g.ny + 7) / 8);
  k_polar_fields<<<grid, block, 0, stream>>>(g, f.p, f.txx, f.tyy, f.txyav, f.j2, f.j2xy, accumulated ? f.mask : nullptr,
                                             sgn, snrr, snff, sarr, saff, plast);
  return cudaGetLastError();
}

cudaError_t launch_clear_track(const Geo& g, uint8_t* mask, cudaStream_t stream) {
  const dim3 block(32, 8);
  const dim3 grid((g.nx + 31) / 32, (g.ny + 7) / 8);
  k_clear_track<<<grid, block, 0, stream>>>(g, mask);
  return cudaGetLastError();
}

cudaError_t launch_analytic(const Geo& g, const AnParams& a, const double* unu, const double* j1nu, const double* j2nu,
                            double* uan, double* eu, double* j1an, double* j2an, double* ej1, double* ej2,
                            double* stats, cudaStream_t stream) {
  k_analytic<<<ANALYTIC_BLOCKS, 256, 0, stream>>>(g, a, unu, j1nu, j2nu, uan, eu, j1an, j2an, ej1, ej2, stats);
  return cudaGetLastError();
}

}  // namespace ep2d
