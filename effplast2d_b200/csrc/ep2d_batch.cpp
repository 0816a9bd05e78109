// ep2d_batch.cpp -- batched persistent solver and continuous-batching server.
#include "ep2d_batch.hpp"

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <set>
#include <thread>

namespace ep2d {

#define EP2D_CK(call)                                                                       \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess) return fail(EP2D_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

namespace {
double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

ep2d_params params_of(const ep2d_batch_config& c, const ep2d_rve_spec& s) {
  ep2d_params p{};
  p.nx = s.nx;
  p.ny = s.ny;
  std::memcpy(p.pa, s.pa, sizeof(p.pa));
  p.nl = s.nl;
  p.check_every = c.check_every;
  p.niter = c.niter;
  p.eiter = c.eiter;
  p.precision = c.precision;
  p.device = c.device;
  return p;
}

int validate_config(const ep2d_batch_config& c) {
  if (c.check_every < 2) return fail(EP2D_ERR_ARG, "check_every must be >= 2 in a batch");
  if (c.niter < c.check_every || c.niter % c.check_every != 0)
    return fail(EP2D_ERR_ARG, "niter must be a positive multiple of check_every in a batch");
  if (c.precision == EP2D_F32_BULK)
    return fail(EP2D_ERR_ARG, "the FP32 bulk (EP2D_F32_BULK) runs on single-RVE handles only; batches take EP2D_FP64 "
                              "or EP2D_MIXED");
  if (c.precision != EP2D_FP64 && c.precision != EP2D_MIXED) return fail(EP2D_ERR_ARG, "unknown precision");
  if (c.kernel == EP2D_KERNEL_RESIDENT)
    return fail(EP2D_ERR_ARG, "the resident form (EP2D_KERNEL_RESIDENT) runs on single-RVE handles only");
  if (c.kernel < EP2D_KERNEL_AUTO || c.kernel > EP2D_KERNEL_STREAM) return fail(EP2D_ERR_ARG, "unknown kernel form");
  if (c.rows != 0) {
    IterShape sh;
    sh.form = c.kernel == EP2D_KERNEL_TILE ? FORM_TILE : FORM_STREAM;
    sh.rows = c.rows;
    if (!shape_valid(sh))
      return fail(EP2D_ERR_ARG, "rows must be 0, or 8, 16 or 32 for the tile form and 4..1024 for the stream form");
  }
  if (c.graph_len < 0 || (c.graph_len % 2) != 0) return fail(EP2D_ERR_ARG, "graph_len must be even");
  return EP2D_OK;
}
}  // namespace

BatchEngine::~BatchEngine() {
  if (!stream) return;
  DeviceScope ds(device);
  cudaStreamSynchronize(stream);
  slots_.clear();
  if (graph_) cudaGraphExecDestroy(graph_);
  for (auto& e : ev_)
    if (e) cudaEventDestroy(e);
  cudaFree(d_ents_);
  cudaFree(d_tiles_);
  cudaFree(d_ntiles_);
  cudaFree(d_vmax_);
  if (h_vmax_) cudaFreeHost(h_vmax_);
  cudaStreamDestroy(stream);
}

int BatchEngine::init(const ep2d_batch_config& c) {
  int rc = validate_config(c);
  if (rc) return rc;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(EP2D_ERR_NODEV, "no CUDA device");
  }
  if (c.device < 0 || c.device >= ndev) return fail(EP2D_ERR_ARG, "device index out of range");
  cfg = c;
  if (cfg.graph_len == 0) cfg.graph_len = 64;
  device = c.device;
  DeviceScope ds(device);
  rc = prepare_device(device);
  if (rc) return rc;
  EP2D_CK(cudaDeviceGetAttribute(&sm_count_, cudaDevAttrMultiProcessorCount, device));
  EP2D_CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  EP2D_CK(cudaEventCreate(&ev_[0]));
  EP2D_CK(cudaEventCreate(&ev_[1]));
  EP2D_CK(cudaMalloc(&d_ntiles_, sizeof(int)));
  shape.form = c.kernel == EP2D_KERNEL_TILE ? FORM_TILE : FORM_STREAM;
  shape.rows = c.rows ? c.rows : (shape.form == FORM_TILE ? TILE_Y : SEG_DEFAULT);
  tuned = c.rows != 0;
  blocks = sm_count_ * iter_blocks_per_sm(false, c.precision == EP2D_MIXED, shape);
  return grow(16);
}

size_t BatchEngine::footprint(const ep2d_rve_spec& s) const { return Rve::footprint(params_of(cfg, s)); }

void BatchEngine::fill_stats(ep2d_batch_stats* st) const {
  st->rows = shape.rows;
  st->blocks = blocks;
  st->kernel = shape.form == FORM_TILE ? EP2D_KERNEL_TILE : EP2D_KERNEL_STREAM;
  st->n_tuned = n_tuned;
  for (int q = 0; q < 7; q++) st->tune_us[q] = tune_us[q];
  st->n_tunes = n_tunes;
  st->solo_intervals = solo_intervals;
}

int BatchEngine::grow(int need) {
  if (need <= cap_slots_) return EP2D_OK;
  const int cap = std::max(need, 2 * cap_slots_);
  DeviceScope ds(device);
  EP2D_CK(cudaStreamSynchronize(stream));
  cudaFree(d_ents_);
  cudaFree(d_vmax_);
  if (h_vmax_) cudaFreeHost(h_vmax_);
  d_ents_ = nullptr;
  d_vmax_ = nullptr;
  h_vmax_ = nullptr;
  EP2D_CK(cudaMalloc(&d_ents_, cap * sizeof(BatchEntry)));
  EP2D_CK(cudaMalloc(&d_vmax_, cap * 2 * sizeof(unsigned long long)));
  EP2D_CK(cudaMallocHost(&h_vmax_, cap * 2 * sizeof(unsigned long long)));
  cap_slots_ = cap;
  if (graph_) {  // the graph holds the old pointers
    cudaGraphExecDestroy(graph_);
    graph_ = nullptr;
  }
  tiles_dirty_ = true;
  return EP2D_OK;
}

int BatchEngine::active() const {
  int n = 0;
  for (const auto& s : slots_) n += (s.used && !s.task.done) ? 1 : 0;
  return n;
}

int BatchEngine::begin_task_step(Slot& s) {
  Task& t = s.task;
  double lsv, lt[3];
  int nts;
  Rve::step_load(t.step, t.spec.init_load_value, t.spec.load_type, t.spec.n_time_steps, &lsv, lt, &nts);
  if (t.it == 0) {
    const int rc = s.rve->begin_step(t.step, nts);
    if (rc) return rc;
  }
  t.iters = 0;
  const int rc = s.rve->begin_time_step(t.step, t.it, lsv, lt, nts);
  aux_launches += 1;
  return rc;
}

int BatchEngine::add(const ep2d_rve_spec& spec, uint64_t ticket, double submit_s, int* slot_out) {
  DeviceScope ds(device);
  if (spec.n_time_steps < 1) return fail(EP2D_ERR_ARG, "n_time_steps must be >= 1");
  if (spec.nl < 1 || spec.nl > EP2D_MAX_NL)
    return fail(EP2D_ERR_ARG, "a batch runs ComputeEffModuli: nl must be 1, 2 or 3");
  int slot = -1;
  for (size_t k = 0; k < slots_.size(); k++)
    if (!slots_[k].used) {
      slot = (int)k;
      break;
    }
  if (slot < 0) {
    slot = (int)slots_.size();
    slots_.emplace_back();
  }
  int rc = grow((int)slots_.size());
  if (rc) return rc;
  Slot& s = slots_[slot];
  s.rve.reset(new Rve());
  rc = s.rve->create(params_of(cfg, spec), stream);
  if (rc) {
    s.rve.reset();
    return rc;
  }
  s.rve->shape = shape;
  s.solo = fills_gpu(*s.rve);
  s.used = true;
  s.task = Task{};
  s.task.spec = spec;
  s.task.ticket = ticket;
  s.task.submit_s = submit_s;
  s.task.admit_s = now_s();
  s.rve->begin_chain(spec.load_type);
  rc = begin_task_step(s);
  if (rc) {
    s.rve.reset();
    s.used = false;
    return rc;
  }
  bytes_ += footprint(spec);
  tiles_dirty_ = true;
  set_version_++;
  if (slot_out) *slot_out = slot;
  return EP2D_OK;
}

int BatchEngine::rebuild_tiles() {
  std::vector<int2> tiles;
  for (size_t k = 0; k < slots_.size(); k++) {
    const Slot& s = slots_[k];
    if (!s.used || s.task.done || (s.solo && cfg.rows == 0)) continue;
    int tx = 0, ty = 0;
    shape_units(shape, s.rve->g.nx, s.rve->g.ny, &tx, &ty);
    for (int by = 0; by < ty; by++)
      for (int bx = 0; bx < tx; bx++) tiles.push_back(make_int2((int)k, bx | (by << 16)));
  }
  if ((int)tiles.size() > cap_tiles_) {
    const int cap = std::max((int)tiles.size(), 2 * cap_tiles_);
    EP2D_CK(cudaStreamSynchronize(stream));
    cudaFree(d_tiles_);
    d_tiles_ = nullptr;
    EP2D_CK(cudaMalloc(&d_tiles_, (size_t)cap * sizeof(int2)));
    cap_tiles_ = cap;
    if (graph_) {
      cudaGraphExecDestroy(graph_);
      graph_ = nullptr;
    }
  }
  n_tiles_ = (int)tiles.size();
  if (n_tiles_)
    EP2D_CK(cudaMemcpyAsync(d_tiles_, tiles.data(), tiles.size() * sizeof(int2), cudaMemcpyHostToDevice, stream));
  EP2D_CK(cudaMemcpyAsync(d_ntiles_, &n_tiles_, sizeof(int), cudaMemcpyHostToDevice, stream));
  EP2D_CK(cudaStreamSynchronize(stream));  // the host vectors go out of scope
  tiles_dirty_ = false;
  return EP2D_OK;
}

int BatchEngine::ensure_graph() {
  if (graph_ && graph_shape_.form == shape.form && graph_shape_.rows == shape.rows) return EP2D_OK;
  if (graph_) {
    cudaGraphExecDestroy(graph_);
    graph_ = nullptr;
  }
  const bool mixed = cfg.precision == EP2D_MIXED;
  cudaGraph_t g = nullptr;
  EP2D_CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t le = cudaSuccess;
  for (int k = 0; k < cfg.graph_len && le == cudaSuccess; k++)
    le = launch_iter_batch(d_ents_, d_tiles_, d_ntiles_, k & 1, false, mixed, shape, blocks, stream);
  const cudaError_t ee = cudaStreamEndCapture(stream, &g);
  if (le != cudaSuccess || ee != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return fail(EP2D_ERR_CUDA, std::string("batch graph capture: ") + cudaGetErrorString(le != cudaSuccess ? le : ee));
  }
  const cudaError_t ie = cudaGraphInstantiate(&graph_, g, 0);
  cudaGraphDestroy(g);
  if (ie != cudaSuccess) return fail(EP2D_ERR_CUDA, std::string("batch graph instantiate: ") + cudaGetErrorString(ie));
  graph_shape_ = shape;
  return EP2D_OK;
}

// launches k0 .. k0+n-1 of the interval (parity k & 1), graphs where aligned
int BatchEngine::launch_plain_run(int64_t k0, int64_t n) {
  const bool mixed = cfg.precision == EP2D_MIXED;
  int64_t k = k0;
  while (n > 0) {
    if ((k & 1) == 0 && n >= cfg.graph_len && graph_) {
      EP2D_CK(cudaGraphLaunch(graph_, stream));
      k += cfg.graph_len;
      n -= cfg.graph_len;
    } else {
      EP2D_CK(launch_iter_batch(d_ents_, d_tiles_, d_ntiles_, (int)(k & 1), false, mixed, shape, blocks, stream));
      k++;
      n--;
    }
  }
  return EP2D_OK;
}

// Time the candidate kernel shapes (tile form, rows 8/16/32; stream form, rows
// 8/16/32/64; only the form cfg.kernel names unless it is AUTO) on real iterations of
// the first interval -- they advance the solution like any other launch -- and keep
// the fastest.  *k: launches done so far.
int BatchEngine::autotune(int64_t* k, int64_t n_avail) {
  IterShape cand[7];
  int slot[7], nc = 0;
  if (cfg.kernel != EP2D_KERNEL_TILE)
    for (int q = 0; q < 4; q++) {
      cand[nc].form = FORM_STREAM;
      cand[nc].rows = SEG_CHOICES[q];
      slot[nc++] = 3 + q;
    }
  if (cfg.kernel != EP2D_KERNEL_STREAM)
    for (int q = 0; q < 3; q++) {
      cand[nc].form = FORM_TILE;
      cand[nc].rows = TILE_Y_CHOICES[q];
      slot[nc++] = q;
    }
  const int per = 24;  // 4 warm-up + 20 timed launches per candidate
  tuned_version_ = set_version_;
  if (n_avail < nc * per) {
    tuned = true;
    return EP2D_OK;
  }
  n_tunes++;
  n_tuned = 0;
  for (double& u : tune_us) u = 0.0;
  const bool mixed = cfg.precision == EP2D_MIXED;
  float best = 1e30f;
  IterShape best_shape = shape;
  for (int c = 0; c < nc; c++) {
    shape = cand[c];
    blocks = sm_count_ * iter_blocks_per_sm(false, mixed, shape);
    int rc = rebuild_tiles();
    if (rc) return rc;
    for (int w = 0; w < 4; w++, (*k)++)
      EP2D_CK(launch_iter_batch(d_ents_, d_tiles_, d_ntiles_, (int)(*k & 1), false, mixed, shape, blocks, stream));
    EP2D_CK(cudaEventRecord(ev_[0], stream));
    for (int w = 0; w < per - 4; w++, (*k)++)
      EP2D_CK(launch_iter_batch(d_ents_, d_tiles_, d_ntiles_, (int)(*k & 1), false, mixed, shape, blocks, stream));
    EP2D_CK(cudaEventRecord(ev_[1], stream));
    EP2D_CK(cudaEventSynchronize(ev_[1]));
    float ms = 0.0f;
    EP2D_CK(cudaEventElapsedTime(&ms, ev_[0], ev_[1]));
    kernel_ms += ms;
    const float us = 1000.0f * ms / (per - 4);
    tune_us[slot[c]] = us;
    n_tuned++;
    if (us < best) {
      best = us;
      best_shape = shape;
    }
  }
  shape = best_shape;
  blocks = sm_count_ * iter_blocks_per_sm(false, mixed, shape);
  for (auto& s : slots_)
    if (s.used) s.rve->shape = shape;
  tuned = true;
  return rebuild_tiles();
}

int BatchEngine::advance(Slot& s, double error) {
  Task& t = s.task;
  Rve& r = *s.rve;
  ep2d_step_record& rec = r.rec[t.step][t.it];
  r.checks[t.step][t.it].push_back(error);
  rec.n_checks++;
  const bool conv = error < cfg.eiter;
  if (!conv && t.iters < cfg.niter) return EP2D_OK;  // keep iterating
  rec.iterations = conv ? t.iters : cfg.niter;
  rec.converged = conv ? 1 : 0;
  rec.error = error;
  int rc = r.finish_time_step(t.step, t.it);
  aux_launches += 4;
  if (rc) return rc;
  if (t.it + 1 < r.nts[t.step]) {
    t.it++;
    return begin_task_step(s);
  }
  if (t.step + 1 < r.prm.nl) {
    t.step++;
    t.it = 0;
    return begin_task_step(s);
  }
  r.finish_chain(t.spec.n_time_steps, &t.result);
  t.done = true;
  t.done_s = now_s();
  finished_.push_back(t);
  bytes_ -= footprint(t.spec);
  s.rve.reset();  // release the RVE's device memory
  s.used = false;
  tiles_dirty_ = true;
  set_version_++;
  return EP2D_OK;
}

// True if the RVE keeps the GPU busy alone: its own kernel shape (shape_of) is the stream
// form with segments of 16 rows or more and 16 warps' worth of them on every SM.  Such
// an RVE gains nothing from sharing launches with others and runs its iterations through
// the single-RVE path (its own shape, overlapped launches, its own captured graphs);
// smaller ones share the batched launches.  Shorter segments are the single-RVE path's
// answer to a grid too small to fill the GPU (768^2 alone: 8-row segments, 41 G
// cell-updates/s), which a shared launch beats.
bool BatchEngine::fills_gpu(const Rve& r) const {
  const IterShape sh = shape_of(r.prm, sm_count_);
  if (sh.form != FORM_STREAM || sh.rows < 16) return false;
  int ux = 0, uy = 0;
  shape_units(sh, r.g.nx, r.g.ny, &ux, &uy);
  return (int64_t)ux * uy >= 16 * (int64_t)sm_count_;
}

// One checkpoint interval of slot q through the single-RVE path: ce - 1 plain launches
// and the recording one, its max|V| into the slot's pair of d_vmax_.  Every form rounds
// alike, so the result is the one the batched launches would give.
int BatchEngine::run_solo_launches(int q) {
  Slot& s = slots_[q];
  Rve& r = *s.rve;
  const int64_t ce = cfg.check_every;
  r.f.vmax = d_vmax_ + 2 * q;
  r.shape = shape_of(r.prm, sm_count_);  // always the same shape: its cached graphs stay valid
  const double ms0 = r.kernel_ms;
  const int rc = r.iterate(ce, true);  // cur follows the launches
  if (rc) return rc;
  kernel_ms += r.kernel_ms - ms0;
  launches += ce;
  cell_updates += ce * (int64_t)r.g.nx * r.g.ny;
  solo_intervals++;
  return EP2D_OK;
}

// After an interval: every active RVE's checkpoint (convergence test, next time step or
// load step, retirement).  Slots marked `batched` ran the interval in batched launches,
// which leave the ping-pong parity to be advanced here; the others advanced their own.
void BatchEngine::finish_interval(const std::vector<char>& batched) {
  const int64_t ce = cfg.check_every;
  for (size_t q = 0; q < slots_.size(); q++) {
    Slot& s = slots_[q];
    if (!s.used || s.task.done) continue;
    if (batched[q]) s.rve->cur ^= (int)(ce & 1);
    s.task.iters += ce;
    double vmx, vmy;
    std::memcpy(&vmx, &h_vmax_[2 * q], sizeof(double));
    std::memcpy(&vmy, &h_vmax_[2 * q + 1], sizeof(double));
    const int rc = advance(s, s.rve->error_from_vmax(vmx, vmy));
    if (rc) {
      s.task.status = rc;
      s.task.error = last_error();
      s.task.done = true;
      s.task.done_s = now_s();
      finished_.push_back(s.task);
      bytes_ -= footprint(s.task.spec);
      s.rve.reset();
      s.used = false;
      tiles_dirty_ = true;
      set_version_++;
    }
  }
}

// One checkpoint interval (check_every iterations) of every active RVE: the RVEs that
// fill the GPU alone (and a lone RVE of any size) through the single-RVE path, one after
// another; the others together in batched launches.  A pinned shape batches every RVE.
int BatchEngine::run_interval() {
  if (active() == 0) return EP2D_OK;
  DeviceScope ds(device);
  const bool mixed = cfg.precision == EP2D_MIXED;
  const bool pinned = cfg.rows != 0;
  const int n_active = active();
  std::vector<char> batched(slots_.size(), 0);
  std::vector<int> solo;
  int n_batched = 0;
  int64_t cells = 0;
  for (size_t q = 0; q < slots_.size(); q++) {
    const Slot& s = slots_[q];
    if (!s.used || s.task.done) continue;
    if (!pinned && (s.solo || n_active == 1)) {
      solo.push_back((int)q);
    } else {
      batched[q] = 1;
      n_batched++;
      cells += (int64_t)s.rve->g.nx * s.rve->g.ny;
    }
  }
  const int64_t ce = cfg.check_every;
  EP2D_CK(cudaMemsetAsync(d_vmax_, 0, slots_.size() * 2 * sizeof(unsigned long long), stream));
  if (n_batched > 0) {
    // the fastest shape depends on the batched set: tune again after it changed
    if (!pinned && tuned && tuned_version_ != set_version_) tuned = false;
    // entries: geometry, pointers, current ping-pong parity, per-slot vmax
    std::vector<BatchEntry> ents(slots_.size());
    for (size_t k = 0; k < slots_.size(); k++) {
      Slot& s = slots_[k];
      if (!s.used) continue;
      s.rve->f.vmax = d_vmax_ + 2 * k;
      ents[k].g = s.rve->g;
      ents[k].f = s.rve->f;
      ents[k].src0 = s.rve->cur;
      ents[k].plastic = s.rve->prm.nl > 1 ? 1 : 0;
    }
    EP2D_CK(cudaMemcpyAsync(d_ents_, ents.data(), ents.size() * sizeof(BatchEntry), cudaMemcpyHostToDevice, stream));
    if (tiles_dirty_) {
      const int rc = rebuild_tiles();
      if (rc) return rc;
    } else {
      EP2D_CK(cudaStreamSynchronize(stream));
    }
    int64_t k = 0;
    if (!tuned) {
      const int rc = autotune(&k, ce - 1);
      if (rc) return rc;
    }
    int rc = ensure_graph();
    if (rc) return rc;
    EP2D_CK(cudaEventRecord(ev_[0], stream));
    rc = launch_plain_run(k, ce - 1 - k);
    if (rc) return rc;
    EP2D_CK(launch_iter_batch(d_ents_, d_tiles_, d_ntiles_, (int)((ce - 1) & 1), true, mixed, shape, blocks, stream));
    EP2D_CK(cudaEventRecord(ev_[1], stream));
    EP2D_CK(cudaEventSynchronize(ev_[1]));
    float ms = 0.0f;
    EP2D_CK(cudaEventElapsedTime(&ms, ev_[0], ev_[1]));
    kernel_ms += ms;
    launches += ce;
    cell_updates += ce * cells;
  }
  for (int q : solo) {
    const int rc = run_solo_launches(q);
    if (rc) return rc;
  }
  EP2D_CK(cudaMemcpyAsync(h_vmax_, d_vmax_, slots_.size() * 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                          stream));
  EP2D_CK(cudaStreamSynchronize(stream));
  finish_interval(batched);
  return EP2D_OK;
}

std::vector<Task> BatchEngine::take_finished() {
  std::vector<Task> out;
  out.swap(finished_);
  return out;
}

void BatchEngine::abort_all(int status, const std::string& error) {
  for (auto& s : slots_) {
    if (!s.used) continue;
    s.task.status = status;
    s.task.error = error;
    s.task.done = true;
    s.task.done_s = now_s();
    finished_.push_back(s.task);
    bytes_ -= footprint(s.task.spec);
    s.rve.reset();
    s.used = false;
  }
  tiles_dirty_ = true;
  set_version_++;
}

// ---- server -------------------------------------------------------------------------
class Server {
 public:
  int start(const ep2d_batch_config& c, int64_t budget, int32_t max_active) {
    budget_ = budget;
    max_active_ = max_active > 0 ? max_active : 1 << 30;
    std::unique_lock<std::mutex> lk(mu_);
    worker_ = std::thread([this, c] { loop(c); });
    cv_.wait(lk, [this] { return started_; });
    return init_rc_;
  }
  void stop() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    if (worker_.joinable()) worker_.join();
  }
  int submit(const ep2d_rve_spec& s, uint64_t* ticket) {
    std::lock_guard<std::mutex> lk(mu_);
    if (!init_ok_)
      return fail(EP2D_ERR_STATE, stop_msg_.empty() ? "server is not running" : "server stopped: " + stop_msg_);
    Task t;
    t.spec = s;
    t.ticket = ++next_ticket_;
    t.submit_s = now_s();
    pending_.push_back(t);
    outstanding_.insert(t.ticket);
    submitted_++;
    if (ticket) *ticket = t.ticket;
    cv_.notify_all();
    return EP2D_OK;
  }
  // A finished request's result is handed out once: the wait that reports *done = 1
  // releases it, and a later wait on the ticket is an argument error, like a wait on a
  // ticket this server never issued.
  int wait(uint64_t ticket, int32_t timeout_ms, int32_t* done, ep2d_result* res, double* lat, double* queue) {
    std::unique_lock<std::mutex> lk(mu_);
    if (done) *done = 0;
    if (!outstanding_.count(ticket)) return fail(EP2D_ERR_ARG, "unknown ticket, or its result was already collected");
    auto ready = [&] { return done_.count(ticket) > 0 || !init_ok_ || !outstanding_.count(ticket); };
    if (timeout_ms < 0) cv_.wait(lk, ready);
    else cv_.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready);
    auto it = done_.find(ticket);
    if (it == done_.end()) {
      if (!outstanding_.count(ticket)) return fail(EP2D_ERR_ARG, "the result was collected by another wait");
      return init_ok_ ? EP2D_OK : fail(EP2D_ERR_STATE, "server stopped");
    }
    const Task t = it->second;
    done_.erase(it);
    outstanding_.erase(ticket);
    if (done) *done = 1;
    if (res) *res = t.result;
    if (lat) *lat = t.done_s - t.submit_s;
    if (queue) *queue = t.admit_s - t.submit_s;
    return t.status == EP2D_OK ? EP2D_OK : fail(t.status, "request failed: " + t.error);
  }
  void stats(int64_t* sub, int64_t* adm, int64_t* fin, int64_t* bytes, ep2d_batch_stats* es) {
    std::lock_guard<std::mutex> lk(mu_);
    if (sub) *sub = submitted_;
    if (adm) *adm = admitted_;
    if (fin) *fin = finished_;
    if (bytes) *bytes = (int64_t)bytes_snapshot_;
    if (es) *es = stats_snapshot_;
  }

 private:
  void loop(ep2d_batch_config c) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      init_rc_ = eng_.init(c);
      init_ok_ = init_rc_ == EP2D_OK;
      started_ = true;
      if (!init_ok_) init_msg_ = last_error();
    }
    cv_.notify_all();
    if (!init_ok_) return;
    // host-side fault injection for tests: EP2D_SERVER_FAIL_AFTER = k makes the worker treat
    // its k-th checkpoint interval as failed (status EP2D_ERR_CUDA), without touching the GPU
    const char* inj = std::getenv("EP2D_SERVER_FAIL_AFTER");
    const int64_t fail_after = inj ? std::atoll(inj) : 0;
    int64_t intervals = 0;
    while (true) {
      std::vector<Task> admit;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return stop_ || !pending_.empty() || !eng_.idle(); });
        if (stop_) break;
        size_t bytes = eng_.bytes_in_use();
        int act = eng_.active();
        while (!pending_.empty() && act < max_active_) {
          const size_t need = eng_.footprint(pending_.front().spec);
          if ((int64_t)(bytes + need) > budget_ && act > 0) break;  // wait for memory to free up
          admit.push_back(pending_.front());
          pending_.pop_front();
          bytes += need;
          act++;
        }
      }
      for (auto& t : admit) {
        const int rc = eng_.add(t.spec, t.ticket, t.submit_s, nullptr);
        std::lock_guard<std::mutex> lk(mu_);
        if (rc) {
          t.status = rc;
          t.error = last_error();
          t.done = true;
          t.admit_s = t.done_s = now_s();
          done_[t.ticket] = t;
          finished_++;
        } else {
          admitted_++;
        }
      }
      // An interval that fails leaves the engine's state unknown (a CUDA error may have
      // ended the context): every active and queued request fails with its status, and
      // the server stops taking requests.
      int rc = EP2D_OK;
      if (!eng_.idle()) {
        rc = eng_.run_interval();
        intervals++;
        if (rc == EP2D_OK && fail_after > 0 && intervals >= fail_after)
          rc = fail(EP2D_ERR_CUDA, "injected failure of checkpoint interval " + std::to_string(intervals));
        if (rc) eng_.abort_all(rc, last_error());
      }
      std::vector<Task> fin = eng_.take_finished();
      {
        std::lock_guard<std::mutex> lk(mu_);
        for (auto& t : fin) {
          done_[t.ticket] = t;
          finished_++;
        }
        if (rc) {
          stop_msg_ = last_error();
          init_ok_ = false;  // no request is accepted from here on
          for (auto& t : pending_) {
            t.status = rc;
            t.error = stop_msg_;
            t.done = true;
            t.admit_s = t.done_s = now_s();
            done_[t.ticket] = t;
            finished_++;
          }
          pending_.clear();
        }
        bytes_snapshot_ = eng_.bytes_in_use();
        stats_snapshot_.kernel_ms = eng_.kernel_ms;
        stats_snapshot_.launches = eng_.launches;
        stats_snapshot_.all_launches = eng_.launches + eng_.aux_launches;
        stats_snapshot_.cell_updates = eng_.cell_updates;
        eng_.fill_stats(&stats_snapshot_);
      }
      if (!fin.empty() || rc) cv_.notify_all();
      if (rc) break;
    }
    std::lock_guard<std::mutex> lk(mu_);
    init_ok_ = false;
    cv_.notify_all();
  }

  BatchEngine eng_;
  std::thread worker_;
  std::mutex mu_;
  std::condition_variable cv_;
  std::deque<Task> pending_;
  std::map<uint64_t, Task> done_;
  std::set<uint64_t> outstanding_;  // issued tickets whose result has not been collected
  std::string stop_msg_;            // why the worker stopped, if it failed
  uint64_t next_ticket_ = 0;
  int64_t budget_ = 0;
  int max_active_ = 0;
  int64_t submitted_ = 0, admitted_ = 0, finished_ = 0;
  size_t bytes_snapshot_ = 0;
  ep2d_batch_stats stats_snapshot_{};
  bool started_ = false, init_ok_ = false, stop_ = false;
  int init_rc_ = EP2D_OK;
  std::string init_msg_;
};

}  // namespace ep2d

using ep2d::fail;

struct ep2d_server {
  ep2d::Server srv;
};

extern "C" {

int64_t ep2d_rve_footprint(const ep2d_rve_spec* spec, int32_t precision) {
  if (!spec) return -1;
  ep2d_batch_config c{};
  c.check_every = 2;
  c.niter = 2;
  c.precision = precision;
  return (int64_t)ep2d::Rve::footprint(ep2d::params_of(c, *spec));
}

int ep2d_batch_solve(const ep2d_batch_config* cfg, const ep2d_rve_spec* specs, int32_t n, ep2d_result* results,
                     ep2d_batch_stats* stats) {
  if (!cfg || (!specs && n > 0) || n < 0) return fail(EP2D_ERR_ARG, "null argument");
  try {
    const double t0 = ep2d::now_s();
    ep2d::BatchEngine eng;
    int rc = eng.init(*cfg);
    if (rc) return rc;
    size_t need = 0;
    for (int k = 0; k < n; k++) {
      rc = ep2d::validate_params(ep2d::params_of(*cfg, specs[k]));
      if (rc) return rc;
      need += eng.footprint(specs[k]);
    }
    size_t free_b = 0, total_b = 0;
    {
      ep2d::DeviceScope ds(cfg->device);
      if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess && need > free_b)
        return fail(EP2D_ERR_NOMEM, "the batch needs " + std::to_string(need) + " bytes, " + std::to_string(free_b) +
                                        " are free; use the server for progressive admission");
    }
    for (int k = 0; k < n; k++) {
      rc = eng.add(specs[k], (uint64_t)k, t0, nullptr);
      if (rc) return rc;
    }
    std::vector<ep2d::Task> done;
    while (!eng.idle()) {
      rc = eng.run_interval();
      if (rc) return rc;
      for (auto& t : eng.take_finished()) done.push_back(t);
    }
    for (auto& t : eng.take_finished()) done.push_back(t);
    int status = EP2D_OK;
    for (auto& t : done) {
      if (results) results[t.ticket] = t.result;
      if (t.status && !status) status = t.status;
    }
    if (stats) {
      std::memset(stats, 0, sizeof(*stats));
      stats->kernel_ms = eng.kernel_ms;
      stats->wall_ms = 1000.0 * (ep2d::now_s() - t0);
      stats->launches = eng.launches;
      stats->all_launches = eng.launches + eng.aux_launches;
      stats->cell_updates = eng.cell_updates;
      eng.fill_stats(stats);
    }
    return status ? fail(status, "a batch member failed") : EP2D_OK;
  } catch (const std::exception& ex) {
    return fail(EP2D_ERR_STATE, std::string("exception: ") + ex.what());
  }
}

int ep2d_server_create(const ep2d_batch_config* cfg, int64_t mem_budget_bytes, int32_t max_active, ep2d_server** out) {
  if (!cfg || !out) return fail(EP2D_ERR_ARG, "null argument");
  *out = nullptr;
  try {
    ep2d_server* s = new ep2d_server();
    const int rc = s->srv.start(*cfg, mem_budget_bytes, max_active);
    if (rc) {
      s->srv.stop();
      delete s;
      return rc;
    }
    *out = s;
    return EP2D_OK;
  } catch (const std::exception& ex) {
    return fail(EP2D_ERR_STATE, std::string("exception: ") + ex.what());
  }
}

int ep2d_server_submit(ep2d_server* s, const ep2d_rve_spec* spec, uint64_t* ticket_out) {
  if (!s || !spec) return fail(EP2D_ERR_ARG, "null argument");
  const int rc = ep2d::validate_params([&] {
    ep2d_batch_config c{};
    c.check_every = 2;
    c.niter = 2;
    return ep2d::params_of(c, *spec);
  }());
  if (rc) return rc;
  return s->srv.submit(*spec, ticket_out);
}

int ep2d_server_wait(ep2d_server* s, uint64_t ticket, int32_t timeout_ms, int32_t* done, ep2d_result* result,
                     double* latency_s, double* queue_s) {
  if (!s) return fail(EP2D_ERR_ARG, "null server");
  return s->srv.wait(ticket, timeout_ms, done, result, latency_s, queue_s);
}

int ep2d_server_stats(ep2d_server* s, int64_t* submitted, int64_t* admitted, int64_t* finished, int64_t* bytes_in_use,
                      ep2d_batch_stats* engine) {
  if (!s) return fail(EP2D_ERR_ARG, "null server");
  s->srv.stats(submitted, admitted, finished, bytes_in_use, engine);
  return EP2D_OK;
}

int ep2d_server_destroy(ep2d_server* s) {
  if (!s) return EP2D_OK;
  s->srv.stop();
  delete s;
  return EP2D_OK;
}

}  // extern "C"
