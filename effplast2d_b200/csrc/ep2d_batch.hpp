// ep2d_batch.hpp -- many RVEs on one B200: batched persistent iteration under a CUDA
// graph and the continuous-batching engine the server uses.
//
// Every RVE runs its own ComputeEffModuli chain (EffPlast2D.cu:179-229): preload time
// steps, then the load increments, each iterated until the reference's convergence
// test passes at one of its checkpoints.  All active RVEs iterate in lockstep, one
// batched launch per pseudo-time iteration; an RVE only joins at a checkpoint boundary,
// so its checkpoints fall at the same launches as everybody else's and each RVE sees
// exactly the reference's cadence (check every check_every iterations of its own time
// step).  At a checkpoint, one recording launch folds every RVE's max|V| into a
// per-RVE slot, one copy brings all of them to the host, and RVEs that converged (or
// reached NITER) are post-processed, advanced to their next time step, or retired.
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include "ep2d.h"
#include "ep2d_rve.hpp"

namespace ep2d {

struct Task {
  ep2d_rve_spec spec{};
  int step = 0, it = 0;        // current load step and time step
  int64_t iters = 0;           // iterations of the current time step
  bool done = false;
  int status = EP2D_OK;
  ep2d_result result{};
  std::string error;           // why it failed (status != EP2D_OK)
  uint64_t ticket = 0;
  double submit_s = 0.0, admit_s = 0.0, done_s = 0.0;  // host clock (server latency)
};

class BatchEngine {
 public:
  BatchEngine() = default;
  ~BatchEngine();
  BatchEngine(const BatchEngine&) = delete;
  BatchEngine& operator=(const BatchEngine&) = delete;

  int init(const ep2d_batch_config& cfg);
  // admit one RVE (allocates its fields, applies the first preload); returns its slot
  int add(const ep2d_rve_spec& spec, uint64_t ticket, double submit_s, int* slot);
  // one checkpoint interval (check_every iterations) for every active RVE
  int run_interval();
  int active() const;
  bool idle() const { return active() == 0; }
  // finished tasks since the last call (slot memory released)
  std::vector<Task> take_finished();
  // end every active RVE with `status` (slot memory released); they go to take_finished()
  void abort_all(int status, const std::string& error);
  size_t footprint(const ep2d_rve_spec& s) const;
  size_t bytes_in_use() const { return bytes_; }

  ep2d_batch_config cfg{};
  int device = 0;
  cudaStream_t stream = nullptr;
  // statistics
  double kernel_ms = 0.0;
  int64_t launches = 0, aux_launches = 0, cell_updates = 0;
  IterShape shape{};  // kernel form and rows of the batched launches
  int blocks = 0;
  bool tuned = false;
  int n_tuned = 0;   // candidates of the latest tuning run
  int n_tunes = 0;   // tuning runs
  int solo_intervals = 0;  // checkpoint intervals an RVE ran through the single-RVE path
  double tune_us[7] = {0, 0, 0, 0, 0, 0, 0};  // tile rows 8/16/32, stream rows 8/16/32/64
  void fill_stats(ep2d_batch_stats* st) const;

 private:
  struct Slot {
    std::unique_ptr<Rve> rve;
    Task task;
    bool used = false;
    bool solo = false;  // fills the GPU alone: runs through the single-RVE path
  };
  int begin_task_step(Slot& s);
  int advance(Slot& s, double error);  // after a checkpoint of this slot's time step
  int rebuild_tiles();  // the work list: tiles or strip segments of every active RVE
  int ensure_graph();
  int launch_plain_run(int64_t k0, int64_t n);
  bool fills_gpu(const Rve& r) const;  // the RVE keeps the GPU busy on its own
  int run_solo_launches(int slot);     // one checkpoint interval through the single-RVE path
  void finish_interval(const std::vector<char>& batched);  // every active RVE's checkpoint
  int autotune(int64_t* k, int64_t n_avail);
  int grow(int need);

  std::vector<Slot> slots_;
  std::vector<Task> finished_;
  size_t bytes_ = 0;
  bool tiles_dirty_ = true;
  int n_tiles_ = 0;
  BatchEntry* d_ents_ = nullptr;
  int2* d_tiles_ = nullptr;
  int* d_ntiles_ = nullptr;
  unsigned long long* d_vmax_ = nullptr;
  unsigned long long* h_vmax_ = nullptr;
  int cap_slots_ = 0, cap_tiles_ = 0;
  uint64_t set_version_ = 0;    // bumped whenever an RVE joins or retires
  uint64_t tuned_version_ = 0;  // set_version_ the current shape was tuned for
  cudaGraphExec_t graph_ = nullptr;
  IterShape graph_shape_{};
  cudaEvent_t ev_[2] = {nullptr, nullptr};
  int sm_count_ = 148;
};

}  // namespace ep2d
