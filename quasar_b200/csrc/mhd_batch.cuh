// Batched MHD step: many independent instances (uneven grids, own gamma and
// boundaries, one reconstruction order) advanced together, one persistent
// launch per phase of every RK stage, the whole step captured in a CUDA graph.
//
// Each instance is a full MhdSolver2D (its own arena, seeding, preflights,
// diagnostics and positivity controller); the batch only replaces the
// per-instance stage launches by batched ones over tables of the instances'
// stage arguments.  Persistent grid sizes per phase come from autotune(),
// which times real profiled steps of the batch itself.
#pragma once

#include "mhd_kernels.cuh"
#include "mhd_solver.cuh"

#include <memory>
#include <vector>

namespace qb {

class MhdBatch2D {
 public:
  explicit MhdBatch2D(const std::vector<Config>& configs);
  ~MhdBatch2D();
  MhdBatch2D(const MhdBatch2D&) = delete;
  MhdBatch2D& operator=(const MhdBatch2D&) = delete;

  int size() const { return int(inst_.size()); }
  MhdSolver2D& instance(int i) { return *inst_.at(size_t(i)); }
  long long zones() const;

  // `steps` auto-dt steps of every instance without host round trips inside
  // a chunk.  An instance whose candidate the positivity controller must
  // retry stops in that chunk; its step is then completed by its own
  // controller on the host.  done[i] (optional) = steps taken by instance i.
  void advance(int steps, int* done);

  // Device time of `steps` batched steps (CUDA events on the batch stream);
  // *zone_updates = sum over instances of zones x steps taken.
  double time_steps(int steps, long long* zone_updates);

  // Choose each phase's persistent grid (CTAs per SM, or one CTA per tile)
  // from profiled batched steps; every instance advances by the steps used.
  // Returns the number of profiled steps taken.
  int autotune();
  // per phase: CTAs per SM of the persistent grid, 0 = one CTA per tile
  const std::vector<int>& tuning() const { return ctas_per_sm_; }
  void set_tuning(const std::vector<int>& ctas_per_sm);
  // One step with per-phase device times in ms: kBpCount tuned phases, then
  // the control kernels (and in learned mode the indicator and face lists).
  std::vector<double> profile_step();

  // Learned troubled-cell mode for every instance (batched indicator, face
  // lists and two-pass reconstruction inside the batched step); nullptr
  // returns to the plain step.  The indicator must outlive its use.
  void set_indicator(const Indicator* ind, float threshold);

 private:
  void prepare();                 // instance preflights, tables, plans
  void build_tables();
  void build_plans();
  void enqueue_step(int parity, std::vector<cudaEvent_t>* marks, std::vector<int>* phases);
  void ensure_graphs();
  void release_graphs();
  void collect(int* done);        // promote / retry per instance after a chunk
  const BatchRec* recs(int parity, int stage) const {
    return recs_ + size_t(parity * 3 + stage) * inst_.size();
  }

  std::vector<std::unique_ptr<MhdSolver2D>> inst_;
  std::vector<int> slot_;         // table slot -> instance (largest first)
  int order_ = 5;
  int sms_ = 148;
  cudaStream_t stream_ = nullptr;
  BatchRec* recs_ = nullptr;      // device [parity 2][stage 3][slot]
  int* prefix_ = nullptr;         // device [phase][slot + 1]
  BatchPlan plan_[kBpAll];
  std::vector<int> ctas_per_sm_;  // per phase
  std::vector<int> max_ctas_;     // per phase, occupancy limit
  cudaGraphExec_t graph_[2] = {nullptr, nullptr};
  // learned mode
  const Indicator* ind_ = nullptr;
  float ind_threshold_ = 0.f;
  BatchLearnRec* learn_ = nullptr;  // device, slot order
  int* ind_status_ = nullptr;
};

}  // namespace qb
