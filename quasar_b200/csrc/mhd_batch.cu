// Batched MHD step (see mhd_batch.cuh).
#include "mhd_batch.cuh"
#include "indicator.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <numeric>
#include <stdexcept>
#include <string>

namespace qb {

namespace {

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

double bits_to_double(unsigned long long b) {
  double d;
  std::memcpy(&d, &b, sizeof d);
  return d;
}

constexpr double kInfT = std::numeric_limits<double>::infinity();
constexpr int kChunk = 32;  // graph steps between host checks in advance()

}  // namespace

MhdBatch2D::MhdBatch2D(const std::vector<Config>& configs) {
  if (configs.empty()) throw std::invalid_argument("MhdBatch2D: at least one instance is required");
  order_ = configs[0].order;
  if (order_ != 5 && order_ != 7)
    throw std::invalid_argument("MhdBatch2D: batched stepping supports mp5 and mp7");
  for (const Config& c : configs)
    if (c.order != order_)
      throw std::invalid_argument("MhdBatch2D: every instance must use the same reconstruction");
  for (const Config& c : configs) inst_.emplace_back(new MhdSolver2D(c));
  const int n = size();
  slot_.resize(size_t(n));
  std::iota(slot_.begin(), slot_.end(), 0);
  std::stable_sort(slot_.begin(), slot_.end(), [&](int a, int b) {
    const Grid& ga = inst_[size_t(a)]->grid();
    const Grid& gb = inst_[size_t(b)]->grid();
    return (long long)ga.nx * ga.ny > (long long)gb.nx * gb.ny;
  });
  int dev = 0;
  ck(cudaGetDevice(&dev), "device");
  ck(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, dev), "SM count");
  ck(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream");
  ck(cudaMalloc(&recs_, sizeof(BatchRec) * 6 * size_t(n)), "batch records");
  ck(cudaMalloc(&prefix_, sizeof(int) * kBpAll * size_t(n + 1)), "batch plans");
  max_ctas_.resize(kBpCount);
  ctas_per_sm_.resize(kBpCount);
  for (int ph = 0; ph < kBpCount; ++ph) {
    max_ctas_[ph] = batch_phase_max_ctas_per_sm(ph, order_);
    ctas_per_sm_[ph] = max_ctas_[ph];
  }
  build_plans();
}

MhdBatch2D::~MhdBatch2D() {
  release_graphs();
  if (stream_) cudaStreamSynchronize(stream_);
  cudaFree(recs_);
  cudaFree(prefix_);
  cudaFree(learn_);
  cudaFree(ind_status_);
  if (stream_) cudaStreamDestroy(stream_);
}

long long MhdBatch2D::zones() const {
  long long z = 0;
  for (const auto& s : inst_) z += (long long)s->grid().nx * s->grid().ny;
  return z;
}

void MhdBatch2D::set_tuning(const std::vector<int>& ctas) {
  if (ctas.size() != size_t(kBpCount))
    throw std::invalid_argument("MhdBatch2D: tuning needs one entry per phase");
  for (int ph = 0; ph < kBpCount; ++ph)
    if (ctas[ph] < 0 || ctas[ph] > max_ctas_[ph])
      throw std::invalid_argument("MhdBatch2D: CTAs per SM outside [0, occupancy limit]");
  ctas_per_sm_ = ctas;
  build_plans();
  release_graphs();
}

void MhdBatch2D::build_plans() {
  const int n = size();
  std::vector<int> h(size_t(kBpAll) * (n + 1));
  for (int ph = 0; ph < kBpAll; ++ph) {
    int* p = h.data() + size_t(ph) * (n + 1);
    long long acc = 0;
    for (int s = 0; s < n; ++s) {
      p[s] = int(acc);
      int tx, ty;
      batch_tiles(ph, inst_[size_t(slot_[size_t(s)])]->grid(), &tx, &ty);
      acc += (long long)tx * ty;
    }
    if (acc > std::numeric_limits<int>::max())
      throw std::invalid_argument("MhdBatch2D: batch too large for one launch");
    p[n] = int(acc);
    const int total = int(acc);
    const int c = ph < kBpCount ? ctas_per_sm_[size_t(ph)] : 0;
    plan_[ph].prefix = prefix_ + size_t(ph) * (n + 1);
    plan_[ph].n = n;
    plan_[ph].total = total;
    plan_[ph].grid = c == 0 ? total : std::min(total, c * sms_);
  }
  ck(cudaMemcpy(prefix_, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice), "plans");
}

// Stage records of both parities: parity 0 takes each instance's current
// live register as U^n, parity 1 the one its next step writes.
void MhdBatch2D::build_tables() {
  const int n = size();
  std::vector<BatchRec> h(6 * size_t(n));
  for (int s = 0; s < n; ++s) {
    MhdSolver2D& m = *inst_[size_t(slot_[size_t(s)])];
    const double eff = std::min(m.cfg_.cfl, 0.2);
    for (int par = 0; par < 2; ++par) {
      const int live = par == 0 ? m.live_ : m.next_;
      const int nxt = par == 0 ? m.next_ : m.live_;
      const int in[3] = {live, m.s1_, m.s2_};
      const int out[3] = {m.s1_, m.s2_, nxt};
      for (int st = 0; st < 3; ++st) {
        BatchRec& r = h[size_t(par * 3 + st) * n + s];
        r.a = m.stage_args(m.st_[in[st]], order_);
        r.live = m.st_[live];
        r.out = m.st_[out[st]];
        r.cfl_eff = eff;
        r.hmin = std::min(m.g_.dx, m.g_.dy);
        r.hmax = std::max(m.g_.dx, m.g_.dy);
      }
    }
  }
  ck(cudaMemcpyAsync(recs_, h.data(), sizeof(BatchRec) * h.size(), cudaMemcpyHostToDevice,
                     stream_),
     "records");
  ck(cudaStreamSynchronize(stream_), "records");
}

void MhdBatch2D::set_indicator(const Indicator* ind, float threshold) {
  if (ind && !ind_status_) {
    ck(cudaMalloc(&ind_status_, sizeof(int)), "indicator status");
    ck(cudaMemset(ind_status_, 0, sizeof(int)), "indicator status");
    ck(cudaMalloc(&learn_, sizeof(BatchLearnRec) * size_t(size())), "learned records");
  }
  for (auto& m : inst_) m->set_indicator(ind, threshold);
  if (ind) {
    std::vector<BatchLearnRec> h(static_cast<size_t>(size()));
    for (int s = 0; s < size(); ++s) {
      MhdSolver2D& m = *inst_[size_t(slot_[size_t(s)])];
      h[size_t(s)] = BatchLearnRec{m.flags_, m.flists_, m.flists_ + m.g_.size(), m.fcounts_};
    }
    ck(cudaMemcpy(learn_, h.data(), sizeof(BatchLearnRec) * h.size(), cudaMemcpyHostToDevice),
       "learned records");
  }
  ind_ = ind;
  ind_threshold_ = threshold;
  release_graphs();
}

void MhdBatch2D::prepare() {
  for (auto& m : inst_) {
    m->ensure_live_ready();
    m->front_order_ = 0;
  }
  for (auto& m : inst_) ck(cudaStreamSynchronize(m->stream()), "instance stream");
  build_tables();
}

// One SSP-RK3 step of every instance (the sequence of MhdSolver2D's
// front_impl(order, 2, -1) + finish_impl(order, &ctl->dt, 0, true)).
void MhdBatch2D::enqueue_step(int par, std::vector<cudaEvent_t>* marks,
                              std::vector<int>* phases) {
  const int n = size();
  auto mark = [&](int ph) {
    if (!marks) return;
    cudaEvent_t e;
    ck(cudaEventCreate(&e), "event");
    ck(cudaEventRecord(e, stream_), "event record");
    marks->push_back(e);
    phases->push_back(ph);
  };
  launch_batch_ctl(recs(par, 0), n, 0, 0.0, 0.0, stream_);
  mark(-1);
  if (ind_) {
    // score every instance's live state once per step
    launch_batch_learned_reset(recs(par, 0), learn_, plan_[kBpCells], stream_);
    ck(launch_batch_indicator(recs(par, 0), learn_, plan_[kBpInd], ind_->dev(), ind_threshold_,
                              ind_status_, stream_),
       "batched indicator");
    launch_batch_face_lists(recs(par, 0), learn_, plan_[kBpCells], stream_);
    mark(-1);
  }
  for (int st = 0; st < 3; ++st) {
    const BatchRec* r = recs(par, st);
    const bool first = st == 0;
    if (ind_) {
      launch_batch_reconstruct_learned(r, learn_, plan_[kBpRecon0], 0, order_, 4 * sms_, stream_);
      mark(kBpRecon0);
      launch_batch_reconstruct_learned(r, learn_, plan_[kBpRecon1], 1, order_, 4 * sms_, stream_);
      mark(kBpRecon1);
    } else {
      launch_batch_reconstruct(r, plan_[kBpRecon0], 0, order_, stream_);
      mark(kBpRecon0);
      launch_batch_reconstruct(r, plan_[kBpRecon1], 1, order_, stream_);
      mark(kBpRecon1);
    }
    launch_batch_face_flux(r, plan_[kBpFlux], 0, order_, first, stream_);
    launch_batch_face_flux(r, plan_[kBpFlux], 1, order_, first, stream_);
    mark(kBpFlux);
    launch_batch_cell_emf(r, plan_[kBpCell], order_, first, stream_);
    mark(kBpCell);
    launch_batch_corner_emf(r, plan_[kBpCorner], order_, stream_);
    mark(kBpCorner);
    if (first) {
      launch_batch_ctl(r, n, 1, 0.0, 0.0, stream_);
      mark(-1);
    }
    launch_batch_update(r, plan_[kBpUpdate], st, stream_);
    mark(kBpUpdate);
    launch_batch_fill_ghosts(r, plan_[kBpFill0], 0, stream_);
    mark(kBpFill0);
    launch_batch_fill_ghosts(r, plan_[kBpFill1], 1, stream_);
    mark(kBpFill1);
    launch_batch_colloc_check(r, plan_[kBpColloc], order_, st == 2 ? (1 | 4) : 1, st == 2,
                              stream_);
    mark(kBpColloc);
  }
  launch_batch_ctl(recs(par, 0), n, 2, 0.0, 0.0, stream_);
  mark(-1);
  ck(cudaGetLastError(), "batched step launch");
}

void MhdBatch2D::ensure_graphs() {
  if (graph_[0]) return;
  for (int par = 0; par < 2; ++par) {
    cudaGraph_t g;
    ck(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "capture");
    try {
      enqueue_step(par, nullptr, nullptr);
    } catch (...) {
      cudaStreamEndCapture(stream_, &g);
      throw;
    }
    ck(cudaStreamEndCapture(stream_, &g), "capture end");
    ck(cudaGraphInstantiate(&graph_[par], g, 0), "graph instantiate");
    cudaGraphDestroy(g);
  }
}

void MhdBatch2D::release_graphs() {
  for (auto& g : graph_) {
    if (g) cudaGraphExecDestroy(g);
    g = nullptr;
  }
}

// After a chunk: promote every accepted step; an instance stopped by a
// positivity retry completes that step with its own host controller.
void MhdBatch2D::collect(int* done) {
  for (int i = 0; i < size(); ++i) {
    MhdSolver2D& m = *inst_[size_t(i)];
    const Ctl c = m.read_ctl();
    for (int s = 0; s < c.steps_done; ++s) m.promote();
    int taken = c.steps_done;
    try {
      if (c.status & kStatusRetry) {
        m.controller(c.dt, bits_to_double(c.theta), c.anchor_ok != 0);
        ++taken;
      } else if (c.status & ~kStatusDone) {
        m.throw_status(c.status);
      }
    } catch (const std::invalid_argument& e) {
      throw std::invalid_argument("MhdBatch2D instance " + std::to_string(i) + ": " + e.what());
    } catch (const CudaError&) {
      throw;
    } catch (const std::exception& e) {
      throw std::runtime_error("MhdBatch2D instance " + std::to_string(i) + ": " + e.what());
    }
    if (done) done[i] += taken;
  }
}

void MhdBatch2D::advance(int steps, int* done) {
  if (done) std::fill(done, done + size(), 0);
  int left = steps;
  while (left > 0) {
    const int chunk = std::min(left, kChunk);
    prepare();
    ensure_graphs();
    launch_batch_ctl(recs(0, 0), size(), 3, 0.0, kInfT, stream_);
    for (int k = 0; k < chunk; ++k) ck(cudaGraphLaunch(graph_[k & 1], stream_), "graph launch");
    ck(cudaStreamSynchronize(stream_), "batched steps");
    collect(done);
    left -= chunk;
  }
}

double MhdBatch2D::time_steps(int steps, long long* zone_updates) {
  prepare();
  ensure_graphs();
  launch_batch_ctl(recs(0, 0), size(), 3, 0.0, kInfT, stream_);
  cudaEvent_t a, b;
  ck(cudaEventCreate(&a), "event");
  ck(cudaEventCreate(&b), "event");
  ck(cudaEventRecord(a, stream_), "event record");
  for (int k = 0; k < steps; ++k) ck(cudaGraphLaunch(graph_[k & 1], stream_), "graph launch");
  ck(cudaEventRecord(b, stream_), "event record");
  ck(cudaStreamSynchronize(stream_), "batched steps");
  float ms = 0.f;
  ck(cudaEventElapsedTime(&ms, a, b), "elapsed");
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  long long zu = 0;
  for (int i = 0; i < size(); ++i) {
    MhdSolver2D& m = *inst_[size_t(i)];
    const Ctl c = m.read_ctl();
    zu += (long long)m.grid().nx * m.grid().ny * c.steps_done;
  }
  collect(nullptr);
  if (zone_updates) *zone_updates = zu;
  return double(ms);
}

std::vector<double> MhdBatch2D::profile_step() {
  prepare();
  launch_batch_ctl(recs(0, 0), size(), 3, 0.0, kInfT, stream_);
  cudaEvent_t start;
  ck(cudaEventCreate(&start), "event");
  ck(cudaEventRecord(start, stream_), "event record");
  std::vector<cudaEvent_t> marks;
  std::vector<int> phases;
  enqueue_step(0, &marks, &phases);
  ck(cudaStreamSynchronize(stream_), "profiled step");
  std::vector<double> per(kBpCount + 1, 0.0);
  cudaEvent_t prev = start;
  for (size_t k = 0; k < marks.size(); ++k) {
    float e = 0.f;
    ck(cudaEventElapsedTime(&e, prev, marks[k]), "elapsed");
    per[phases[k] >= 0 ? size_t(phases[k]) : size_t(kBpCount)] += e;
    prev = marks[k];
  }
  for (cudaEvent_t e : marks) cudaEventDestroy(e);
  cudaEventDestroy(start);
  collect(nullptr);
  return per;
}

int MhdBatch2D::autotune() {
  // candidates per phase: every CTAs-per-SM count up to the occupancy limit,
  // then one CTA per tile (0)
  std::vector<std::vector<int>> cand(kBpCount);
  size_t trials = 0;
  for (int ph = 0; ph < kBpCount; ++ph) {
    for (int c = max_ctas_[ph]; c >= 1; --c) cand[ph].push_back(c);
    cand[ph].push_back(0);
    trials = std::max(trials, cand[ph].size());
  }
  std::vector<std::vector<double>> ms(kBpCount);
  int taken = 0;
  for (size_t t = 0; t <= trials; ++t) {  // trial 0 warms up with the current tuning
    std::vector<int> pick = ctas_per_sm_;
    if (t > 0)
      for (int ph = 0; ph < kBpCount; ++ph) pick[ph] = cand[ph][std::min(t - 1, cand[ph].size() - 1)];
    ctas_per_sm_ = pick;
    build_plans();
    prepare();
    launch_batch_ctl(recs(0, 0), size(), 3, 0.0, kInfT, stream_);
    cudaEvent_t start;
    ck(cudaEventCreate(&start), "event");
    ck(cudaEventRecord(start, stream_), "event record");
    std::vector<cudaEvent_t> marks;
    std::vector<int> phases;
    enqueue_step(0, &marks, &phases);
    ck(cudaStreamSynchronize(stream_), "profiled step");
    std::vector<double> per(kBpCount, 0.0);
    cudaEvent_t prev = start;
    for (size_t k = 0; k < marks.size(); ++k) {
      float e = 0.f;
      ck(cudaEventElapsedTime(&e, prev, marks[k]), "elapsed");
      if (phases[k] >= 0) per[size_t(phases[k])] += e;
      prev = marks[k];
    }
    for (cudaEvent_t e : marks) cudaEventDestroy(e);
    cudaEventDestroy(start);
    collect(nullptr);
    ++taken;
    if (t > 0)
      for (int ph = 0; ph < kBpCount; ++ph)
        if (t - 1 < cand[ph].size()) ms[ph].push_back(per[size_t(ph)]);
  }
  std::vector<int> best(kBpCount);
  for (int ph = 0; ph < kBpCount; ++ph) {
    const auto it = std::min_element(ms[ph].begin(), ms[ph].end());
    best[ph] = cand[ph][size_t(it - ms[ph].begin())];
  }
  ctas_per_sm_ = best;
  build_plans();
  release_graphs();
  return taken;
}

}  // namespace qb
