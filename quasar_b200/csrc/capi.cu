// extern "C" boundary over qb::MhdSolver2D (declarations: include/quasar_mhd.h).
#include "../../include/quasar_mhd.h"
#include "../../include/quasar_mhd_ext.h"
#include "../../include/quasar_mhd_batch.h"
#include "../../include/quasar_mhd_indicator.h"
#include "indicator.cuh"
#include "mhd_batch.cuh"
#include "mhd_solver.cuh"
#include "noalloc.cuh"

#include <cstdio>
#include <cstring>
#include <exception>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace qb {
double fp64_fma_peak_tflops();
}

// A solver handle: an owned solver, or a view of one instance of a batch
// (owned by the batch; destroying a view does nothing).
struct qmhd_solver {
  qb::MhdSolver2D* impl = nullptr;
  bool owned = false;
};

struct qmhd_indicator {
  qb::Indicator impl;
  explicit qmhd_indicator(unsigned long long seed) : impl(seed) {}
};

struct qmhd_batch {
  std::unique_ptr<qb::MhdBatch2D> impl;
  std::vector<qmhd_solver> views;
};

namespace {

thread_local std::string g_error;

template <class F>
int guarded(F&& f) {
  try {
    f();
    g_error.clear();
    return QMHD_OK;
  } catch (const qb::CudaError& e) {
    g_error = e.what();
    return QMHD_DEVICE_ERROR;
  } catch (const std::invalid_argument& e) {
    g_error = e.what();
    return QMHD_INVALID_ARGUMENT;
  } catch (const std::exception& e) {
    g_error = e.what();
    return QMHD_RUNTIME_ERROR;
  } catch (...) {
    g_error = "unknown error";
    return QMHD_RUNTIME_ERROR;
  }
}

// Component spellings of MhdSolver2D::component_buffer (mhd_solver.cpp:507-519).
// Reads of "bx"/"by" return the collocated field (indices 8/9).
int component_index(const char* name, bool for_read) {
  if (!name) throw std::invalid_argument("MhdSolver2D: unknown state component ''");
  const std::string c(name);
  if (c == "rho") return 0;
  if (c == "mx") return 1;
  if (c == "my") return 2;
  if (c == "mz") return 3;
  if (c == "energy") return 4;
  if (c == "bx") return for_read ? 8 : 5;
  if (c == "bx_face") return 5;
  if (c == "by") return for_read ? 9 : 6;
  if (c == "by_face") return 6;
  if (c == "bz" || c == "bz_cell") return 7;
  throw std::invalid_argument("MhdSolver2D: unknown state component '" + c + "'");
}

void need(const void* p) {
  if (!p) throw std::invalid_argument("qmhd: null pointer argument");
}

qb::Config to_config(const qmhd_config& q) {
  qb::Config c;
  c.nx = q.nx;
  c.ny = q.ny;
  c.lx = q.lx;
  c.ly = q.ly;
  c.ox = q.origin_x;
  c.oy = q.origin_y;
  c.order = q.reconstruction_order;
  c.gamma = q.gamma;
  c.cfl = q.cfl;
  for (int s = 0; s < 4; ++s) c.bc[s] = q.boundary[s];
  return c;
}

}  // namespace

namespace qb {
// Status code and thread-local message of f() under the C ABI's rules; the
// per-kernel launch interface (launch_abi.cu) reports through it.
int capi_guarded(const std::function<void()>& f) { return guarded(f); }
}  // namespace qb

extern "C" {

const char* qmhd_last_error(void) { return g_error.c_str(); }

int qmhd_solver_create(const qmhd_config* config, qmhd_solver** out) {
  return guarded([&] {
    need(config);
    need(out);
    *out = nullptr;
    std::unique_ptr<qb::MhdSolver2D> impl(new qb::MhdSolver2D(to_config(*config)));
    *out = new qmhd_solver{impl.release(), true};
  });
}

void qmhd_solver_destroy(qmhd_solver* solver) {
  if (!solver || !solver->owned) return;
  delete solver->impl;
  delete solver;
}

int qmhd_solver_grid(const qmhd_solver* s, int* nx, int* ny, int* nghost) {
  return guarded([&] {
    need(s);
    const qb::Grid& g = s->impl->grid();
    if (nx) *nx = g.nx;
    if (ny) *ny = g.ny;
    if (nghost) *nghost = g.ng;
  });
}

long long qmhd_solver_storage_size(const qmhd_solver* s) {
  return s ? s->impl->storage_size() : -1;
}

int qmhd_solver_seed_state(qmhd_solver* s, const char* component, const double* values,
                           size_t n) {
  return guarded([&] {
    need(s);
    need(values);
    s->impl->seed_state(component_index(component, false), values, (long long)n);
  });
}

int qmhd_solver_set_owned_window(qmhd_solver* s, int x0, int x1, int y0, int y1) {
  return guarded([&] {
    need(s);
    s->impl->set_owned_window(x0, x1, y0, y1);
  });
}

int qmhd_solver_write_halo(qmhd_solver* s, const char* component, const double* values,
                           size_t n) {
  return guarded([&] {
    need(s);
    need(values);
    s->impl->write_halo(component_index(component, false), values, (long long)n);
  });
}

int qmhd_solver_gather_live(qmhd_solver* s, const char* component, const long long* idx,
                            size_t n, double* out) {
  return guarded([&] {
    need(s);
    if (n > 0) {
      need(idx);
      need(out);
    }
    s->impl->gather_live(component_index(component, false), idx, (long long)n, out);
  });
}

int qmhd_solver_scatter_halo(qmhd_solver* s, const char* component, const long long* idx,
                             size_t n, const double* values) {
  return guarded([&] {
    need(s);
    if (n > 0) {
      need(idx);
      need(values);
    }
    s->impl->scatter_halo(component_index(component, false), idx, (long long)n, values);
  });
}

int qmhd_solver_state_component_to_host(qmhd_solver* s, const char* component, double* out,
                                        size_t n) {
  return guarded([&] {
    need(s);
    need(out);
    s->impl->state_component_to_host(component_index(component, true), out, (long long)n);
  });
}

int qmhd_solver_cfl_limit(qmhd_solver* s, double* dt) {
  return guarded([&] {
    need(s);
    need(dt);
    *dt = s->impl->cfl_limit();
  });
}

int qmhd_solver_step(qmhd_solver* s, double dt) {
  return guarded([&] {
    need(s);
    s->impl->step(dt);
  });
}

int qmhd_solver_step_unchecked(qmhd_solver* s, double dt) {
  return guarded([&] {
    need(s);
    s->impl->step_unchecked(dt);
  });
}

int qmhd_solver_advance(qmhd_solver* s, double t_end, double dt) {
  return guarded([&] {
    need(s);
    s->impl->advance(t_end, dt);
  });
}

int qmhd_solver_divergence_b_max(qmhd_solver* s, double* out) {
  return guarded([&] {
    need(s);
    need(out);
    *out = s->impl->divergence_b_max();
  });
}

int qmhd_solver_conserved_cell_totals(qmhd_solver* s, double* mass, double* energy) {
  return guarded([&] {
    need(s);
    need(mass);
    need(energy);
    s->impl->conserved_cell_totals(mass, energy);
  });
}

int qmhd_solver_last_positivity_substeps(const qmhd_solver* s) {
  return s ? s->impl->last_positivity_substeps() : -1;
}

int qmhd_solver_advance_auto(qmhd_solver* s, double* t, double t_end, int max_steps,
                             int* steps_taken) {
  return guarded([&] {
    need(s);
    need(t);
    const int n = s->impl->advance_auto(t, t_end, max_steps);
    if (steps_taken) *steps_taken = n;
  });
}

int qmhd_solver_time_auto_steps(qmhd_solver* s, int steps, double* ms, int* done) {
  return guarded([&] {
    need(s);
    need(ms);
    *ms = s->impl->time_auto_steps(steps, done);
  });
}

int qmhd_solver_profile_step(qmhd_solver* s, double* ms, int n) {
  return guarded([&] {
    need(s);
    need(ms);
    if (n < qb::MhdSolver2D::kPhases) throw std::invalid_argument("qmhd: phase buffer too small");
    s->impl->profile_step(ms);
  });
}

int qmhd_fp64_fma_peak(double* tflops) {
  return guarded([&] {
    need(tflops);
    *tflops = qb::fp64_fma_peak_tflops();
    if (!(*tflops > 0.0)) throw qb::CudaError("FP64 probe failed");
  });
}

// ---- batched instances (include/quasar_mhd_batch.h) ------------------------
int qmhd_batch_create(const qmhd_config* configs, int n, qmhd_batch** out) {
  return guarded([&] {
    need(configs);
    need(out);
    *out = nullptr;
    if (n < 1) throw std::invalid_argument("qmhd_batch_create: need at least one instance");
    std::vector<qb::Config> cfgs;
    for (int i = 0; i < n; ++i) cfgs.push_back(to_config(configs[i]));
    std::unique_ptr<qmhd_batch> b(new qmhd_batch);
    b->impl.reset(new qb::MhdBatch2D(cfgs));
    b->views.resize(size_t(n));
    for (int i = 0; i < n; ++i) b->views[size_t(i)] = qmhd_solver{&b->impl->instance(i), false};
    *out = b.release();
  });
}

void qmhd_batch_destroy(qmhd_batch* batch) { delete batch; }

int qmhd_batch_size(const qmhd_batch* batch) { return batch ? int(batch->views.size()) : -1; }

qmhd_solver* qmhd_batch_instance(qmhd_batch* batch, int i) {
  if (!batch || i < 0 || i >= int(batch->views.size())) return nullptr;
  return &batch->views[size_t(i)];
}

int qmhd_batch_advance(qmhd_batch* batch, int steps, int* steps_taken) {
  return guarded([&] {
    need(batch);
    if (steps < 0) throw std::invalid_argument("qmhd_batch_advance: steps must be >= 0");
    batch->impl->advance(steps, steps_taken);
  });
}

int qmhd_batch_time_steps(qmhd_batch* batch, int steps, double* ms, long long* zone_updates) {
  return guarded([&] {
    need(batch);
    need(ms);
    if (steps < 1) throw std::invalid_argument("qmhd_batch_time_steps: steps must be >= 1");
    *ms = batch->impl->time_steps(steps, zone_updates);
  });
}

int qmhd_batch_autotune(qmhd_batch* batch, int* ctas_per_sm, int* trial_steps) {
  return guarded([&] {
    need(batch);
    const int t = batch->impl->autotune();
    if (trial_steps) *trial_steps = t;
    if (ctas_per_sm)
      for (int ph = 0; ph < QMHD_BATCH_PHASES; ++ph) ctas_per_sm[ph] = batch->impl->tuning()[size_t(ph)];
  });
}

int qmhd_batch_profile_step(qmhd_batch* batch, double* ms_by_phase, int n) {
  return guarded([&] {
    need(batch);
    need(ms_by_phase);
    if (n < QMHD_BATCH_PHASES + 1)
      throw std::invalid_argument("qmhd_batch_profile_step: n must be >= QMHD_BATCH_PHASES + 1");
    const std::vector<double> per = batch->impl->profile_step();
    for (int ph = 0; ph <= QMHD_BATCH_PHASES; ++ph) ms_by_phase[ph] = per[size_t(ph)];
  });
}

int qmhd_batch_set_tuning(qmhd_batch* batch, const int* ctas_per_sm) {
  return guarded([&] {
    need(batch);
    need(ctas_per_sm);
    batch->impl->set_tuning(std::vector<int>(ctas_per_sm, ctas_per_sm + QMHD_BATCH_PHASES));
  });
}

long long qmhd_batch_zones(const qmhd_batch* batch) { return batch ? batch->impl->zones() : -1; }

int qmhd_batch_set_indicator(qmhd_batch* batch, const qmhd_indicator* ind, float threshold) {
  return guarded([&] {
    need(batch);
    batch->impl->set_indicator(ind ? &ind->impl : nullptr, threshold);
  });
}

static_assert(QMHD_BATCH_PHASES == qb::kBpCount, "phase count");

// ---- learned troubled-cell indicator (include/quasar_mhd_indicator.h) -----
static_assert(QMHD_INDICATOR_PARAMS == qb::kParamCount, "parameter count");

int qmhd_indicator_create(unsigned long long seed, qmhd_indicator** out) {
  return guarded([&] {
    need(out);
    *out = nullptr;
    *out = new qmhd_indicator(seed);
  });
}

void qmhd_indicator_destroy(qmhd_indicator* ind) { delete ind; }

int qmhd_indicator_get_params(qmhd_indicator* ind, float* params, size_t n) {
  return guarded([&] {
    need(ind);
    need(params);
    if (n != size_t(QMHD_INDICATOR_PARAMS))
      throw std::invalid_argument("qmhd_indicator_get_params: need QMHD_INDICATOR_PARAMS floats");
    ind->impl.get_params(params);
  });
}

int qmhd_indicator_set_params(qmhd_indicator* ind, const float* params, size_t n) {
  return guarded([&] {
    need(ind);
    need(params);
    if (n != size_t(QMHD_INDICATOR_PARAMS))
      throw std::invalid_argument("qmhd_indicator_set_params: need QMHD_INDICATOR_PARAMS floats");
    ind->impl.set_params(params);
  });
}

int qmhd_indicator_forward(qmhd_indicator* ind, const float* features, long long rows,
                           float* logits) {
  return guarded([&] {
    need(ind);
    need(features);
    need(logits);
    if (rows < 0) throw std::invalid_argument("qmhd_indicator_forward: rows must be >= 0");
    ind->impl.forward(features, rows, logits);
  });
}

int qmhd_indicator_gradient(qmhd_indicator* ind, const float* features,
                            const unsigned char* labels, long long rows, float pos_weight,
                            float* grad, size_t n, double* loss) {
  return guarded([&] {
    need(ind);
    need(features);
    need(labels);
    need(grad);
    if (n != size_t(QMHD_INDICATOR_PARAMS))
      throw std::invalid_argument("qmhd_indicator_gradient: need QMHD_INDICATOR_PARAMS floats");
    const double l = ind->impl.gradient(features, labels, rows, pos_weight, grad);
    if (loss) *loss = l;
  });
}

int qmhd_indicator_collect(qmhd_indicator* ind, qmhd_solver* solver, float tol) {
  return guarded([&] {
    need(ind);
    need(solver);
    ind->impl.collect(solver->impl->live_args(), solver->impl->stream(), tol);
  });
}

long long qmhd_indicator_rows(const qmhd_indicator* ind) { return ind ? ind->impl.rows() : -1; }

int qmhd_indicator_labels(const qmhd_indicator* ind, unsigned char* labels, long long n) {
  return guarded([&] {
    need(ind);
    need(labels);
    ind->impl.labels_to_host(labels, n);
  });
}

int qmhd_indicator_clear(qmhd_indicator* ind) {
  return guarded([&] {
    need(ind);
    ind->impl.clear_rows();
  });
}

int qmhd_indicator_train(qmhd_indicator* ind, int epochs, int tiles_per_step, float lr,
                         float pos_weight, int holdout, unsigned long long seed, double* loss) {
  return guarded([&] {
    need(ind);
    if (epochs < 0 || tiles_per_step < 1 || !(lr > 0.f))
      throw std::invalid_argument("qmhd_indicator_train: need epochs >= 0, tiles >= 1, lr > 0");
    const double l = ind->impl.train(epochs, tiles_per_step, lr, pos_weight, holdout, seed);
    if (loss) *loss = l;
  });
}

int qmhd_indicator_evaluate(qmhd_indicator* ind, float threshold, int holdout, double* recall,
                            double* flagged, long long* positives, long long* total) {
  return guarded([&] {
    need(ind);
    double r = 0, f = 0;
    long long p = 0, t = 0;
    ind->impl.evaluate(threshold, holdout, &r, &f, &p, &t);
    if (recall) *recall = r;
    if (flagged) *flagged = f;
    if (positives) *positives = p;
    if (total) *total = t;
  });
}

int qmhd_indicator_threshold_for_recall(qmhd_indicator* ind, double recall, int holdout,
                                        float* threshold) {
  return guarded([&] {
    need(ind);
    need(threshold);
    *threshold = ind->impl.threshold_for_recall(recall, holdout);
  });
}

int qmhd_solver_set_indicator(qmhd_solver* solver, const qmhd_indicator* ind, float threshold) {
  return guarded([&] {
    need(solver);
    solver->impl->set_indicator(ind ? &ind->impl : nullptr, threshold);
  });
}

int qmhd_solver_learned_face_counts(qmhd_solver* solver, long long* x_faces, long long* y_faces) {
  return guarded([&] {
    need(solver);
    long long a = 0, b = 0;
    solver->impl->learned_face_counts(&a, &b);
    if (x_faces) *x_faces = a;
    if (y_faces) *y_faces = b;
  });
}

// Allocation-free totals over caller-owned device arrays: validation, then
// the scratch lookup and the two reductions under the device's lock.  Returns codes
// directly (no exceptions) so the success path allocates nothing on the host.
static_assert(QMHD_TOTALS_DEVICE_MAX_CELLS == qb::kTotalsMaxCells, "scratch limit");

int qmhd_conserved_cell_totals_device(const double* rho, const double* energy, int nx, int ny,
                                      int nghost, void* stream, double* mass,
                                      double* energy_total) {
  char msg[256];
  auto fail = [&](int code) {
    g_error = msg;
    return code;
  };
  if (!rho || !energy || !mass || !energy_total) {
    std::snprintf(msg, sizeof msg, "qmhd_conserved_cell_totals_device: null pointer argument");
    return fail(QMHD_INVALID_ARGUMENT);
  }
  if (nx < 1 || ny < 1 || nghost < 0) {
    std::snprintf(msg, sizeof msg,
                  "qmhd_conserved_cell_totals_device: need nx >= 1, ny >= 1, nghost >= 0 "
                  "(got %d, %d, %d)", nx, ny, nghost);
    return fail(QMHD_INVALID_ARGUMENT);
  }
  const long long cells = (long long)nx * ny;
  if (cells > qb::kTotalsMaxCells) {
    std::snprintf(msg, sizeof msg,
                  "qmhd_conserved_cell_totals_device: %lld cells exceed the fixed scratch "
                  "limit of %lld cells (QMHD_TOTALS_DEVICE_MAX_CELLS)",
                  cells, (long long)qb::kTotalsMaxCells);
    return fail(QMHD_INVALID_ARGUMENT);
  }
  int device = -1;
  cudaError_t rc = cudaGetDevice(&device);
  if (rc != cudaSuccess) {
    std::snprintf(msg, sizeof msg, "qmhd_conserved_cell_totals_device: cudaGetDevice: %s",
                  cudaGetErrorString(rc));
    return fail(QMHD_DEVICE_ERROR);
  }
  for (const double* p : {rho, energy}) {
    cudaPointerAttributes a{};
    rc = cudaPointerGetAttributes(&a, p);
    if (rc != cudaSuccess ||
        !(a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) ||
        a.device != device) {
      cudaGetLastError();
      std::snprintf(msg, sizeof msg,
                    "qmhd_conserved_cell_totals_device: %s is not device memory of the "
                    "current device %d", p == rho ? "rho" : "energy", device);
      return fail(QMHD_INVALID_ARGUMENT);
    }
  }
  double totals[2];
  rc = qb::totals_noalloc(device, rho, energy, nx, ny, nghost, (cudaStream_t)stream, totals);
  if (rc != cudaSuccess) {
    std::snprintf(msg, sizeof msg, "qmhd_conserved_cell_totals_device: device %d: %s", device,
                  cudaGetErrorString(rc));
    return fail(QMHD_DEVICE_ERROR);
  }
  *mass = totals[0];
  *energy_total = totals[1];
  g_error.clear();
  return QMHD_OK;
}

}  // extern "C"
