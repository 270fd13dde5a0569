// Learned troubled-cell indicator: a 200 -> 64 -> 64 -> 1 GELU MLP over the
// 5 x 5 stencil of 8 normalised primitives, BF16 weights and FP32
// accumulation on the tcgen05 tensor cores.  A cell scored above the
// threshold keeps the characteristic MP reconstruction at its faces; other
// faces take the component-wise unlimited interpolation, which equals the
// characteristic one wherever the MP limiter would not fire (R L = I).
#pragma once

#include "mhd_kernels.cuh"

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace qb {

constexpr int kFeat = 200;     // 25 stencil cells x 8 primitives
constexpr int kFeatPad = 208;  // padded to the MMA K step (16)
constexpr int kHidden = 64;

// Parameter block of the MLP in FP32 (master copy); the kernels read BF16
// copies of w1 and w2.
struct MlpParams {
  float w1[kHidden * kFeat];   // [out][in]
  float b1[kHidden];
  float w2[kHidden * kHidden];  // [out][in]
  float b2[kHidden];
  float w3[kHidden];
  float b3;
};
constexpr int kParamCount = kHidden * kFeat + kHidden + kHidden * kHidden + kHidden + kHidden + 1;

// Device-side BF16/FP32 parameter views used by the kernels.
struct MlpDev {
  const uint16_t* w1;  // bf16 [64][208], zero padded
  const uint16_t* w2;  // bf16 [64][64]
  const float* b1;
  const float* b2;
  const float* w3;
  const float* b3;
};

// Forward pass of `rows` BF16 feature rows (row stride kFeatPad) -> logits.
// A tensor-core wait that runs out sets bit 0 of *status.
cudaError_t launch_mlp_forward(const uint16_t* x, long long rows, const MlpDev& p, float* logit,
                               int* status, cudaStream_t s);

uint16_t bf16_bits(float x);  // round to nearest even

// Feature rows (BF16, row stride kFeatPad, zero padded) of the interior cells
// of a padded state, row r = cell (r % nx, r / nx); cells whose centre is not
// admissible get an all-zero row and `bad[r] = 1` (they are always flagged).
void launch_cell_features(const Grid& g, const StateP& u, double gamma, uint16_t* rows,
                          unsigned char* bad, cudaStream_t s);
// Per-row labels: 1 where the per-padded-cell limiter departure exceeds tol.
void launch_gather_labels(const Grid& g, const int* label, float tol, unsigned char* y,
                          cudaStream_t s);

// One gradient pass of the MLP over `ntiles` 128-row tiles of (x, y) listed
// in `tiles`: per-CTA partial gradients (parameter packing, then the loss)
// in partial[cta * (kParamCount + 1)].  pos_weight scales the positive rows'
// loss; inv_n = 1 / rows in the pass.  Returns the CTA count used.
int launch_mlp_grad(const uint16_t* x, const unsigned char* y, long long rows, const int* tiles,
                    int ntiles, const MlpDev& p, const uint16_t* w2t, float pos_weight,
                    float inv_n, float* partial, int* status, cudaStream_t s);
// Sum the partials (fixed order) into grad[kParamCount + 1].
void launch_reduce_partials(const float* partial, int ctas, float* grad, cudaStream_t s);
// Adam step on the FP32 master parameters, then refresh the BF16 copies
// (w1 padded, w2 and its transpose).
void launch_adam(float* params, float* m, float* v, const float* grad, int step, float lr,
                 float beta1, float beta2, float eps, uint16_t* w1b, uint16_t* w2b,
                 uint16_t* w2tb, cudaStream_t s);

// Fused inference over the padded cells of a state: the 5 x 5 primitive
// stencil is staged in shared memory, normalised into BF16 feature rows in
// the tensor-core layout, run through the MLP, and flag[cell] = (logit >
// threshold) or the cell has no full stencil or an inadmissible centre.
// Kernel attributes of launch_indicator; call once before it is launched or
// captured into a graph.
cudaError_t configure_indicator_kernels();
// The same over the stage-0 (live) records of a batch, one learned buffer
// set per instance; plan = the kBpInd tile plan.
cudaError_t launch_batch_indicator(const BatchRec* r, const BatchLearnRec* l, const BatchPlan& plan,
                                   const MlpDev& p, float threshold, int* status, cudaStream_t s);
cudaError_t launch_indicator(const Grid& g, const StateP& u, double gamma, const MlpDev& p,
                             float threshold, unsigned char* flag, int* status, cudaStream_t s);

// Parameters of one indicator network on the device: the FP32 master copy
// (layout of MlpParams) and the BF16 weight copies the kernels read.
class Indicator {
 public:
  explicit Indicator(unsigned long long seed);
  ~Indicator();
  Indicator(const Indicator&) = delete;
  Indicator& operator=(const Indicator&) = delete;

  void set_params(const float* host);  // kParamCount floats
  void get_params(float* host);
  // Logits of host feature rows (rows x kFeat floats, rounded to BF16).
  void forward(const float* features, long long rows, float* logits);

  // Mean weighted BCE and its gradient over host rows (one pass, no update).
  double gradient(const float* features, const unsigned char* labels, long long rows,
                  float pos_weight, float* grad);

  // Training set on the device: feature rows and limiter labels collected
  // from solver states (MhdSolver2D::live_args).
  void collect(const StageArgs& live, cudaStream_t solver_stream, float tol);
  long long rows() const { return rows_; }
  // Copy the collected labels (one byte per row, collection order) to host.
  void labels_to_host(unsigned char* out, long long n) const;
  void clear_rows() { rows_ = 0; }
  // Adam over random 128-row tiles of the training rows; one tile in
  // `holdout` (chosen by a hash of its index) is held out (0 = none).
  // Returns the mean loss of the last epoch.
  double train(int epochs, int tiles_per_step, float lr, float pos_weight, int holdout,
               unsigned long long seed);
  // Recall of the positive rows and fraction flagged at `threshold` over the
  // held-out tiles (all tiles when holdout = 0).
  void evaluate(float threshold, int holdout, double* recall, double* flagged,
                long long* positives, long long* total);
  // Smallest logit threshold whose held-out recall is at least `recall`.
  float threshold_for_recall(double recall, int holdout);

  MlpDev dev() const;
  float* master() { return params_; }
  cudaStream_t stream() const { return stream_; }
  void check_status(const char* what);

 private:
  void upload_bf16_from_host(const std::vector<float>& h);
  void ensure_capacity(long long rows);
  void logits_of_tiles(int holdout, std::vector<float>* logit, std::vector<unsigned char>* y);
  float* params_ = nullptr;   // kParamCount
  uint16_t* w1b_ = nullptr;   // [64][208]
  uint16_t* w2b_ = nullptr;   // [64][64]
  uint16_t* w2tb_ = nullptr;  // [64][64] transposed
  float* adam_m_ = nullptr;
  float* adam_v_ = nullptr;
  float* grad_ = nullptr;     // kParamCount + 1
  float* partial_ = nullptr;  // per CTA
  int* tiles_ = nullptr;      // tile list of one step
  int tiles_cap_ = 0;
  int adam_step_ = 0;
  int* status_ = nullptr;
  cudaStream_t stream_ = nullptr;
  // training set
  uint16_t* xs_ = nullptr;
  unsigned char* ys_ = nullptr;
  long long rows_ = 0, cap_ = 0;
  int* label_ = nullptr;      // per padded cell of the last collected state
  long long label_cap_ = 0;
};

}  // namespace qb
