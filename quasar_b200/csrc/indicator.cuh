// Learned troubled-cell indicator: a 200 -> 64 -> 64 -> 1 GELU MLP over the
// 5 x 5 stencil of 8 normalised primitives, BF16 weights and FP32
// accumulation on the tcgen05 tensor cores.  A cell scored above the
// threshold keeps the characteristic MP reconstruction at its faces; other
// faces take the component-wise unlimited interpolation, which equals the
// characteristic one wherever the MP limiter would not fire (R L = I).
#pragma once

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

  MlpDev dev() const;
  float* master() { return params_; }
  uint16_t* w1_bf16() { return w1b_; }
  uint16_t* w2_bf16() { return w2b_; }
  cudaStream_t stream() const { return stream_; }
  void check_status(const char* what);

 private:
  void upload_bf16_from_host(const std::vector<float>& h);
  float* params_ = nullptr;   // kParamCount
  uint16_t* w1b_ = nullptr;   // [64][208]
  uint16_t* w2b_ = nullptr;   // [64][64]
  int* status_ = nullptr;
  cudaStream_t stream_ = nullptr;
};

}  // namespace qb
