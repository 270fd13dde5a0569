// Learned troubled-cell indicator: tcgen05 BF16 MLP kernels (see indicator.cuh).
#include "indicator.cuh"
#include "tc.cuh"

#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>

namespace qb {
namespace {

constexpr int kRowsPerTile = 128;  // MMA M
constexpr int kThreads = 128;      // 4 warps: warp w owns TMEM lanes 32w..32w+31

__device__ __forceinline__ float gelu(float x) {
  return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f));
}

__device__ __forceinline__ uint16_t to_bf16(float x) {
  return __bfloat16_as_ushort(__float2bfloat16_rn(x));
}

// Copy a row-major bf16 matrix [R][K] (K a multiple of 8, 16-byte aligned
// rows) into the K-major core layout, 16 bytes at a time.
__device__ __forceinline__ void stage_rows(uint8_t* dst, const uint16_t* src, int R, int K,
                                           long long row0, long long rows_valid, int tid,
                                           int nthreads) {
  const int chunks = K >> 3;
  for (int e = tid; e < R * chunks; e += nthreads) {
    const int r = e / chunks, kc = e - r * chunks;
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (row0 + r < rows_valid)
      v = *reinterpret_cast<const uint4*>(src + (row0 + r) * (long long)K + kc * 8);
    *reinterpret_cast<uint4*>(dst + tc::kmajor_offset(r, kc * 8, K)) = v;
  }
}

struct FwdSmem {
  static constexpr int kX = kRowsPerTile * kFeatPad * 2;  // 53248
  static constexpr int kW1 = kHidden * kFeatPad * 2;      // 26624
  static constexpr int kW2 = kHidden * kHidden * 2;       // 8192
  static constexpr int kA1 = kRowsPerTile * kHidden * 2;  // 16384
  static constexpr int kTotal = kX + kW1 + kW2 + kA1 + 64;
};

// Logits of `rows` feature rows: per 128-row tile, Z1 = X W1^T and
// Z2 = GELU(Z1 + b1) W2^T on the tensor cores (TMEM columns 0-63 and
// 64-127), then GELU(Z2 + b2) . w3 + b3 on the CUDA cores.
__global__ void __launch_bounds__(kThreads) k_mlp_forward(const uint16_t* __restrict__ x,
                                                          long long rows, MlpDev p,
                                                          float* __restrict__ logit,
                                                          int* status) {
  extern __shared__ __align__(1024) uint8_t sm[];
  uint8_t* xs = sm;
  uint8_t* w1s = xs + FwdSmem::kX;
  uint8_t* w2s = w1s + FwdSmem::kW1;
  uint8_t* a1s = w2s + FwdSmem::kW2;
  uint64_t* bar = reinterpret_cast<uint64_t*>(a1s + FwdSmem::kA1);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    tc::mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tc::tmem_alloc(tslot, 128);
  stage_rows(w1s, p.w1, kHidden, kFeatPad, 0, kHidden, tid, kThreads);
  stage_rows(w2s, p.w2, kHidden, kHidden, 0, kHidden, tid, kThreads);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = *tslot;
  const uint32_t idesc = tc::idesc_bf16(kRowsPerTile, kHidden);
  uint32_t phase = 0;
  bool ok = true;
  const long long tiles = (rows + kRowsPerTile - 1) / kRowsPerTile;
  const int row = warp * 32 + lane;
  for (long long t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
    const long long row0 = t * kRowsPerTile;
    stage_rows(xs, x, kRowsPerTile, kFeatPad, row0, rows, tid, kThreads);
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (tid == 0) {
      const uint32_t xa = tc::smem_u32(xs), wa = tc::smem_u32(w1s);
      for (int s = 0; s < kFeatPad / 16; ++s)
        tc::mma_bf16(tbase, tc::smem_desc(xa + 256 * s, 128, (kFeatPad / 8) * 128),
                     tc::smem_desc(wa + 256 * s, 128, (kFeatPad / 8) * 128), idesc, s > 0);
      tc::commit(bar);
    }
    ok = __syncthreads_and(tc::mbar_wait(bar, phase) ? 1 : 0) != 0;
    phase ^= 1;
    if (!ok) break;
    tc::fence_after_sync();
    for (int c0 = 0; c0 < kHidden; c0 += 16) {
      float z[16];
      tc::tmem_ld16(tc::tmem_addr(tbase, warp * 32, c0), z);
#pragma unroll
      for (int c = 0; c < 16; ++c) {
        const float h = gelu(z[c] + p.b1[c0 + c]);
        *reinterpret_cast<uint16_t*>(a1s + tc::kmajor_offset(row, c0 + c, kHidden)) = to_bf16(h);
      }
    }
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (tid == 0) {
      const uint32_t aa = tc::smem_u32(a1s), wa = tc::smem_u32(w2s);
      for (int s = 0; s < kHidden / 16; ++s)
        tc::mma_bf16(tbase + 64, tc::smem_desc(aa + 256 * s, 128, (kHidden / 8) * 128),
                     tc::smem_desc(wa + 256 * s, 128, (kHidden / 8) * 128), idesc, s > 0);
      tc::commit(bar);
    }
    ok = __syncthreads_and(tc::mbar_wait(bar, phase) ? 1 : 0) != 0;
    phase ^= 1;
    if (!ok) break;
    tc::fence_after_sync();
    float acc = p.b3[0];
    for (int c0 = 0; c0 < kHidden; c0 += 16) {
      float z[16];
      tc::tmem_ld16(tc::tmem_addr(tbase, warp * 32, 64 + c0), z);
#pragma unroll
      for (int c = 0; c < 16; ++c) acc += p.w3[c0 + c] * gelu(z[c] + p.b2[c0 + c]);
    }
    if (row0 + row < rows) logit[row0 + row] = acc;
    tc::fence_before_sync();
    __syncthreads();
  }
  if (!ok) {
    // a wait ran out: report, then give the outstanding MMAs a bounded
    // chance to finish before the TMEM they write is released
    if (tid == 0) atomicOr(status, 1);
    tc::mbar_wait(bar, phase ^ 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_free(tbase, 128);
}

}  // namespace

cudaError_t launch_mlp_forward(const uint16_t* x, long long rows, const MlpDev& p, float* logit,
                               int* status, cudaStream_t s) {
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         FwdSmem::kTotal);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long tiles = (rows + kRowsPerTile - 1) / kRowsPerTile;
  const int grid = int(tiles < sms ? tiles : sms);
  if (grid <= 0) return cudaSuccess;
  k_mlp_forward<<<grid, kThreads, FwdSmem::kTotal, s>>>(x, rows, p, logit, status);
  return cudaGetLastError();
}

uint16_t bf16_bits(float x) {
  uint32_t u;
  std::memcpy(&u, &x, 4);
  if ((u & 0x7F800000u) == 0x7F800000u) return uint16_t(u >> 16);  // inf / nan kept
  u += 0x7FFFu + ((u >> 16) & 1u);
  return uint16_t(u >> 16);
}

namespace {
void ick(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}
// splitmix64, for the initial weights
uint64_t mix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
}  // namespace

Indicator::Indicator(unsigned long long seed) {
  ick(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "indicator stream");
  ick(cudaMalloc(&params_, sizeof(float) * kParamCount), "indicator params");
  ick(cudaMalloc(&w1b_, sizeof(uint16_t) * kHidden * kFeatPad), "indicator w1");
  ick(cudaMalloc(&w2b_, sizeof(uint16_t) * kHidden * kHidden), "indicator w2");
  ick(cudaMalloc(&status_, sizeof(int)), "indicator status");
  ick(cudaMemset(status_, 0, sizeof(int)), "indicator status");
  // Glorot-uniform weights, zero biases
  std::vector<float> h(kParamCount, 0.0f);
  uint64_t st = seed;
  auto uni = [&](float a) { return float((double(mix(st) >> 11) * 0x1.0p-53 * 2.0 - 1.0) * a); };
  const float a1 = std::sqrt(6.0f / float(kFeat + kHidden));
  const float a2 = std::sqrt(6.0f / float(kHidden + kHidden));
  const float a3 = std::sqrt(6.0f / float(kHidden + 1));
  float* w1 = h.data();
  float* w2 = w1 + kHidden * kFeat + kHidden;
  float* w3 = w2 + kHidden * kHidden + kHidden;
  for (int i = 0; i < kHidden * kFeat; ++i) w1[i] = uni(a1);
  for (int i = 0; i < kHidden * kHidden; ++i) w2[i] = uni(a2);
  for (int i = 0; i < kHidden; ++i) w3[i] = uni(a3);
  set_params(h.data());
}

Indicator::~Indicator() {
  if (stream_) cudaStreamSynchronize(stream_);
  cudaFree(params_);
  cudaFree(w1b_);
  cudaFree(w2b_);
  cudaFree(status_);
  if (stream_) cudaStreamDestroy(stream_);
}

void Indicator::upload_bf16_from_host(const std::vector<float>& h) {
  std::vector<uint16_t> w1(size_t(kHidden) * kFeatPad, 0), w2(size_t(kHidden) * kHidden);
  for (int o = 0; o < kHidden; ++o)
    for (int i = 0; i < kFeat; ++i) w1[size_t(o) * kFeatPad + i] = bf16_bits(h[size_t(o) * kFeat + i]);
  const float* hw2 = h.data() + kHidden * kFeat + kHidden;
  for (int i = 0; i < kHidden * kHidden; ++i) w2[size_t(i)] = bf16_bits(hw2[i]);
  ick(cudaMemcpyAsync(w1b_, w1.data(), sizeof(uint16_t) * w1.size(), cudaMemcpyHostToDevice, stream_),
      "indicator w1");
  ick(cudaMemcpyAsync(w2b_, w2.data(), sizeof(uint16_t) * w2.size(), cudaMemcpyHostToDevice, stream_),
      "indicator w2");
  ick(cudaStreamSynchronize(stream_), "indicator upload");
}

void Indicator::set_params(const float* host) {
  std::vector<float> h(host, host + kParamCount);
  for (float v : h)
    if (!std::isfinite(v)) throw std::invalid_argument("indicator: parameters must be finite");
  ick(cudaMemcpyAsync(params_, h.data(), sizeof(float) * kParamCount, cudaMemcpyHostToDevice, stream_),
      "indicator params");
  upload_bf16_from_host(h);
}

void Indicator::get_params(float* host) {
  ick(cudaMemcpyAsync(host, params_, sizeof(float) * kParamCount, cudaMemcpyDeviceToHost, stream_),
      "indicator params");
  ick(cudaStreamSynchronize(stream_), "indicator params");
}

MlpDev Indicator::dev() const {
  MlpDev d;
  d.w1 = w1b_;
  d.w2 = w2b_;
  d.b1 = params_ + kHidden * kFeat;
  d.b2 = d.b1 + kHidden + kHidden * kHidden;
  d.w3 = d.b2 + kHidden;
  d.b3 = d.w3 + kHidden;
  return d;
}

void Indicator::check_status(const char* what) {
  int st = 0;
  ick(cudaMemcpyAsync(&st, status_, sizeof(int), cudaMemcpyDeviceToHost, stream_), what);
  ick(cudaStreamSynchronize(stream_), what);
  if (st) {
    cudaMemsetAsync(status_, 0, sizeof(int), stream_);
    throw std::runtime_error(std::string(what) + ": a tensor-core wait ran out");
  }
}

void Indicator::forward(const float* features, long long rows, float* logits) {
  if (rows <= 0) return;
  std::vector<uint16_t> x(size_t(rows) * kFeatPad, 0);
  for (long long r = 0; r < rows; ++r)
    for (int i = 0; i < kFeat; ++i) x[size_t(r) * kFeatPad + i] = bf16_bits(features[r * kFeat + i]);
  uint16_t* dx = nullptr;
  float* dl = nullptr;
  ick(cudaMalloc(&dx, sizeof(uint16_t) * x.size()), "forward rows");
  ick(cudaMalloc(&dl, sizeof(float) * size_t(rows)), "forward logits");
  try {
    ick(cudaMemcpyAsync(dx, x.data(), sizeof(uint16_t) * x.size(), cudaMemcpyHostToDevice, stream_),
        "forward rows");
    ick(launch_mlp_forward(dx, rows, dev(), dl, status_, stream_), "forward launch");
    ick(cudaMemcpyAsync(logits, dl, sizeof(float) * size_t(rows), cudaMemcpyDeviceToHost, stream_),
        "forward logits");
    check_status("indicator forward");
  } catch (...) {
    cudaFree(dx);
    cudaFree(dl);
    throw;
  }
  cudaFree(dx);
  cudaFree(dl);
}

}  // namespace qb
