// Learned troubled-cell indicator: tcgen05 BF16 MLP kernels (see indicator.cuh).
#include "indicator.cuh"
#include "tc.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <stdexcept>
#include <string>

namespace qb {
namespace {

constexpr int kRowsPerTile = 128;  // MMA M
constexpr int kThreads = 128;      // 4 warps: warp w owns TMEM lanes 32w..32w+31

// GELU in its tanh form (Hendrycks and Gimpel, "Gaussian Error Linear
// Units", the approximation 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3)))),
// with the hardware tanh approximation (MUFU, a few ulp of FP32): a handful
// of instructions per activation where the erf form takes dozens.
constexpr float kGeluK0 = 0.7978845608028654f;  // sqrt(2 / pi)
constexpr float kGeluK1 = 0.044715f;
__device__ __forceinline__ float tanh_fast(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float gelu(float x) {
  const float t = tanh_fast(kGeluK0 * fmaf(kGeluK1 * x, x * x, x));
  return 0.5f * x * (1.0f + t);
}

// Two floats rounded to BF16 (nearest even) in one conversion, the first in
// the low half: the packing of consecutive K-major operand columns.
__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
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

// ---- features ----------------------------------------------------------------
// Primitives (rho, vx, vy, vz, p, bx, by, bz) of padded cell k with the
// collocated field; ok = finite, rho > 0 and p > 0.
__device__ __forceinline__ bool cell_prim(const StateP& u, long long k, double gamma, float* w) {
  const double rho = u.c[0][k], mx = u.c[1][k], my = u.c[2][k], mz = u.c[3][k];
  const double e = u.c[4][k], bx = u.bxc[k], by = u.byc[k], bz = u.c[7][k];
  const double ir = 1.0 / rho;
  const double vx = mx * ir, vy = my * ir, vz = mz * ir;
  const double p = (gamma - 1.0) * ((e - 0.5 * (mx * vx + my * vy + mz * vz)) -
                                    0.5 * (bx * bx + by * by + bz * bz));
  w[0] = float(rho); w[1] = float(vx); w[2] = float(vy); w[3] = float(vz);
  w[4] = float(p);   w[5] = float(bx); w[6] = float(by); w[7] = float(bz);
  return isfinite(rho) && rho > 0.0 && isfinite(p) && p > 0.0 && isfinite(vx) && isfinite(vy) &&
         isfinite(vz) && isfinite(bx) && isfinite(by) && isfinite(bz);
}

// Normalisation constants of a centre cell: 1/rho_c, 1/a_c, 1/p_c, 1/(sqrt(rho_c) a_c).
struct Norm {
  float irho, ia, ip, isb;
};
__device__ __forceinline__ Norm make_norm(const float* c, double gamma) {
  const float a = sqrtf(float(gamma) * c[4] / c[0]);
  Norm n;
  n.irho = 1.0f / c[0];
  n.ia = 1.0f / a;
  n.ip = 1.0f / c[4];
  n.isb = 1.0f / (sqrtf(c[0]) * a);
  return n;
}
__device__ __forceinline__ float clampf(float x) {
  return isfinite(x) ? fminf(fmaxf(x, -64.0f), 64.0f) : 64.0f;
}
// The same from the two 16-byte halves of the stencil cell (rho, vx, vy, vz)
// and (p, bx, by, bz) and of the centre c.
__device__ __forceinline__ uint4 features8h(const float4 qa, const float4 qb, const float4 ca,
                                            const float4 cb, const Norm& n) {
  float f[8];
  f[0] = clampf(qa.x * n.irho - 1.0f);
  f[1] = clampf((qa.y - ca.y) * n.ia);
  f[2] = clampf((qa.z - ca.z) * n.ia);
  f[3] = clampf((qa.w - ca.w) * n.ia);
  f[4] = clampf(qb.x * n.ip - 1.0f);
  f[5] = clampf((qb.y - cb.y) * n.isb);
  f[6] = clampf((qb.z - cb.z) * n.isb);
  f[7] = clampf((qb.w - cb.w) * n.isb);
  uint4 r;
  r.x = pack_bf16x2(f[0], f[1]);
  r.y = pack_bf16x2(f[2], f[3]);
  r.z = pack_bf16x2(f[4], f[5]);
  r.w = pack_bf16x2(f[6], f[7]);
  return r;
}
// 8 normalised features of stencil cell q (primitives) as packed BF16.
__device__ __forceinline__ uint4 features8(const float* q, const float* c, const Norm& n) {
  float f[8];
  f[0] = clampf(q[0] * n.irho - 1.0f);
  f[1] = clampf((q[1] - c[1]) * n.ia);
  f[2] = clampf((q[2] - c[2]) * n.ia);
  f[3] = clampf((q[3] - c[3]) * n.ia);
  f[4] = clampf(q[4] * n.ip - 1.0f);
  f[5] = clampf((q[5] - c[5]) * n.isb);
  f[6] = clampf((q[6] - c[6]) * n.isb);
  f[7] = clampf((q[7] - c[7]) * n.isb);
  uint4 r;
  r.x = pack_bf16x2(f[0], f[1]);
  r.y = pack_bf16x2(f[2], f[3]);
  r.z = pack_bf16x2(f[4], f[5]);
  r.w = pack_bf16x2(f[6], f[7]);
  return r;
}

__global__ void k_cell_features(Grid g, StateP u, double gamma, uint16_t* __restrict__ rows,
                                unsigned char* __restrict__ bad) {
  const long long n = (long long)g.nx * g.ny;
  const long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int i = int(r % g.nx), j = int(r / g.nx);
  uint4* dst = reinterpret_cast<uint4*>(rows + r * kFeatPad);
  float c[8];
  const bool ok = cell_prim(u, g.idx(i, j), gamma, c);
  const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
  bad[r] = ok ? 0 : 1;
  if (!ok) {
    for (int q = 0; q < kFeatPad / 8; ++q) dst[q] = zero;
    return;
  }
  const Norm nm = make_norm(c, gamma);
  for (int dj = -2; dj <= 2; ++dj)
    for (int di = -2; di <= 2; ++di) {
      float q[8];
      cell_prim(u, g.idx(i + di, j + dj), gamma, q);
      dst[5 * (dj + 2) + (di + 2)] = features8(q, c, nm);
    }
  dst[25] = zero;
}

__global__ void k_gather_labels(Grid g, const int* __restrict__ label, float tol,
                                unsigned char* y) {
  const long long n = (long long)g.nx * g.ny;
  const long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int i = int(r % g.nx), j = int(r / g.nx);
  y[r] = __int_as_float(label[g.idx(i, j)]) > tol ? 1 : 0;
}

// ---- training: forward + backward of 128-row tiles on the tensor cores -------
// d/dx of the tanh-form GELU above
__device__ __forceinline__ float gelu_grad(float x) {
  const float x2 = x * x;
  const float t = tanh_fast(kGeluK0 * fmaf(kGeluK1 * x, x2, x));
  return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * kGeluK0 * fmaf(3.0f * kGeluK1, x2, 1.0f);
}

struct GradSmem {
  static constexpr int kBufA = 208 * 128 * 2;   // X, then X^T
  static constexpr int kW1 = 64 * 208 * 2;
  static constexpr int kW2 = 64 * 64 * 2;
  static constexpr int kW2T = 64 * 64 * 2;
  static constexpr int kA1 = 128 * 64 * 2;
  static constexpr int kA1T = 64 * 128 * 2;
  static constexpr int kDZ2 = 128 * 64 * 2;
  static constexpr int kBufB = 128 * 128 * 2;   // dZ2^T, then dZ1^T (rows 64-127 zero)
  static constexpr int kSmall = 1024;
  static constexpr int kTotal = kBufA + kW1 + kW2 + kW2T + kA1 + kA1T + kDZ2 + kBufB + kSmall;
};
constexpr int kColZ1 = 0, kColZ2 = 64, kColDA1 = 128, kColDW2 = 192, kColDW1 = 256;
constexpr int kOffW1 = 0, kOffB1 = kHidden * kFeat, kOffW2 = kOffB1 + kHidden,
              kOffB2 = kOffW2 + kHidden * kHidden, kOffW3 = kOffB2 + kHidden,
              kOffB3 = kOffW3 + kHidden;

__global__ void __launch_bounds__(kThreads) k_mlp_grad(
    const uint16_t* __restrict__ x, const unsigned char* __restrict__ y, long long rows,
    const int* __restrict__ tiles, int ntiles, MlpDev p, const uint16_t* __restrict__ w2t,
    float pos_weight, float inv_n, float* __restrict__ partial, int* status) {
  extern __shared__ __align__(1024) uint8_t sm[];
  uint8_t* bufA = sm;
  uint8_t* w1s = bufA + GradSmem::kBufA;
  uint8_t* w2s = w1s + GradSmem::kW1;
  uint8_t* w2ts = w2s + GradSmem::kW2;
  uint8_t* a1s = w2ts + GradSmem::kW2T;
  uint8_t* a1ts = a1s + GradSmem::kA1;
  uint8_t* dz2s = a1ts + GradSmem::kA1T;
  uint8_t* bufB = dz2s + GradSmem::kDZ2;
  float* gb1 = reinterpret_cast<float*>(bufB + GradSmem::kBufB);
  float* gb2 = gb1 + 64;
  float* gw3 = gb2 + 64;
  float* gsc = gw3 + 64;  // [0] b3, [1] loss
  uint64_t* bar = reinterpret_cast<uint64_t*>(gsc + 4);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, row = warp * 32 + lane;
  if (tid == 0) {
    tc::mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tc::tmem_alloc(tslot, 512);
  for (int e = tid; e < GradSmem::kBufB / 16; e += kThreads)
    reinterpret_cast<uint4*>(bufB)[e] = make_uint4(0u, 0u, 0u, 0u);
  if (tid < 64) {
    gb1[tid] = 0.f;
    gb2[tid] = 0.f;
    gw3[tid] = 0.f;
  }
  if (tid < 4) gsc[tid] = 0.f;
  stage_rows(w1s, p.w1, kHidden, kFeatPad, 0, kHidden, tid, kThreads);
  stage_rows(w2s, p.w2, kHidden, kHidden, 0, kHidden, tid, kThreads);
  stage_rows(w2ts, w2t, kHidden, kHidden, 0, kHidden, tid, kThreads);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tb = *tslot;
  const uint32_t id64 = tc::idesc_bf16(128, 64), id208 = tc::idesc_bf16(128, 208);
  uint32_t phase = 0;
  bool ok = true;
  int done = 0;
  auto sync_async = [&]() {
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
  };
  auto wait_all = [&]() {
    ok = __syncthreads_and(tc::mbar_wait(bar, phase) ? 1 : 0) != 0;
    phase ^= 1;
    tc::fence_after_sync();
    return ok;
  };
  for (int ti = blockIdx.x; ti < ntiles && ok; ti += gridDim.x, ++done) {
    const long long row0 = (long long)tiles[ti] * 128;
    const long long grow = row0 + row;
    const bool valid = grow < rows;
    // 1. X tile (K-major) -> Z1 = X W1^T
    stage_rows(bufA, x, 128, kFeatPad, row0, rows, tid, kThreads);
    sync_async();
    if (tid == 0) {
      const uint32_t xa = tc::smem_u32(bufA), wa = tc::smem_u32(w1s);
      for (int s = 0; s < kFeatPad / 16; ++s)
        tc::mma_bf16(tb + kColZ1, tc::smem_desc(xa + 256 * s, 128, 26 * 128),
                     tc::smem_desc(wa + 256 * s, 128, 26 * 128), id64, s > 0);
      tc::commit(bar);
    }
    if (!wait_all()) break;
    // 2. A1 = GELU(Z1 + b1) as layer-2 operand and its transpose; X^T
    for (int c0 = 0; c0 < 64; c0 += 16) {
      float z[16];
      tc::tmem_ld16(tc::tmem_addr(tb, warp * 32, kColZ1 + c0), z);
#pragma unroll
      for (int c = 0; c < 16; ++c) {
        const uint16_t h = to_bf16(gelu(z[c] + p.b1[c0 + c]));
        *reinterpret_cast<uint16_t*>(a1s + tc::kmajor_offset(row, c0 + c, 64)) = h;
        *reinterpret_cast<uint16_t*>(a1ts + tc::kmajor_offset(c0 + c, row, 128)) = h;
      }
    }
    for (int q = 0; q < kFeatPad / 8; ++q) {
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (valid) v = *reinterpret_cast<const uint4*>(x + grow * kFeatPad + q * 8);
      const uint16_t* h = reinterpret_cast<const uint16_t*>(&v);
#pragma unroll
      for (int e = 0; e < 8; ++e)
        *reinterpret_cast<uint16_t*>(bufA + tc::kmajor_offset(q * 8 + e, row, 128)) = h[e];
    }
    sync_async();
    if (tid == 0) {
      const uint32_t aa = tc::smem_u32(a1s), wa = tc::smem_u32(w2s);
      for (int s = 0; s < 4; ++s)
        tc::mma_bf16(tb + kColZ2, tc::smem_desc(aa + 256 * s, 128, 8 * 128),
                     tc::smem_desc(wa + 256 * s, 128, 8 * 128), id64, s > 0);
      tc::commit(bar);
    }
    if (!wait_all()) break;
    // 3. head, loss and dZ2
    {
      float u2[64];
      for (int c0 = 0; c0 < 64; c0 += 16) tc::tmem_ld16(tc::tmem_addr(tb, warp * 32, kColZ2 + c0), u2 + c0);
      float logit = p.b3[0];
#pragma unroll 8
      for (int c = 0; c < 64; ++c) {
        u2[c] += p.b2[c];
        logit += p.w3[c] * gelu(u2[c]);
      }
      const float yv = valid ? float(y[grow]) : 0.f;
      const float wgt = valid ? (yv > 0.5f ? pos_weight : 1.0f) : 0.0f;
      const float pr = 1.0f / (1.0f + expf(-logit));
      const float sp = logit > 0.f ? logit + log1pf(expf(-logit)) : log1pf(expf(logit));
      const float dz3 = wgt * (pr - yv) * inv_n;
      if (valid) {
        atomicAdd(&gsc[1], wgt * (sp - yv * logit) * inv_n);
        atomicAdd(&gsc[0], dz3);
      }
#pragma unroll 4
      for (int c = 0; c < 64; ++c) {
        const float a2 = gelu(u2[c]);
        const float dz2 = dz3 * p.w3[c] * gelu_grad(u2[c]);
        if (valid) {
          atomicAdd(&gw3[c], dz3 * a2);
          atomicAdd(&gb2[c], dz2);
        }
        const uint16_t h = to_bf16(dz2);
        *reinterpret_cast<uint16_t*>(dz2s + tc::kmajor_offset(row, c, 64)) = h;
        *reinterpret_cast<uint16_t*>(bufB + tc::kmajor_offset(c, row, 128)) = h;
      }
    }
    sync_async();
    if (tid == 0) {
      const uint32_t da = tc::smem_u32(dz2s), wt = tc::smem_u32(w2ts);
      for (int s = 0; s < 4; ++s)
        tc::mma_bf16(tb + kColDA1, tc::smem_desc(da + 256 * s, 128, 8 * 128),
                     tc::smem_desc(wt + 256 * s, 128, 8 * 128), id64, s > 0);
      const uint32_t bt = tc::smem_u32(bufB), at = tc::smem_u32(a1ts);
      for (int s = 0; s < 8; ++s)
        tc::mma_bf16(tb + kColDW2, tc::smem_desc(bt + 256 * s, 128, 16 * 128),
                     tc::smem_desc(at + 256 * s, 128, 16 * 128), id64, (done > 0 || s > 0) ? 1 : 0);
      tc::commit(bar);
    }
    if (!wait_all()) break;
    // 4. dZ1 = dA1 * GELU'(Z1 + b1), transposed into bufB
    for (int c0 = 0; c0 < 64; c0 += 16) {
      float da[16], z[16];
      tc::tmem_ld16(tc::tmem_addr(tb, warp * 32, kColDA1 + c0), da);
      tc::tmem_ld16(tc::tmem_addr(tb, warp * 32, kColZ1 + c0), z);
#pragma unroll
      for (int c = 0; c < 16; ++c) {
        const float dz1 = da[c] * gelu_grad(z[c] + p.b1[c0 + c]);
        if (valid) atomicAdd(&gb1[c0 + c], dz1);
        *reinterpret_cast<uint16_t*>(bufB + tc::kmajor_offset(c0 + c, row, 128)) = to_bf16(dz1);
      }
    }
    sync_async();
    if (tid == 0) {
      const uint32_t bt = tc::smem_u32(bufB), xt = tc::smem_u32(bufA);
      for (int s = 0; s < 8; ++s)
        tc::mma_bf16(tb + kColDW1, tc::smem_desc(bt + 256 * s, 128, 16 * 128),
                     tc::smem_desc(xt + 256 * s, 128, 16 * 128), id208, (done > 0 || s > 0) ? 1 : 0);
      tc::commit(bar);
    }
    if (!wait_all()) break;
  }
  float* out = partial + (size_t)blockIdx.x * (kParamCount + 1);
  if (ok && done > 0) {
    if (warp < 2) {
      for (int c0 = 0; c0 < 64; c0 += 16) {
        float v[16];
        tc::tmem_ld16(tc::tmem_addr(tb, warp * 32, kColDW2 + c0), v);
        for (int c = 0; c < 16; ++c) out[kOffW2 + row * 64 + c0 + c] = v[c];
      }
      for (int c0 = 0; c0 < 208; c0 += 16) {
        float v[16];
        tc::tmem_ld16(tc::tmem_addr(tb, warp * 32, kColDW1 + c0), v);
        for (int c = 0; c < 16; ++c)
          if (c0 + c < kFeat) out[kOffW1 + row * kFeat + c0 + c] = v[c];
      }
    }
  } else {
    for (int e = tid; e < kHidden * kFeat; e += kThreads) out[kOffW1 + e] = 0.f;
    for (int e = tid; e < kHidden * kHidden; e += kThreads) out[kOffW2 + e] = 0.f;
  }
  __syncthreads();
  if (tid < 64) {
    out[kOffB1 + tid] = gb1[tid];
    out[kOffB2 + tid] = gb2[tid];
    out[kOffW3 + tid] = gw3[tid];
  }
  if (tid == 0) {
    out[kOffB3] = gsc[0];
    out[kParamCount] = gsc[1];
  }
  if (!ok) {
    if (tid == 0) atomicOr(status, 1);
    tc::mbar_wait(bar, phase ^ 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_free(tb, 512);
}

__global__ void k_reduce_partials(const float* __restrict__ partial, int ctas, float* grad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > kParamCount) return;
  float s = 0.f;
  for (int c = 0; c < ctas; ++c) s += partial[(size_t)c * (kParamCount + 1) + i];
  grad[i] = s;
}

__global__ void k_adam(float* params, float* m, float* v, const float* grad, float lr, float b1,
                       float b2, float eps, float c1, float c2, uint16_t* w1b, uint16_t* w2b,
                       uint16_t* w2tb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kParamCount) return;
  const float g = grad[i];
  const float mi = b1 * m[i] + (1.f - b1) * g;
  const float vi = b2 * v[i] + (1.f - b2) * g * g;
  m[i] = mi;
  v[i] = vi;
  const float pv = params[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
  params[i] = pv;
  if (i < kOffB1) {
    w1b[(i / kFeat) * kFeatPad + i % kFeat] = to_bf16(pv);
  } else if (i >= kOffW2 && i < kOffB2) {
    const int o = (i - kOffW2) / kHidden, in = (i - kOffW2) % kHidden;
    w2b[o * kHidden + in] = to_bf16(pv);
    w2tb[in * kHidden + o] = to_bf16(pv);
  }
}

// ---- fused inference over a state ----------------------------------------------
constexpr int kTileX = 16, kTileY = 8;            // 128 cells per tile
constexpr int kHaloX = kTileX + 4, kHaloY = kTileY + 4;  // 5 x 5 stencil halo
struct InfSmem {
  static constexpr int kX = 128 * kFeatPad * 2;
  static constexpr int kW1 = kHidden * kFeatPad * 2;
  static constexpr int kW2 = kHidden * kHidden * 2;
  static constexpr int kA1 = 128 * kHidden * 2;
  static constexpr int kPrim = kHaloX * kHaloY * 8 * 4;
  static constexpr int kOk = 256;
  static constexpr int kVec = (3 * kHidden + 4) * 4;  // b1, b2, w3 (+ pad)
  static constexpr int kTotal = kX + kW1 + kW2 + kA1 + kPrim + kOk + kVec + 64;
};

// One 16 x 8 block of padded cells per tile: primitives of its 20 x 12 halo
// into shared memory, each thread's feature row straight into the
// tensor-core operand layout, then the two MMAs and the head.
// Tile sources: one state, or every instance of a batch (live state, stage-0
// records, learned buffers).
struct SingleSrc {
  Grid g;
  StateP u;
  double gamma;
  unsigned char* flag;
  __device__ long long tiles() const {
    return (long long)((g.pitch + kTileX - 1) / kTileX) * ((g.ny + 2 * g.ng + kTileY - 1) / kTileY);
  }
  __device__ void get(long long t, const Grid** gg, const StateP** uu, double* ga,
                      unsigned char** fl, int* i0, int* j0) const {
    const int ntx = (g.pitch + kTileX - 1) / kTileX;
    *gg = &g;
    *uu = &u;
    *ga = gamma;
    *fl = flag;
    *i0 = int(t % ntx) * kTileX - g.ng;
    *j0 = int(t / ntx) * kTileY - g.ng;
  }
};
struct BatchSrc {
  const BatchRec* r;
  const BatchLearnRec* l;
  BatchPlan p;
  __device__ long long tiles() const { return p.total; }
  __device__ void get(long long t, const Grid** gg, const StateP** uu, double* ga,
                      unsigned char** fl, int* i0, int* j0) const {
    int local, bx, by;
    const int inst = batch_locate(p, int(t), &local);
    const BatchRec& q = r[inst];
    batch_block(kBpInd, q.a.g, local, &bx, &by);
    *gg = &q.a.g;
    *uu = &q.a.u;
    *ga = q.a.gamma;
    *fl = l[inst].flag;
    *i0 = bx * kTileX - q.a.g.ng;
    *j0 = by * kTileY - q.a.g.ng;
  }
};

template <class Src>
__global__ void __launch_bounds__(kThreads) k_indicator(Src src, MlpDev p, float thr, int* status) {
  extern __shared__ __align__(1024) uint8_t sm[];
  uint8_t* xs = sm;
  uint8_t* w1s = xs + InfSmem::kX;
  uint8_t* w2s = w1s + InfSmem::kW1;
  uint8_t* a1s = w2s + InfSmem::kW2;
  // halo primitives in two planes of 16-byte records, (rho, vx, vy, vz) and
  // (p, bx, by, bz) per cell, so that eight lanes reading eight neighbouring
  // cells read 128 contiguous bytes (one 32-byte record per cell put two
  // lanes on the same banks)
  float* prim = reinterpret_cast<float*>(a1s + InfSmem::kA1);
  float4* pra = reinterpret_cast<float4*>(prim);            // [12][20]
  float4* prb = pra + kHaloX * kHaloY;                       // [12][20]
  unsigned char* okt = reinterpret_cast<unsigned char*>(prim + kHaloX * kHaloY * 8);
  // the bias and head vectors, which every thread reads at the same index
  float* vb1 = reinterpret_cast<float*>(okt + InfSmem::kOk);
  float* vb2 = vb1 + kHidden;
  float* vw3 = vb2 + kHidden;
  uint64_t* bar = reinterpret_cast<uint64_t*>(okt + InfSmem::kOk + InfSmem::kVec);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, row = warp * 32 + lane;
  const int tx = row % kTileX, ty = row / kTileX;
  if (tid == 0) {
    tc::mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tc::tmem_alloc(tslot, 128);
  stage_rows(w1s, p.w1, kHidden, kFeatPad, 0, kHidden, tid, kThreads);
  stage_rows(w2s, p.w2, kHidden, kHidden, 0, kHidden, tid, kThreads);
  for (int e = tid; e < kHidden; e += kThreads) {
    vb1[e] = p.b1[e];
    vb2[e] = p.b2[e];
    vw3[e] = p.w3[e];
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tb = *tslot;
  const uint32_t idesc = tc::idesc_bf16(128, kHidden);
  const long long tiles = src.tiles();
  uint32_t phase = 0;
  bool ok = true;
  for (long long t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
    const Grid* gp;
    const StateP* up;
    double gamma;
    unsigned char* flag;
    int i0, j0;
    src.get(t, &gp, &up, &gamma, &flag, &i0, &j0);
    const Grid& g = *gp;
    const StateP& u = *up;
    for (int e = tid; e < kHaloX * kHaloY; e += kThreads) {
      const int rr = e / kHaloX, cc = e - rr * kHaloX;
      const int ci = i0 - 2 + cc, cj = j0 - 2 + rr;
      bool good = false;
      float w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      if (ci >= -g.ng && ci < g.nx + g.ng && cj >= -g.ng && cj < g.ny + g.ng)
        good = cell_prim(u, g.idx(ci, cj), gamma, w);
      pra[e] = make_float4(w[0], w[1], w[2], w[3]);
      prb[e] = make_float4(w[4], w[5], w[6], w[7]);
      okt[e] = good ? 1 : 0;
    }
    __syncthreads();
    bool forced = false;
    {
      bool all = true;
      for (int dj = 0; dj < 5; ++dj)
        for (int di = 0; di < 5; ++di) all = all && okt[(ty + dj) * kHaloX + tx + di] != 0;
      const int ce = (ty + 2) * kHaloX + tx + 2;
      const float4 ca = pra[ce], cb = prb[ce];
      if (all) {
        const float c[8] = {ca.x, ca.y, ca.z, ca.w, cb.x, cb.y, cb.z, cb.w};
        const Norm nm = make_norm(c, gamma);
        for (int dj = 0; dj < 5; ++dj)
          for (int di = 0; di < 5; ++di) {
            const int q = (ty + dj) * kHaloX + tx + di;
            *reinterpret_cast<uint4*>(xs + tc::kmajor_offset(row, 8 * (5 * dj + di), kFeatPad)) =
                features8h(pra[q], prb[q], ca, cb, nm);
          }
      } else {
        forced = true;
        for (int q = 0; q < 25; ++q)
          *reinterpret_cast<uint4*>(xs + tc::kmajor_offset(row, 8 * q, kFeatPad)) =
              make_uint4(0u, 0u, 0u, 0u);
      }
      *reinterpret_cast<uint4*>(xs + tc::kmajor_offset(row, 200, kFeatPad)) = make_uint4(0u, 0u, 0u, 0u);
    }
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (tid == 0) {
      const uint32_t xa = tc::smem_u32(xs), wa = tc::smem_u32(w1s);
      for (int s = 0; s < kFeatPad / 16; ++s)
        tc::mma_bf16(tb, tc::smem_desc(xa + 256 * s, 128, 26 * 128),
                     tc::smem_desc(wa + 256 * s, 128, 26 * 128), idesc, s > 0);
      tc::commit(bar);
    }
    ok = __syncthreads_and(tc::mbar_wait(bar, phase) ? 1 : 0) != 0;
    phase ^= 1;
    if (!ok) break;
    tc::fence_after_sync();
    for (int c0 = 0; c0 < kHidden; c0 += 16) {
      float z[16];
      tc::tmem_ld16(tc::tmem_addr(tb, warp * 32, c0), z);
      // eight consecutive columns of a row are one 16-byte core-matrix row
#pragma unroll
      for (int h = 0; h < 16; h += 8) {
        uint32_t w[4];
#pragma unroll
        for (int c = 0; c < 8; c += 2)
          w[c / 2] = pack_bf16x2(gelu(z[h + c] + vb1[c0 + h + c]),
                                 gelu(z[h + c + 1] + vb1[c0 + h + c + 1]));
        *reinterpret_cast<uint4*>(a1s + tc::kmajor_offset(row, c0 + h, kHidden)) =
            make_uint4(w[0], w[1], w[2], w[3]);
      }
    }
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (tid == 0) {
      const uint32_t aa = tc::smem_u32(a1s), wa = tc::smem_u32(w2s);
      for (int s = 0; s < kHidden / 16; ++s)
        tc::mma_bf16(tb + 64, tc::smem_desc(aa + 256 * s, 128, 8 * 128),
                     tc::smem_desc(wa + 256 * s, 128, 8 * 128), idesc, s > 0);
      tc::commit(bar);
    }
    ok = __syncthreads_and(tc::mbar_wait(bar, phase) ? 1 : 0) != 0;
    phase ^= 1;
    if (!ok) break;
    tc::fence_after_sync();
    float acc = p.b3[0];
    for (int c0 = 0; c0 < kHidden; c0 += 16) {
      float z[16];
      tc::tmem_ld16(tc::tmem_addr(tb, warp * 32, 64 + c0), z);
#pragma unroll
      for (int c = 0; c < 16; ++c) acc += vw3[c0 + c] * gelu(z[c] + vb2[c0 + c]);
    }
    const int i = i0 + tx, j = j0 + ty;
    if (i < g.nx + g.ng && j < g.ny + g.ng) flag[g.idx(i, j)] = (forced || !(acc <= thr)) ? 1 : 0;
    tc::fence_before_sync();
    __syncthreads();
  }
  if (!ok) {
    if (tid == 0) atomicOr(status, 1);
    tc::mbar_wait(bar, phase ^ 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_free(tb, 128);
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

namespace {
// Held-out tiles: a multiplicative hash of the tile index, so that the
// held-out set samples every column block of every snapshot.
bool held_out(long long t, int holdout) {
  if (holdout <= 0) return true;
  return ((unsigned long long)t * 0x9E3779B97F4A7C15ull >> 40) % (unsigned long long)holdout == 0;
}
int sm_count() {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}
unsigned cdivu(long long a, int b) { return unsigned((a + b - 1) / b); }
}  // namespace

void launch_cell_features(const Grid& g, const StateP& u, double gamma, uint16_t* rows,
                          unsigned char* bad, cudaStream_t s) {
  const long long n = (long long)g.nx * g.ny;
  k_cell_features<<<cdivu(n, 128), 128, 0, s>>>(g, u, gamma, rows, bad);
}

void launch_gather_labels(const Grid& g, const int* label, float tol, unsigned char* y,
                          cudaStream_t s) {
  const long long n = (long long)g.nx * g.ny;
  k_gather_labels<<<cdivu(n, 256), 256, 0, s>>>(g, label, tol, y);
}

int launch_mlp_grad(const uint16_t* x, const unsigned char* y, long long rows, const int* tiles,
                    int ntiles, const MlpDev& p, const uint16_t* w2t, float pos_weight,
                    float inv_n, float* partial, int* status, cudaStream_t s) {
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, GradSmem::kTotal);
    configured = true;
  }
  const int grid = ntiles < sm_count() ? ntiles : sm_count();
  if (grid <= 0) return 0;
  k_mlp_grad<<<grid, kThreads, GradSmem::kTotal, s>>>(x, y, rows, tiles, ntiles, p, w2t,
                                                       pos_weight, inv_n, partial, status);
  return grid;
}

void launch_reduce_partials(const float* partial, int ctas, float* grad, cudaStream_t s) {
  k_reduce_partials<<<cdivu(kParamCount + 1, 256), 256, 0, s>>>(partial, ctas, grad);
}

void launch_adam(float* params, float* m, float* v, const float* grad, int step, float lr,
                 float beta1, float beta2, float eps, uint16_t* w1b, uint16_t* w2b,
                 uint16_t* w2tb, cudaStream_t s) {
  const float c1 = float(1.0 / (1.0 - std::pow(double(beta1), step)));
  const float c2 = float(1.0 / (1.0 - std::pow(double(beta2), step)));
  k_adam<<<cdivu(kParamCount, 256), 256, 0, s>>>(params, m, v, grad, lr, beta1, beta2, eps, c1,
                                                   c2, w1b, w2b, w2tb);
}

cudaError_t configure_indicator_kernels() {
  cudaError_t e = cudaFuncSetAttribute(k_indicator<SingleSrc>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, InfSmem::kTotal);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_indicator<BatchSrc>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              InfSmem::kTotal);
}

cudaError_t launch_indicator(const Grid& g, const StateP& u, double gamma, const MlpDev& p,
                             float threshold, unsigned char* flag, int* status, cudaStream_t s) {
  const long long tiles = (long long)((g.pitch + kTileX - 1) / kTileX) *
                          ((g.ny + 2 * g.ng + kTileY - 1) / kTileY);
  const int grid = int(tiles < 2 * sm_count() ? tiles : 2 * sm_count());
  SingleSrc src{g, u, gamma, flag};
  k_indicator<SingleSrc><<<grid, kThreads, InfSmem::kTotal, s>>>(src, p, threshold, status);
  return cudaGetLastError();
}

cudaError_t launch_batch_indicator(const BatchRec* r, const BatchLearnRec* l, const BatchPlan& plan,
                                   const MlpDev& p, float threshold, int* status, cudaStream_t s) {
  const int grid = int(plan.total < 2 * sm_count() ? plan.total : 2 * sm_count());
  if (grid <= 0) return cudaSuccess;
  BatchSrc src{r, l, plan};
  k_indicator<BatchSrc><<<grid, kThreads, InfSmem::kTotal, s>>>(src, p, threshold, status);
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
  ick(cudaMalloc(&w2tb_, sizeof(uint16_t) * kHidden * kHidden), "indicator w2t");
  ick(cudaMalloc(&adam_m_, sizeof(float) * kParamCount), "indicator adam");
  ick(cudaMalloc(&adam_v_, sizeof(float) * kParamCount), "indicator adam");
  ick(cudaMalloc(&grad_, sizeof(float) * (kParamCount + 1)), "indicator grad");
  ick(cudaMalloc(&partial_, sizeof(float) * (kParamCount + 1) * size_t(sm_count())), "indicator partials");
  ick(cudaMemset(adam_m_, 0, sizeof(float) * kParamCount), "indicator adam");
  ick(cudaMemset(adam_v_, 0, sizeof(float) * kParamCount), "indicator adam");
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
  cudaFree(w2tb_);
  cudaFree(adam_m_);
  cudaFree(adam_v_);
  cudaFree(grad_);
  cudaFree(partial_);
  cudaFree(tiles_);
  cudaFree(xs_);
  cudaFree(ys_);
  cudaFree(label_);
  cudaFree(status_);
  if (stream_) cudaStreamDestroy(stream_);
}

void Indicator::upload_bf16_from_host(const std::vector<float>& h) {
  std::vector<uint16_t> w1(size_t(kHidden) * kFeatPad, 0), w2(size_t(kHidden) * kHidden),
      w2t(size_t(kHidden) * kHidden);
  for (int o = 0; o < kHidden; ++o)
    for (int i = 0; i < kFeat; ++i) w1[size_t(o) * kFeatPad + i] = bf16_bits(h[size_t(o) * kFeat + i]);
  const float* hw2 = h.data() + kHidden * kFeat + kHidden;
  for (int o = 0; o < kHidden; ++o)
    for (int i = 0; i < kHidden; ++i) {
      w2[size_t(o) * kHidden + i] = bf16_bits(hw2[o * kHidden + i]);
      w2t[size_t(i) * kHidden + o] = bf16_bits(hw2[o * kHidden + i]);
    }
  ick(cudaMemcpyAsync(w2tb_, w2t.data(), sizeof(uint16_t) * w2t.size(), cudaMemcpyHostToDevice,
                      stream_),
      "indicator w2t");
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

double Indicator::gradient(const float* features, const unsigned char* labels, long long rows,
                           float pos_weight, float* grad) {
  if (rows <= 0) throw std::invalid_argument("indicator gradient: rows must be > 0");
  std::vector<uint16_t> x(size_t(rows) * kFeatPad, 0);
  for (long long r = 0; r < rows; ++r)
    for (int i = 0; i < kFeat; ++i) x[size_t(r) * kFeatPad + i] = bf16_bits(features[r * kFeat + i]);
  const int ntiles = int((rows + 127) / 128);
  std::vector<int> tl(static_cast<size_t>(ntiles));
  std::iota(tl.begin(), tl.end(), 0);
  uint16_t* dx = nullptr;
  unsigned char* dy = nullptr;
  int* dt = nullptr;
  ick(cudaMalloc(&dx, sizeof(uint16_t) * x.size()), "gradient rows");
  ick(cudaMalloc(&dy, size_t(rows)), "gradient labels");
  ick(cudaMalloc(&dt, sizeof(int) * tl.size()), "gradient tiles");
  std::vector<float> g(kParamCount + 1);
  try {
    ick(cudaMemcpyAsync(dx, x.data(), sizeof(uint16_t) * x.size(), cudaMemcpyHostToDevice, stream_), "rows");
    ick(cudaMemcpyAsync(dy, labels, size_t(rows), cudaMemcpyHostToDevice, stream_), "labels");
    ick(cudaMemcpyAsync(dt, tl.data(), sizeof(int) * tl.size(), cudaMemcpyHostToDevice, stream_), "tiles");
    const int ctas = launch_mlp_grad(dx, dy, rows, dt, ntiles, dev(), w2tb_, pos_weight,
                                     1.0f / float(rows), partial_, status_, stream_);
    launch_reduce_partials(partial_, ctas, grad_, stream_);
    ick(cudaGetLastError(), "gradient launch");
    ick(cudaMemcpyAsync(g.data(), grad_, sizeof(float) * g.size(), cudaMemcpyDeviceToHost, stream_), "grad");
    check_status("indicator gradient");
  } catch (...) {
    cudaFree(dx);
    cudaFree(dy);
    cudaFree(dt);
    throw;
  }
  cudaFree(dx);
  cudaFree(dy);
  cudaFree(dt);
  std::copy(g.begin(), g.begin() + kParamCount, grad);
  return double(g[kParamCount]);
}

void Indicator::ensure_capacity(long long rows) {
  if (rows <= cap_) return;
  long long ncap = std::max<long long>(rows, cap_ * 2);
  ncap = (ncap + 127) / 128 * 128;
  uint16_t* nx = nullptr;
  unsigned char* ny = nullptr;
  ick(cudaMalloc(&nx, sizeof(uint16_t) * size_t(ncap) * kFeatPad), "training rows");
  ick(cudaMalloc(&ny, size_t(ncap)), "training labels");
  if (rows_ > 0) {
    ick(cudaMemcpyAsync(nx, xs_, sizeof(uint16_t) * size_t(rows_) * kFeatPad,
                        cudaMemcpyDeviceToDevice, stream_), "grow rows");
    ick(cudaMemcpyAsync(ny, ys_, size_t(rows_), cudaMemcpyDeviceToDevice, stream_), "grow labels");
  }
  ick(cudaStreamSynchronize(stream_), "grow");
  cudaFree(xs_);
  cudaFree(ys_);
  xs_ = nx;
  ys_ = ny;
  cap_ = ncap;
}

// Feature rows and limiter labels of every interior cell of a live state
// (the solver's own reconstruction run once per direction with recording):
// label 1 where a limited face state departs by more than `tol`, or, for a
// negative tol, where the limiter fired on any characteristic field.
void Indicator::collect(const StageArgs& a, cudaStream_t solver_stream, float tol) {
  if (tol != tol) throw std::invalid_argument("indicator: label tolerance is NaN");
  const int literal = tol < 0.0f ? 1 : 0;
  if (literal) tol = 0.0f;
  if (a.order != 5 && a.order != 7)
    throw std::invalid_argument("indicator: training data needs an mp5 or mp7 solver");
  const Grid& g = a.g;
  const long long n = (long long)g.nx * g.ny;
  ensure_capacity(rows_ + n);
  if (g.size() > label_cap_) {
    cudaFree(label_);
    label_ = nullptr;
    ick(cudaMalloc(&label_, sizeof(int) * size_t(g.size())), "labels");
    label_cap_ = g.size();
  }
  cudaEvent_t ev;
  ick(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "event");
  ick(cudaEventRecord(ev, solver_stream), "event");
  ick(cudaStreamWaitEvent(stream_, ev, 0), "event wait");
  cudaEventDestroy(ev);
  ick(cudaMemsetAsync(label_, 0, sizeof(int) * size_t(g.size()), stream_), "labels");
  launch_reconstruct_label(a, 0, label_, literal, stream_);
  launch_reconstruct_label(a, 1, label_, literal, stream_);
  unsigned char* bad = nullptr;
  ick(cudaMalloc(&bad, size_t(n)), "bad rows");
  launch_cell_features(g, a.u, a.gamma, xs_ + size_t(rows_) * kFeatPad, bad, stream_);
  launch_gather_labels(g, label_, tol, ys_ + rows_, stream_);
  ick(cudaGetLastError(), "collect launch");
  ick(cudaStreamSynchronize(stream_), "collect");
  cudaFree(bad);
  rows_ += n;
}

void Indicator::labels_to_host(unsigned char* out, long long n) const {
  if (n != rows_)
    throw std::invalid_argument("indicator: labels buffer holds " + std::to_string(n) +
                                " rows, " + std::to_string(rows_) + " collected");
  if (n == 0) return;
  ick(cudaMemcpyAsync(out, ys_, size_t(n), cudaMemcpyDeviceToHost, stream_), "labels to host");
  ick(cudaStreamSynchronize(stream_), "labels to host");
}

double Indicator::train(int epochs, int tiles_per_step, float lr, float pos_weight, int holdout,
                        unsigned long long seed) {
  const int total_tiles = int(rows_ / 128);  // whole tiles only
  std::vector<int> pool;
  for (int t = 0; t < total_tiles; ++t)
    if (holdout <= 0 || !held_out(t, holdout)) pool.push_back(t);
  if (pool.empty()) throw std::invalid_argument("indicator: no training rows collected");
  tiles_per_step = std::max(1, std::min<int>(tiles_per_step, int(pool.size())));
  if (tiles_cap_ < tiles_per_step) {
    cudaFree(tiles_);
    tiles_ = nullptr;
    ick(cudaMalloc(&tiles_, sizeof(int) * size_t(tiles_per_step)), "tile list");
    tiles_cap_ = tiles_per_step;
  }
  std::mt19937_64 rng(seed);
  double last = 0.0;
  std::vector<float> lossv(1);
  for (int ep = 0; ep < epochs; ++ep) {
    std::shuffle(pool.begin(), pool.end(), rng);
    double sum = 0.0;
    int steps = 0;
    for (size_t off = 0; off + size_t(tiles_per_step) <= pool.size(); off += size_t(tiles_per_step)) {
      ick(cudaMemcpyAsync(tiles_, pool.data() + off, sizeof(int) * size_t(tiles_per_step),
                          cudaMemcpyHostToDevice, stream_), "tile list");
      const long long nrows = (long long)tiles_per_step * 128;
      const int ctas = launch_mlp_grad(xs_, ys_, rows_, tiles_, tiles_per_step, dev(), w2tb_,
                                       pos_weight, 1.0f / float(nrows), partial_, status_, stream_);
      launch_reduce_partials(partial_, ctas, grad_, stream_);
      launch_adam(params_, adam_m_, adam_v_, grad_, ++adam_step_, lr, 0.9f, 0.999f, 1e-8f, w1b_,
                  w2b_, w2tb_, stream_);
      ick(cudaGetLastError(), "train launch");
      ick(cudaMemcpyAsync(lossv.data(), grad_ + kParamCount, sizeof(float), cudaMemcpyDeviceToHost,
                          stream_), "loss");
      ick(cudaStreamSynchronize(stream_), "train step");
      sum += lossv[0];
      ++steps;
    }
    check_status("indicator train");
    last = steps ? sum / steps : 0.0;
  }
  return last;
}

void Indicator::logits_of_tiles(int holdout, std::vector<float>* logit,
                                std::vector<unsigned char>* y) {
  const long long total_tiles = rows_ / 128;
  logit->clear();
  y->clear();
  if (total_tiles == 0) return;
  const long long n = total_tiles * 128;
  float* dl = nullptr;
  ick(cudaMalloc(&dl, sizeof(float) * size_t(n)), "eval logits");
  std::vector<float> all(static_cast<size_t>(n));
  std::vector<unsigned char> ally(static_cast<size_t>(n));
  try {
    ick(launch_mlp_forward(xs_, n, dev(), dl, status_, stream_), "eval forward");
    ick(cudaMemcpyAsync(all.data(), dl, sizeof(float) * size_t(n), cudaMemcpyDeviceToHost, stream_),
        "eval logits");
    ick(cudaMemcpyAsync(ally.data(), ys_, size_t(n), cudaMemcpyDeviceToHost, stream_), "eval y");
    check_status("indicator evaluate");
  } catch (...) {
    cudaFree(dl);
    throw;
  }
  cudaFree(dl);
  for (long long t = 0; t < total_tiles; ++t) {
    if (!held_out(t, holdout)) continue;
    logit->insert(logit->end(), all.begin() + t * 128, all.begin() + (t + 1) * 128);
    y->insert(y->end(), ally.begin() + t * 128, ally.begin() + (t + 1) * 128);
  }
}

void Indicator::evaluate(float threshold, int holdout, double* recall, double* flagged,
                         long long* positives, long long* total) {
  std::vector<float> lg;
  std::vector<unsigned char> y;
  logits_of_tiles(holdout, &lg, &y);
  long long pos = 0, hit = 0, fl = 0;
  for (size_t k = 0; k < lg.size(); ++k) {
    const bool f = !(lg[k] <= threshold);
    fl += f;
    if (y[k]) {
      ++pos;
      hit += f;
    }
  }
  *recall = pos ? double(hit) / double(pos) : 1.0;
  *flagged = lg.empty() ? 0.0 : double(fl) / double(lg.size());
  *positives = pos;
  *total = (long long)lg.size();
}

float Indicator::threshold_for_recall(double recall, int holdout) {
  std::vector<float> lg;
  std::vector<unsigned char> y;
  logits_of_tiles(holdout, &lg, &y);
  std::vector<float> pos;
  for (size_t k = 0; k < lg.size(); ++k)
    if (y[k]) pos.push_back(lg[k]);
  if (pos.empty()) return 0.f;
  std::sort(pos.begin(), pos.end());
  const size_t miss = size_t(std::floor((1.0 - recall) * double(pos.size())));
  const size_t k = std::min(miss, pos.size() - 1);
  // flag strictly above the threshold: step just below the k-th smallest
  return std::nextafter(pos[k], -INFINITY);
}

}  // namespace qb
