// Conserved-totals reduction over caller-owned device arrays whose scratch is
// a file-scope device array: nothing is allocated per call or per set-up.
//
// Variant of k_cell_sums (the solver's compensated mass / energy totals,
// mhd_solver.cpp:1376-1382) for callers that hold the state in their own
// device buffers and cannot allocate.  Work is split into fixed chunks of
// kTotalsChunk cells, one block each, so the scratch needed grows with the
// cell count and is bounded by kTotalsMaxPartials.
#include "noalloc.cuh"

#include <mutex>

namespace qb {
namespace {

constexpr int kThreads = 256;

// Per-chunk partials (sum, compensation) x (mass, energy), then the two
// final totals.  Every slot a call reads is written earlier by the same
// call, so nothing here has to start at zero.
static __device__ __align__(256) double g_totals_scratch[4 * kTotalsMaxPartials + 2];

// One lock per device, held from the scratch lookup until the stream has
// synchronized: calls from different host threads on one device take turns
// instead of sharing the scratch array at the same time.
std::mutex g_device_mu[kTotalsMaxDevices];

// s + v with its rounding error added to c (Knuth's TwoSum, no contraction).
__device__ __forceinline__ void comp_add(double& s, double& c, double v) {
  const double t = __dadd_rn(s, v);
  const double bp = __dsub_rn(t, s);
  const double e = __dadd_rn(__dsub_rn(s, __dsub_rn(t, bp)), __dsub_rn(v, bp));
  s = t;
  c = __dadd_rn(c, e);
}

// Serial compensated sum of the block's (sum, compensation) pairs by thread 0.
__device__ __forceinline__ void block_pairs(double (*sm)[kThreads], double (*sc)[kThreads],
                                            double out[4]) {
  for (int q = 0; q < 2; ++q) {
    double s = 0.0, c = 0.0;
    for (int t = 0; t < kThreads; ++t) {
      comp_add(s, c, sm[q][t]);
      c = __dadd_rn(c, sc[q][t]);
    }
    out[2 * q] = s;
    out[2 * q + 1] = c;
  }
}

__global__ void __launch_bounds__(kThreads)
k_cell_sums_chunk(const double* __restrict__ rho, const double* __restrict__ energy, int nx,
                  long long cells, int ng, long long pitch, double* __restrict__ partial) {
  __shared__ double sm[2][kThreads], sc[2][kThreads];
  const int tid = threadIdx.x;
  const long long begin = (long long)blockIdx.x * kTotalsChunk;
  const long long end = begin + kTotalsChunk < cells ? begin + kTotalsChunk : cells;
  double s0 = 0.0, c0 = 0.0, s1 = 0.0, c1 = 0.0;
  for (long long t = begin + tid; t < end; t += kThreads) {
    const long long i = t % nx, j = t / nx;
    const long long k = (i + ng) + pitch * (j + ng);
    comp_add(s0, c0, rho[k]);
    comp_add(s1, c1, energy[k]);
  }
  sm[0][tid] = s0; sc[0][tid] = c0;
  sm[1][tid] = s1; sc[1][tid] = c1;
  __syncthreads();
  if (tid == 0) {
    double out[4];
    block_pairs(sm, sc, out);
    for (int q = 0; q < 4; ++q) partial[4 * (long long)blockIdx.x + q] = out[q];
  }
}

__global__ void __launch_bounds__(kThreads)
k_sum_partials(const double* __restrict__ partial, int parts, double* __restrict__ totals) {
  __shared__ double sm[2][kThreads], sc[2][kThreads];
  const int tid = threadIdx.x;
  double s0 = 0.0, c0 = 0.0, s1 = 0.0, c1 = 0.0;
  for (int b = tid; b < parts; b += kThreads) {
    comp_add(s0, c0, partial[4 * b]);
    c0 = __dadd_rn(c0, partial[4 * b + 1]);
    comp_add(s1, c1, partial[4 * b + 2]);
    c1 = __dadd_rn(c1, partial[4 * b + 3]);
  }
  sm[0][tid] = s0; sc[0][tid] = c0;
  sm[1][tid] = s1; sc[1][tid] = c1;
  __syncthreads();
  if (tid == 0) {
    double out[4];
    block_pairs(sm, sc, out);
    totals[0] = __dadd_rn(out[0], out[1]);
    totals[1] = __dadd_rn(out[2], out[3]);
  }
}

}  // namespace

cudaError_t totals_noalloc(int device, const double* rho, const double* energy, int nx, int ny,
                          int ng, cudaStream_t stream, double totals[2]) {
  if (device < 0 || device >= kTotalsMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_device_mu[device]);
  // The symbol's address is looked up on every call (it allocates nothing),
  // so it always belongs to the context that is current now, also after a
  // cudaDeviceReset.
  double* scratch = nullptr;
  cudaError_t rc = cudaGetSymbolAddress((void**)&scratch, g_totals_scratch);
  if (rc != cudaSuccess) return rc;
  const long long cells = (long long)nx * ny;
  const int parts = int((cells + kTotalsChunk - 1) / kTotalsChunk);
  double* partial = scratch;
  double* result = scratch + 4 * kTotalsMaxPartials;
  k_cell_sums_chunk<<<parts, kThreads, 0, stream>>>(rho, energy, nx, cells, ng,
                                                    (long long)nx + 2 * ng, partial);
  k_sum_partials<<<1, kThreads, 0, stream>>>(partial, parts, result);
  rc = cudaGetLastError();
  if (rc != cudaSuccess) return rc;
  rc = cudaMemcpyAsync(totals, result, 2 * sizeof(double), cudaMemcpyDeviceToHost, stream);
  if (rc != cudaSuccess) return rc;
  return cudaStreamSynchronize(stream);
}

}  // namespace qb
