// FP64 FMA throughput probe: the denominator of the FP64 roofline, measured
// on the device the solver runs on (eight independent FMA chains per thread,
// enough resident warps to cover the pipe latency).
#include <cuda_runtime.h>

namespace qb {

__global__ void __launch_bounds__(256) k_fp64_fma(double* out, int iters, double a, double b) {
  double x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3;
  double x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
  for (int i = 0; i < iters; ++i) {
    x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
    x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
  }
  const double s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
  if (s == 12345.678) out[0] = s;  // keeps the chains live; never true
}

// Returns the best of three timed launches in TFLOP/s (2 flops per FMA).
double fp64_fma_peak_tflops() {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  double* out = nullptr;
  if (cudaMalloc(&out, sizeof(double)) != cudaSuccess) return -1.0;
  const int blocks = sms * 8, threads = 256, iters = 1 << 14;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  k_fp64_fma<<<blocks, threads>>>(out, 64, 0.9999999, 1e-7);
  double best = 0.0;
  for (int r = 0; r < 3; ++r) {
    cudaEventRecord(a);
    k_fp64_fma<<<blocks, threads>>>(out, iters, 0.9999999, 1e-7);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    const double flops = 2.0 * 8.0 * double(iters) * double(blocks) * threads;
    if (ms > 0.f) best = best > flops / (ms * 1e-3) ? best : flops / (ms * 1e-3);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  return best / 1e12;
}

}  // namespace qb
