// Allocation-free conserved totals over caller-owned device arrays.
#pragma once
#include <cuda_runtime.h>

namespace qb {

constexpr long long kTotalsChunk = 8192;      // cells per partial
constexpr int kTotalsMaxPartials = 8192;      // scratch: 8192 x 4 doubles (256 KiB)
constexpr long long kTotalsMaxCells = kTotalsChunk * kTotalsMaxPartials;  // 67,108,864
constexpr int kTotalsMaxDevices = 64;

// Under a per-device lock: look up the static scratch's address in the
// current context, launch the chunked sums and the final reduction on
// `stream`, copy the two totals to host and synchronize the stream.  `device`
// is the calling thread's current device; sizes must already be checked.
cudaError_t totals_noalloc(int device, const double* rho, const double* energy, int nx, int ny,
                          int ng, cudaStream_t stream, double totals[2]);

}  // namespace qb
