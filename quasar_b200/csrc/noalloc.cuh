// Allocation-free conserved totals over caller-owned device arrays.
#pragma once
#include <cuda_runtime.h>

namespace qb {

constexpr long long kTotalsChunk = 8192;      // cells per partial
constexpr int kTotalsMaxPartials = 8192;      // scratch: 8192 x 4 doubles (256 KiB)
constexpr long long kTotalsMaxCells = kTotalsChunk * kTotalsMaxPartials;  // 67,108,864
constexpr int kTotalsMaxDevices = 64;

// Device address of the static scratch on `device` (the calling thread's
// current device); the lookup runs once per device.
cudaError_t totals_scratch(int device, double** ptr);

// Launch the chunked sums and the final reduction on `stream`, copy the two
// totals to host and synchronize the stream.  Sizes must already be checked.
cudaError_t launch_totals_noalloc(const double* rho, const double* energy, int nx, int ny, int ng,
                                  double* scratch, cudaStream_t stream, double totals[2]);

}  // namespace qb
