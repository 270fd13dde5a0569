// The reference's backend-neutral device interface
// (include/quasar/backend/device.hpp:17-105) over the CUDA runtime, for the
// build that links the reference's own, unmodified MhdSolver2D against this
// project's kernels (oracle/build_seam.sh).  Semantics follow the reference's
// runtime (src/backend/hip/device_memory.cpp): device_alloc zero-fills, a
// zero-byte allocation is a null pointer, device_synchronize synchronises the
// given stream, failures throw DeviceError.  Also stubs the two
// background-builder entry points and the three cylindrical radial-table
// builders that Cartesian, background-free runs never reach (mhd_solver.cpp
// calls them only when background.enabled or geometry == "cylindrical").
//
// Test infrastructure: built only where the reference tree is present; the
// product is libquasar_mhd_b200.so.
#include "quasar/backend/device.hpp"
#include "quasar/numerics/radial_moments.hpp"
#include "quasar/physics/mhd/background_builder.hpp"

#include <cuda_runtime.h>

#include <stdexcept>

namespace quasar::backend {
namespace {
void ok(cudaError_t e, const char* file, int line) {
  if (e != cudaSuccess) throw DeviceError(static_cast<int>(e), cudaGetErrorString(e), file, line);
}
#define SEAM_CUDA(call) ok((call), __FILE__, __LINE__)
cudaStream_t S(stream_t s) { return static_cast<cudaStream_t>(s); }
}  // namespace

int device_count() {
  int n = 0;
  return cudaGetDeviceCount(&n) == cudaSuccess ? n : 0;
}
bool has_hip_runtime() { return device_count() > 0; }
int current_device() {
  int d = 0;
  SEAM_CUDA(cudaGetDevice(&d));
  return d;
}
void set_device(int d) { SEAM_CUDA(cudaSetDevice(d)); }
bool try_set_device(int d) noexcept { return cudaSetDevice(d) == cudaSuccess; }
DeviceGuard::DeviceGuard(int d) {
  previous_device_ = current_device();
  if (d != previous_device_) {
    set_device(d);
    restore_ = true;
  }
}
DeviceGuard::~DeviceGuard() noexcept {
  if (restore_) (void)cudaSetDevice(previous_device_);
}
std::string device_uuid(int d) {
  cudaDeviceProp p{};
  SEAM_CUDA(cudaGetDeviceProperties(&p, d));
  static const char* hex = "0123456789abcdef";
  std::string s;
  for (int k = 0; k < 16; ++k) {
    const unsigned char b = static_cast<unsigned char>(p.uuid.bytes[k]);
    s += hex[b >> 4];
    s += hex[b & 15];
  }
  return s;
}
std::string device_pci_bus_id(int d) {
  char buf[64] = {};
  SEAM_CUDA(cudaDeviceGetPCIBusId(buf, sizeof buf, d));
  return buf;
}
bool device_can_access_peer(int d, int peer) {
  int can = 0;
  SEAM_CUDA(cudaDeviceCanAccessPeer(&can, d, peer));
  return can != 0;
}
void device_enable_peer_access(int peer) {
  const cudaError_t e = cudaDeviceEnablePeerAccess(peer, 0);
  if (e == cudaErrorPeerAccessAlreadyEnabled) {
    (void)cudaGetLastError();
    return;
  }
  SEAM_CUDA(e);
}
stream_t stream_create() {
  cudaStream_t s = nullptr;
  SEAM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  return s;
}
void stream_destroy(stream_t s) noexcept {
  if (s) (void)cudaStreamDestroy(S(s));
}
event_t event_create() {
  cudaEvent_t e = nullptr;
  SEAM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  return e;
}
void event_destroy(event_t e) noexcept {
  if (e) (void)cudaEventDestroy(static_cast<cudaEvent_t>(e));
}
void event_record(event_t e, stream_t s) {
  SEAM_CUDA(cudaEventRecord(static_cast<cudaEvent_t>(e), S(s)));
}
void event_synchronize(event_t e) { SEAM_CUDA(cudaEventSynchronize(static_cast<cudaEvent_t>(e))); }
void stream_wait_event(stream_t s, event_t e) {
  SEAM_CUDA(cudaStreamWaitEvent(S(s), static_cast<cudaEvent_t>(e), 0));
}
void* device_alloc_uninit(std::size_t n) {
  if (n == 0) return nullptr;
  void* p = nullptr;
  SEAM_CUDA(cudaMalloc(&p, n));
  return p;
}
void* device_alloc(std::size_t n) {
  void* p = device_alloc_uninit(n);
  if (!p) return p;
  const cudaError_t e = cudaMemset(p, 0, n);
  if (e != cudaSuccess) {
    (void)cudaFree(p);
    SEAM_CUDA(e);
  }
  return p;
}
void device_free(void* p) noexcept {
  if (p) (void)cudaFree(p);
}
void device_free_on(void* p, int owner) noexcept {
  if (!p) return;
  int cur = 0;
  if (cudaGetDevice(&cur) != cudaSuccess) return;
  if (cur != owner) (void)cudaSetDevice(owner);
  (void)cudaFree(p);
  if (cur != owner) (void)cudaSetDevice(cur);
}
void device_memset(void* p, int v, std::size_t n) {
  if (n) SEAM_CUDA(cudaMemset(p, v, n));
}
void device_memset_async(void* p, int v, std::size_t n, stream_t s) {
  if (n) SEAM_CUDA(cudaMemsetAsync(p, v, n, S(s)));
}
void device_memcpy_h2d(void* d, const void* s, std::size_t n) {
  if (n) SEAM_CUDA(cudaMemcpy(d, s, n, cudaMemcpyHostToDevice));
}
void device_memcpy_d2h(void* d, const void* s, std::size_t n) {
  if (n) SEAM_CUDA(cudaMemcpy(d, s, n, cudaMemcpyDeviceToHost));
}
void device_memcpy_h2d_async(void* d, const void* s, std::size_t n, stream_t st) {
  if (n) SEAM_CUDA(cudaMemcpyAsync(d, s, n, cudaMemcpyHostToDevice, S(st)));
}
void device_memcpy_d2h_async(void* d, const void* s, std::size_t n, stream_t st) {
  if (n) SEAM_CUDA(cudaMemcpyAsync(d, s, n, cudaMemcpyDeviceToHost, S(st)));
}
void device_memcpy_d2d_async(void* d, const void* s, std::size_t n, stream_t st) {
  if (n) SEAM_CUDA(cudaMemcpyAsync(d, s, n, cudaMemcpyDeviceToDevice, S(st)));
}
void device_memcpy_peer_async(void* d, int dd, const void* s, int sd, std::size_t n,
                              stream_t st) {
  if (n) SEAM_CUDA(cudaMemcpyPeerAsync(d, dd, s, sd, n, S(st)));
}
void* pinned_host_alloc(std::size_t n) {
  if (n == 0) return nullptr;
  void* p = nullptr;
  SEAM_CUDA(cudaMallocHost(&p, n));
  return p;
}
void pinned_host_free(void* p) noexcept {
  if (p) (void)cudaFreeHost(p);
}
void device_synchronize(stream_t s) { SEAM_CUDA(cudaStreamSynchronize(S(s))); }

}  // namespace quasar::backend

namespace quasar::mhd {
MhdBackgroundAffineProfile lower_affine_background_profile(
    const numerics::IMhdBackgroundProfile&, const std::string&) {
  throw std::logic_error("background profiles are not part of this library");
}
void build_background_from_profile(const MhdBackgroundBuildSpec&, MhdBackgroundField<Real>&,
                                   backend::stream_t) {
  throw std::logic_error("background profiles are not part of this library");
}
}  // namespace quasar::mhd

namespace quasar::numerics {
std::vector<RadialStencilRow> solve_radial_rows(const std::vector<RadialRowSpec>&,
                                                backend::stream_t) {
  throw std::logic_error("cylindrical radial tables are not part of this library");
}
std::vector<RadialStencilRow> radial_gauss_weight_rows(const std::vector<RadialGaussSpec>&,
                                                       backend::stream_t) {
  throw std::logic_error("cylindrical radial tables are not part of this library");
}
std::vector<Real> radial_face_extrapolation_factors(const std::vector<RadialExtrapolationSpec>&,
                                                    backend::stream_t) {
  throw std::logic_error("cylindrical radial tables are not part of this library");
}
}  // namespace quasar::numerics
