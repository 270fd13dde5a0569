// Host implementation of the reference's backend-neutral device interface
// (include/quasar/backend/device.hpp:17-105) for the CPU build of the
// reference MHD path.  "Device" memory is ordinary host memory; every launch
// completes synchronously inside the shim, so synchronisation is a no-op.
// Also stubs the two background/radial entry points that Cartesian,
// background-free runs never reach (mhd_solver.cpp only calls them when
// background.enabled or geometry == "cylindrical").
#include "quasar/backend/device.hpp"
#include "quasar/numerics/radial_moments.hpp"
#include "quasar/physics/mhd/background_builder.hpp"

#include <cstdlib>
#include <cstring>
#include <stdexcept>

namespace quasar::backend {

int device_count() { return 1; }
bool has_hip_runtime() { return true; }
int current_device() { return 0; }
void set_device(int) {}
bool try_set_device(int) noexcept { return true; }
DeviceGuard::DeviceGuard(int) {}
DeviceGuard::~DeviceGuard() noexcept {}
std::string device_uuid(int) { return "host"; }
std::string device_pci_bus_id(int) { return "host"; }
bool device_can_access_peer(int, int) { return true; }
void device_enable_peer_access(int) {}
stream_t stream_create() { return nullptr; }
void stream_destroy(stream_t) noexcept {}
event_t event_create() { return nullptr; }
void event_destroy(event_t) noexcept {}
void event_record(event_t, stream_t) {}
void event_synchronize(event_t) {}
void stream_wait_event(stream_t, event_t) {}
void* device_alloc(std::size_t n) { return std::calloc(n ? n : 1, 1); }
void* device_alloc_uninit(std::size_t n) { return std::malloc(n ? n : 1); }
void device_free(void* p) noexcept { std::free(p); }
void device_free_on(void* p, int) noexcept { std::free(p); }
void device_memset(void* p, int v, std::size_t n) { std::memset(p, v, n); }
void device_memset_async(void* p, int v, std::size_t n, stream_t) {
  std::memset(p, v, n);
}
void device_memcpy_h2d(void* d, const void* s, std::size_t n) {
  std::memcpy(d, s, n);
}
void device_memcpy_d2h(void* d, const void* s, std::size_t n) {
  std::memcpy(d, s, n);
}
void device_memcpy_h2d_async(void* d, const void* s, std::size_t n, stream_t) {
  std::memcpy(d, s, n);
}
void device_memcpy_d2h_async(void* d, const void* s, std::size_t n, stream_t) {
  std::memcpy(d, s, n);
}
void device_memcpy_d2d_async(void* d, const void* s, std::size_t n, stream_t) {
  std::memmove(d, s, n);
}
void device_memcpy_peer_async(void* d, int, const void* s, int, std::size_t n,
                              stream_t) {
  std::memcpy(d, s, n);
}
void* pinned_host_alloc(std::size_t n) { return std::malloc(n ? n : 1); }
void pinned_host_free(void* p) noexcept { std::free(p); }
void device_synchronize(stream_t) {}

}  // namespace quasar::backend

namespace quasar::mhd {
MhdBackgroundAffineProfile lower_affine_background_profile(
    const numerics::IMhdBackgroundProfile&, const std::string&) {
  throw std::logic_error("background profiles are not part of this library");
}
void build_background_from_profile(const MhdBackgroundBuildSpec&,
                                   MhdBackgroundField<Real>&,
                                   backend::stream_t) {
  throw std::logic_error("background profiles are not part of this library");
}
}  // namespace quasar::mhd

namespace quasar::numerics {
std::vector<RadialStencilRow> solve_radial_rows(
    const std::vector<RadialRowSpec>&, backend::stream_t) {
  throw std::logic_error("cylindrical tables are not part of this library");
}
std::vector<RadialStencilRow> radial_gauss_weight_rows(
    const std::vector<RadialGaussSpec>&, backend::stream_t) {
  throw std::logic_error("cylindrical tables are not part of this library");
}
std::vector<Real> radial_face_extrapolation_factors(
    const std::vector<RadialExtrapolationSpec>&, backend::stream_t) {
  throw std::logic_error("cylindrical tables are not part of this library");
}
}  // namespace quasar::numerics
