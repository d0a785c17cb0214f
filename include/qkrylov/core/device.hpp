// Device selection (the same struct as qkrylov's include/qkrylov/core/device.hpp:27-80):
// "cuda:1", "gpu:0", "gpu" or an integer id.  This library always targets
// CUDA GPUs; "cpu" selects device 0, since there is no CPU back-end.
#pragma once

#include <string>

#include "qkrylov/core/types.hpp"

namespace qkrylov {
namespace detail {
int gpu_count();
void set_default_device(int id);
int default_device();
}  // namespace detail

namespace QKRYLOV_PRECISION_NAMESPACE {

struct Device {
  int id = 0;
  Device() = default;
  explicit Device(int device_id) : id(device_id) {}
  explicit Device(const std::string& s) {
    if (s == "cpu") { id = 0; return; }
    const auto colon = s.find(':');
    id = (colon == std::string::npos) ? 0 : std::stoi(s.substr(colon + 1));
  }
  static bool is_gpu_build() { return true; }
  static std::string backend_name() { return "cuda"; }
  static int gpu_count() { return qkrylov::detail::gpu_count(); }
};

namespace detail {
// First use selects the device every default-constructed vector lives on,
// as Kokkos initialisation does in qkrylov (device.hpp:105-116).
inline void initialize_kokkos(const Device& dev = Device()) { qkrylov::detail::set_default_device(dev.id); }
inline void ensure_kokkos_initialized() {}
}  // namespace detail

}  // namespace QKRYLOV_PRECISION_NAMESPACE
}  // namespace qkrylov
