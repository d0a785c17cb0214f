// Precision-independent pieces of the public C++ API: device selection and
// the reference-counted device allocations behind VectorView.
#include <cuda_runtime.h>

#include <atomic>
#include <memory>

#include "engine/runtime.hpp"
#include "qkrylov/core/device.hpp"
#include "qkrylov/core/kokkos_types.hpp"

namespace qkrylov {
namespace detail {

namespace {
std::atomic<int> g_default_device{-1};
}

int gpu_count() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) { (void)cudaGetLastError(); return 0; }
  return n;
}

void set_default_device(int id) {
  int expected = -1;
  g_default_device.compare_exchange_strong(expected, id);  // first selection wins, as Kokkos init
}

int default_device() {
  const int d = g_default_device.load();
  return d < 0 ? 0 : d;
}

std::shared_ptr<void> device_alloc(std::size_t bytes, int device) {
  qkb::Context& c = qkb::Context::get(device);
  if (bytes == 0) return std::shared_ptr<void>();
  void* p = nullptr;
  qkb::cuda_check(cudaMalloc(&p, bytes), "device allocation");
  qkb::cuda_check(cudaMemsetAsync(p, 0, bytes, c.stream), "memset");
  c.sync();
  return std::shared_ptr<void>(p, [device](void* q) { cudaSetDevice(device); cudaFree(q); });
}

}  // namespace detail
}  // namespace qkrylov
