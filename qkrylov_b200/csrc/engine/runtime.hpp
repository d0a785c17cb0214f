// Device runtime for the host layer: one context (stream, reduction
// workspace, pinned result buffer) per GPU, RAII device vectors, and the
// mapping of CUDA / kernel status codes to C++ exceptions.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "kernels/dev_api.h"

namespace qkb {

struct DeviceError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

void cuda_check(cudaError_t e, const char* what);
void qkd_check(int rc, const char* what);

class Context {
 public:
  static Context& get(int device);
  int device;
  cudaStream_t stream = nullptr;
  qk_workspace* ws = nullptr;
  double* host = nullptr;  // pinned, kHost doubles
  static constexpr int kHost = 4096;

  double* dres(int i = 0) const { return qkd_workspace_results(ws) + i; }
  // Copy n doubles from device memory to the pinned buffer and wait.
  const double* fetch(const double* dev, int n);
  void sync();
  void activate() const;
  // Stream-ordered device memory on this context's stream (the device's
  // default pool, which keeps freed blocks); release() is ordered after all
  // work already issued on the stream.
  void* alloc(size_t bytes);
  void release(void* p);

 private:
  explicit Context(int device);
};

// A device allocation of n elements of one dtype (zero-filled when asked),
// from the context's stream-ordered pool; only the context stream may use it.
class DevVec {
 public:
  DevVec() = default;
  DevVec(size_t n, qk_dtype t, int device, bool zero = true);
  ~DevVec();
  DevVec(const DevVec&) = delete;
  DevVec& operator=(const DevVec&) = delete;
  DevVec(DevVec&& o) noexcept { *this = std::move(o); }
  DevVec& operator=(DevVec&& o) noexcept;

  void* data() const { return p_; }
  size_t size() const { return n_; }
  qk_dtype dtype() const { return t_; }
  size_t bytes() const { return n_ * qk_dtype_size(t_); }
  int device() const { return dev_; }

 private:
  void* p_ = nullptr;
  size_t n_ = 0;
  qk_dtype t_ = QK_C128;
  int dev_ = 0;
};

// A device array of device pointers (for the multi-vector kernels).
class PtrArray {
 public:
  PtrArray(size_t cap, int device);
  ~PtrArray();
  void set(size_t i, const void* p, cudaStream_t s);
  const void* const* data() const { return reinterpret_cast<const void* const*>(d_); }
  const void* const* at(size_t i) const { return data() + i; }
  size_t capacity() const { return cap_; }

 private:
  void** d_ = nullptr;
  std::vector<const void*> h_;
  size_t cap_;
};

}  // namespace qkb
