// Device vector type of the qkrylov API.
//
// qkrylov's VectorView<ExecSpace> is a Kokkos::View of complex numbers in the
// execution space's memory (include/qkrylov/core/kokkos_types.hpp:12-27).
// Here it is a reference-counted HBM allocation of interleaved (re, im)
// values; copies share the allocation like View copies do.  The execution
// space is a single tag, qkrylov::CudaSpace; when the real Kokkos is not
// included, the names callers write (Kokkos::DefaultExecutionSpace,
// Kokkos::Cuda, Kokkos::complex, Kokkos::initialize/finalize) are provided
// as aliases of it so existing call sites compile unchanged.
#pragma once

#include <complex>
#include <memory>
#include <string>

#include "qkrylov/core/types.hpp"

namespace qkrylov {

struct CudaSpace {
  using execution_space = CudaSpace;
  using memory_space = CudaSpace;
};

namespace detail {
// Zero-filled device allocation on `device` (default: the selected device).
std::shared_ptr<void> device_alloc(std::size_t bytes, int device);
int default_device();
}  // namespace detail

namespace QKRYLOV_PRECISION_NAMESPACE {

using KComplex = std::complex<Real>;

template <typename ExecSpace>
class VectorView {
 public:
  using execution_space = ExecSpace;
  using memory_space = typename ExecSpace::memory_space;
  using value_type = KComplex;

  VectorView() = default;
  VectorView(const std::string& label, std::size_t n, int device = -1)
      : label_(label), n_(n), dev_(device < 0 ? qkrylov::detail::default_device() : device),
        buf_(qkrylov::detail::device_alloc(n * sizeof(KComplex), dev_)) {}

  std::size_t extent(int) const { return n_; }
  std::size_t size() const { return n_; }
  KComplex* data() const { return static_cast<KComplex*>(buf_.get()); }
  const std::string& label() const { return label_; }
  int device() const { return dev_; }

 private:
  std::string label_;
  std::size_t n_ = 0;
  int dev_ = 0;
  std::shared_ptr<void> buf_;
};

using ExecutionSpace = CudaSpace;
using MemorySpace = CudaSpace;
using Vector = VectorView<CudaSpace>;

}  // namespace QKRYLOV_PRECISION_NAMESPACE
}  // namespace qkrylov

#ifndef KOKKOS_VERSION
namespace Kokkos {
using Cuda = qkrylov::CudaSpace;
using DefaultExecutionSpace = qkrylov::CudaSpace;
using CudaSpace = qkrylov::CudaSpace;
template <class T> using complex = std::complex<T>;
inline void initialize() {}
inline void initialize(int&, char**) {}
inline void finalize() {}
inline bool is_initialized() { return true; }
}  // namespace Kokkos
#endif
