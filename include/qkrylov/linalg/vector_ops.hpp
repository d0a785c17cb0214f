// Device vector operations (qkrylov's include/qkrylov/linalg/vector_ops.hpp:14-137,
// same names and semantics: dot is conjugate-linear in x; reductions
// accumulate in FP64 on the GPU and are deterministic).
#pragma once

#include <cmath>

#include "qkrylov/core/kokkos_types.hpp"

namespace qkrylov {
namespace QKRYLOV_PRECISION_NAMESPACE {

namespace detail {
KComplex vec_dot(const KComplex* x, const KComplex* y, std::size_t n, int device);
void vec_scal(KComplex a, KComplex* x, std::size_t n, int device);
void vec_axpy(KComplex a, const KComplex* x, KComplex* y, std::size_t n, int device);
void vec_fill(KComplex v, KComplex* x, std::size_t n, int device);
void vec_copy(KComplex* dst, const KComplex* src, std::size_t n, int device);
void vec_h2d(const KComplex* h, KComplex* d, std::size_t n, int device);
void vec_d2h(const KComplex* d, KComplex* h, std::size_t n, int device);
}  // namespace detail

template <typename ViewType>
inline KComplex dot(const ViewType& x, const ViewType& y) {
  return detail::vec_dot(x.data(), y.data(), x.extent(0), x.device());
}
template <typename ViewType>
inline Real norm(const ViewType& x) { return std::sqrt(dot(x, x).real()); }
template <typename ViewType>
inline void scal(KComplex a, ViewType& x) { detail::vec_scal(a, x.data(), x.extent(0), x.device()); }
template <typename ViewType>
inline void scal(Real a, ViewType& x) { scal(KComplex(a, 0.0), x); }
template <typename ViewType>
inline void axpy(KComplex a, const ViewType& x, ViewType& y) {
  detail::vec_axpy(a, x.data(), y.data(), x.extent(0), x.device());
}
template <typename ViewType>
inline void normalize(ViewType& x) {
  const Real n = norm(x);
  if (n == 0.0) return;
  scal(KComplex(Real(1.0) / n, 0.0), x);
}
template <typename ViewType>
inline void zero_fill(ViewType& x) { detail::vec_fill(KComplex(0.0, 0.0), x.data(), x.extent(0), x.device()); }
template <typename ViewType1, typename ViewType2>
inline void deep_copy(ViewType1& dst, const ViewType2& src) {
  detail::vec_copy(dst.data(), src.data(), dst.extent(0), dst.device());
}
template <typename ViewType>
inline void copy_host_to_device(const HostVector& host, ViewType& device) {
  detail::vec_h2d(host.data(), device.data(), host.size(), device.device());
}
template <typename ViewType>
inline void copy_device_to_host(const ViewType& device, HostVector& host) {
  host.resize(device.extent(0));
  detail::vec_d2h(device.data(), host.data(), host.size(), device.device());
}

}  // namespace QKRYLOV_PRECISION_NAMESPACE
}  // namespace qkrylov
