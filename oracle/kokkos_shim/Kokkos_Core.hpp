// Minimal host-only stand-in for the parts of the Kokkos 4.x API that the
// qkrylov reference sources use, so that those sources can be compiled
// UNCHANGED into the CPU oracle (oracle/_ref) without network access to the
// real Kokkos.  Test infrastructure only: nothing in the product links it.
//
// Scope (exactly what qkrylov's src/ and include/ call):
//   View<T*, ...>          label ctor (zero-initialised), unmanaged (ptr, n) ctor,
//                          shallow copies, extent/size/data/operator()/operator[]
//   HostSpace, MemoryUnmanaged, OpenMP (= DefaultExecutionSpace)
//   deep_copy              view<-view and view<-scalar, with/without an instance
//   create_mirror_view     host views alias their source (as in Kokkos)
//   RangePolicy, parallel_for, parallel_reduce (sum)   -- OpenMP backed
//   complex<T>             the arithmetic Kokkos documents (component-wise
//                          product, 1-norm scaled division, hypot abs)
//   initialize / is_initialized / finalize / InitializationSettings
//
// Reductions sum per-thread partials in thread order, so results are
// deterministic for a fixed OMP_NUM_THREADS but not bit-identical to Kokkos.
#pragma once

#include <cmath>
#include <complex>
#include <cstddef>
#include <cstdint>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>
#include <omp.h>

#ifndef KOKKOS_ENABLE_OPENMP
#define KOKKOS_ENABLE_OPENMP 1
#endif
#define KOKKOS_LAMBDA [=]
#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FUNCTION

namespace Kokkos {

struct OpenMP;
struct HostSpace { using execution_space = OpenMP; using memory_space = HostSpace; };
struct MemoryUnmanaged {};
struct OpenMP { using execution_space = OpenMP; using memory_space = HostSpace; };
using DefaultExecutionSpace = OpenMP;
using DefaultHostExecutionSpace = OpenMP;

// ---------------------------------------------------------------- complex
template <class T>
class complex {
 public:
  using value_type = T;
  complex() : re_(0), im_(0) {}
  template <class U, class = std::enable_if_t<std::is_arithmetic_v<U>>>
  complex(U re) : re_(static_cast<T>(re)), im_(0) {}
  template <class U, class V>
  complex(U re, V im) : re_(static_cast<T>(re)), im_(static_cast<T>(im)) {}
  template <class U>
  complex(const complex<U>& o) : re_(static_cast<T>(o.real())), im_(static_cast<T>(o.imag())) {}
  template <class U>
  complex(const std::complex<U>& o) : re_(static_cast<T>(o.real())), im_(static_cast<T>(o.imag())) {}

  T real() const { return re_; }
  T imag() const { return im_; }
  void real(T v) { re_ = v; }
  void imag(T v) { im_ = v; }

  template <class U, class = std::enable_if_t<std::is_arithmetic_v<U>>>
  complex& operator=(U v) { re_ = static_cast<T>(v); im_ = 0; return *this; }

  complex& operator+=(const complex& o) { re_ += o.re_; im_ += o.im_; return *this; }
  complex& operator-=(const complex& o) { re_ -= o.re_; im_ -= o.im_; return *this; }
  complex& operator*=(const complex& o) {
    const T r = re_ * o.re_ - im_ * o.im_;
    const T i = re_ * o.im_ + im_ * o.re_;
    re_ = r; im_ = i; return *this;
  }
  complex& operator*=(T s) { re_ *= s; im_ *= s; return *this; }
  complex& operator/=(T s) { re_ /= s; im_ /= s; return *this; }
  complex& operator/=(const complex& y) { *this = *this / y; return *this; }

  friend complex operator+(complex a, const complex& b) { a += b; return a; }
  friend complex operator-(complex a, const complex& b) { a -= b; return a; }
  friend complex operator-(const complex& a) { return complex(-a.re_, -a.im_); }
  friend complex operator*(const complex& a, const complex& b) {
    return complex(a.re_ * b.re_ - a.im_ * b.im_, a.re_ * b.im_ + a.im_ * b.re_);
  }
  friend complex operator*(T s, const complex& a) { return complex(s * a.re_, s * a.im_); }
  friend complex operator*(const complex& a, T s) { return complex(a.re_ * s, a.im_ * s); }
  friend complex operator+(const complex& a, T s) { return complex(a.re_ + s, a.im_); }
  friend complex operator-(const complex& a, T s) { return complex(a.re_ - s, a.im_); }
  friend complex operator/(const complex& a, T s) { return complex(a.re_ / s, a.im_ / s); }
  // Division scaled by the 1-norm of the divisor, as Kokkos documents it.
  friend complex operator/(const complex& x, const complex& y) {
    const T s = std::fabs(y.re_) + std::fabs(y.im_);
    if (s == T(0)) return complex(x.re_ / s, x.im_ / s);
    const complex xs(x.re_ / s, x.im_ / s);
    const complex yc(y.re_ / s, -y.im_ / s);
    const T den = yc.re_ * yc.re_ + yc.im_ * yc.im_;
    complex r = xs * yc;
    r.re_ /= den; r.im_ /= den;
    return r;
  }
  friend bool operator==(const complex& a, const complex& b) { return a.re_ == b.re_ && a.im_ == b.im_; }

 private:
  T re_, im_;
};

template <class T> inline complex<T> conj(const complex<T>& a) { return complex<T>(a.real(), -a.imag()); }
template <class T> inline T abs(const complex<T>& a) { return std::hypot(a.real(), a.imag()); }
template <class T> inline T real(const complex<T>& a) { return a.real(); }
template <class T> inline T imag(const complex<T>& a) { return a.imag(); }

// ---------------------------------------------------------------- View
template <class DataType, class... Props>
class View;

template <class T, class... Props>
class View<T*, Props...> {
 public:
  using value_type = T;
  using non_const_value_type = std::remove_const_t<T>;
  using reference_type = T&;
  using execution_space = OpenMP;
  using memory_space = HostSpace;

  View() = default;
  View(const std::string& /*label*/, std::size_t n)
      : owner_(std::make_shared<std::vector<non_const_value_type>>(n)), n_(n) {
    ptr_ = owner_->data();
  }
  View(T* p, std::size_t n) : ptr_(p), n_(n) {}

  template <class U, class... P2,
            class = std::enable_if_t<std::is_convertible_v<U*, T*>>>
  View(const View<U*, P2...>& o) : owner_(o.owner_), ptr_(o.ptr_), n_(o.n_) {}

  std::size_t extent(int) const { return n_; }
  std::size_t size() const { return n_; }
  T* data() const { return ptr_; }
  T& operator()(std::size_t i) const { return ptr_[i]; }
  T& operator[](std::size_t i) const { return ptr_[i]; }

  template <class, class...> friend class View;

 private:
  std::shared_ptr<std::vector<non_const_value_type>> owner_;
  T* ptr_ = nullptr;
  std::size_t n_ = 0;
};

template <class V> struct is_view : std::false_type {};
template <class T, class... P> struct is_view<View<T, P...>> : std::true_type {};

template <class V>
inline V create_mirror_view(const V& v) { return v; }

template <class T1, class... P1, class T2, class... P2>
inline void deep_copy(const View<T1*, P1...>& dst, const View<T2*, P2...>& src) {
  const std::size_t n = dst.extent(0);
  T1* d = dst.data();
  const T2* s = src.data();
  if (static_cast<const void*>(d) == static_cast<const void*>(s)) return;
  #pragma omp parallel for schedule(static)
  for (std::int64_t i = 0; i < static_cast<std::int64_t>(n); ++i) d[i] = s[i];
}

template <class T1, class... P1, class S, class = std::enable_if_t<!is_view<S>::value>>
inline void deep_copy(const View<T1*, P1...>& dst, const S& value) {
  const std::size_t n = dst.extent(0);
  T1* d = dst.data();
  const T1 v(value);
  #pragma omp parallel for schedule(static)
  for (std::int64_t i = 0; i < static_cast<std::int64_t>(n); ++i) d[i] = v;
}

template <class D, class S>
inline void deep_copy(const OpenMP&, const D& dst, const S& src) { deep_copy(dst, src); }

// ---------------------------------------------------------------- dispatch
template <class ExecSpace = OpenMP>
struct RangePolicy {
  std::int64_t begin, end;
  template <class A, class B>
  RangePolicy(A b, B e) : begin(static_cast<std::int64_t>(b)), end(static_cast<std::int64_t>(e)) {}
};

template <class E, class F>
inline void parallel_for(const std::string&, const RangePolicy<E>& p, const F& f) {
  #pragma omp parallel for schedule(static)
  for (std::int64_t i = p.begin; i < p.end; ++i) f(i);
}

template <class N, class F, class = std::enable_if_t<std::is_integral_v<N>>>
inline void parallel_for(const std::string&, N n, const F& f) {
  #pragma omp parallel for schedule(static)
  for (std::int64_t i = 0; i < static_cast<std::int64_t>(n); ++i) f(static_cast<N>(i));
}

template <class E, class F, class R>
inline void parallel_reduce(const std::string&, const RangePolicy<E>& p, const F& f, R& result) {
  const int nt = omp_get_max_threads();
  std::vector<R> part(nt, R(0));
  #pragma omp parallel
  {
    const int t = omp_get_thread_num();
    R local(0);
    #pragma omp for schedule(static)
    for (std::int64_t i = p.begin; i < p.end; ++i) f(static_cast<int>(i), local);
    part[t] = local;
  }
  R total(0);
  for (int t = 0; t < nt; ++t) total += part[t];
  result = total;
}

// ---------------------------------------------------------------- lifecycle
struct InitializationSettings {
  int device_id = 0;
  InitializationSettings& set_device_id(int id) { device_id = id; return *this; }
};
namespace detail_shim { inline bool& initialized() { static bool v = false; return v; } }
inline void initialize() { detail_shim::initialized() = true; }
inline void initialize(const InitializationSettings&) { detail_shim::initialized() = true; }
inline bool is_initialized() { return detail_shim::initialized(); }
inline void finalize() { detail_shim::initialized() = false; }

}  // namespace Kokkos
