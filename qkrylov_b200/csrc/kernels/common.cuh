// Shared device helpers: dtype traits, launch accounting, error mapping.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "dev_api.h"

namespace qkd {

// Element access for the four vector dtypes.  Complex values travel as a
// (re, im) pair of the accumulation type R.
template <int DT> struct VT;
template <> struct VT<QK_C128> {
  using E = double2; using R = double; static constexpr bool cplx = true;
  __device__ static void ld(const void* p, uint64_t i, R& re, R& im) {
    const double2 v = __ldg(reinterpret_cast<const double2*>(p) + i); re = v.x; im = v.y;
  }
  __device__ static void ld_plain(const void* p, uint64_t i, R& re, R& im) {
    const double2 v = reinterpret_cast<const double2*>(p)[i]; re = v.x; im = v.y;
  }
  __device__ static void st(void* p, uint64_t i, R re, R im) {
    reinterpret_cast<double2*>(p)[i] = make_double2(re, im);
  }
  __device__ static void st_cs(void* p, uint64_t i, R re, R im) {
    __stcs(reinterpret_cast<double2*>(p) + i, make_double2(re, im));
  }
};
template <> struct VT<QK_C64> {
  using E = float2; using R = float; static constexpr bool cplx = true;
  __device__ static void ld(const void* p, uint64_t i, R& re, R& im) {
    const float2 v = __ldg(reinterpret_cast<const float2*>(p) + i); re = v.x; im = v.y;
  }
  __device__ static void ld_plain(const void* p, uint64_t i, R& re, R& im) {
    const float2 v = reinterpret_cast<const float2*>(p)[i]; re = v.x; im = v.y;
  }
  __device__ static void st(void* p, uint64_t i, R re, R im) {
    reinterpret_cast<float2*>(p)[i] = make_float2(re, im);
  }
  __device__ static void st_cs(void* p, uint64_t i, R re, R im) {
    __stcs(reinterpret_cast<float2*>(p) + i, make_float2(re, im));
  }
};
template <> struct VT<QK_F64> {
  using E = double; using R = double; static constexpr bool cplx = false;
  __device__ static void ld(const void* p, uint64_t i, R& re, R& im) {
    re = __ldg(reinterpret_cast<const double*>(p) + i); im = 0;
  }
  __device__ static void ld_plain(const void* p, uint64_t i, R& re, R& im) {
    re = reinterpret_cast<const double*>(p)[i]; im = 0;
  }
  __device__ static void st(void* p, uint64_t i, R re, R) { reinterpret_cast<double*>(p)[i] = re; }
  __device__ static void st_cs(void* p, uint64_t i, R re, R) { __stcs(reinterpret_cast<double*>(p) + i, re); }
};
template <> struct VT<QK_F32> {
  using E = float; using R = float; static constexpr bool cplx = false;
  __device__ static void ld(const void* p, uint64_t i, R& re, R& im) {
    re = __ldg(reinterpret_cast<const float*>(p) + i); im = 0;
  }
  __device__ static void ld_plain(const void* p, uint64_t i, R& re, R& im) {
    re = reinterpret_cast<const float*>(p)[i]; im = 0;
  }
  __device__ static void st(void* p, uint64_t i, R re, R) { reinterpret_cast<float*>(p)[i] = re; }
  __device__ static void st_cs(void* p, uint64_t i, R re, R) { __stcs(reinterpret_cast<float*>(p) + i, re); }
};

void count_launch();
int sm_count(int device);

// Grid of a persistent (grid-stride) kernel: exactly the CTAs that are
// resident at once, so no CTA starts its whole share after another wave.
template <class K>
inline unsigned resident_grid(K kernel, int threads, size_t smem, unsigned cap) {
  int dev = 0, per_sm = 0;
  cudaGetDevice(&dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess || per_sm < 1) {
    (void)cudaGetLastError();
    per_sm = 1;
  }
  const unsigned g = unsigned(sm_count(dev)) * unsigned(per_sm);
  return g < cap ? g : cap;
}

}  // namespace qkd

#define QKD_LAUNCH_CHECK()                         \
  do {                                             \
    ::qkd::count_launch();                         \
    if (cudaPeekAtLastError() != cudaSuccess) {    \
      (void)cudaGetLastError();                    \
      return QKD_ECUDA;                            \
    }                                              \
  } while (0)

// Dispatch a runtime dtype to a template parameter DT.
#define QKD_DISPATCH(t, ...)                                        \
  switch (t) {                                                      \
    case QK_C128: { constexpr int DT = QK_C128; __VA_ARGS__; break; } \
    case QK_C64: { constexpr int DT = QK_C64; __VA_ARGS__; break; }   \
    case QK_F64: { constexpr int DT = QK_F64; __VA_ARGS__; break; }   \
    case QK_F32: { constexpr int DT = QK_F32; __VA_ARGS__; break; }   \
    default: return QKD_EINVAL;                                     \
  }
