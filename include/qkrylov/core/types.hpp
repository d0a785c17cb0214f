// Precision namespaces and basic types of the qkrylov API
// (same names and meaning as include/qkrylov/core/types.hpp of qkrylov:
// fp64 when QKRYLOV_DOUBLE_PRECISION is defined, fp32 otherwise).
#pragma once

#include <complex>
#include <cstddef>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#ifdef QKRYLOV_DOUBLE_PRECISION
#define QKRYLOV_PRECISION_NAMESPACE fp64
#else
#define QKRYLOV_PRECISION_NAMESPACE fp32
#endif

namespace qkrylov {
namespace QKRYLOV_PRECISION_NAMESPACE {

#ifdef QKRYLOV_DOUBLE_PRECISION
using Real = double;
#else
using Real = float;
#endif
using Complex = std::complex<Real>;
using StateID = uint64_t;
using Index = std::size_t;
using HostVector = std::vector<Complex>;

inline int popcount(uint64_t x) noexcept { return __builtin_popcountll(x); }

}  // namespace QKRYLOV_PRECISION_NAMESPACE
}  // namespace qkrylov
