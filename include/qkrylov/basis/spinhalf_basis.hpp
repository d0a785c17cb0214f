// SpinHalfBasis: spin-1/2 chain of N sites, optional fixed 2*Sz (spinhalf_basis.cpp:86-104)
#pragma once

#include <stdexcept>

#include "qkrylov/basis/basis.hpp"

namespace qkrylov {
namespace QKRYLOV_PRECISION_NAMESPACE {
QKRYLOV_DECLARE_BASIS(SpinHalfBasis, 0)
}  // namespace QKRYLOV_PRECISION_NAMESPACE
}  // namespace qkrylov
