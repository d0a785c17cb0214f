// HubbardBasis: N Hubbard sites (2N bits), optional fixed N_up / N_dn (hubbard_basis.cpp:72-100)
#pragma once

#include <stdexcept>

#include "qkrylov/basis/basis.hpp"

namespace qkrylov {
namespace QKRYLOV_PRECISION_NAMESPACE {
QKRYLOV_DECLARE_BASIS(HubbardBasis, 2)
}  // namespace QKRYLOV_PRECISION_NAMESPACE
}  // namespace qkrylov
