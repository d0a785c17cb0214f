// TJBasis: N t-J sites without double occupancy, optional fixed N_up / N_dn (tj_basis.cpp:56-96)
#pragma once

#include <stdexcept>

#include "qkrylov/basis/basis.hpp"

namespace qkrylov {
namespace QKRYLOV_PRECISION_NAMESPACE {
QKRYLOV_DECLARE_BASIS(TJBasis, 3)
}  // namespace QKRYLOV_PRECISION_NAMESPACE
}  // namespace qkrylov
