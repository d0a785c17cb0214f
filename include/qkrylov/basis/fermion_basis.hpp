// FermionBasis: N spinless-fermion modes, optional fixed N (fermion_basis.cpp:72-89)
#pragma once

#include <stdexcept>

#include "qkrylov/basis/basis.hpp"

namespace qkrylov {
namespace QKRYLOV_PRECISION_NAMESPACE {
QKRYLOV_DECLARE_BASIS(FermionBasis, 1)
}  // namespace QKRYLOV_PRECISION_NAMESPACE
}  // namespace qkrylov
