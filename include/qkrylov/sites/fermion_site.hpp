// FermionSite: N, Id, C, Cdag with Jordan-Wigner signs (fermion_site.cpp:19-84)
#pragma once

#include "qkrylov/sites/site.hpp"

namespace qkrylov {
namespace QKRYLOV_PRECISION_NAMESPACE {
QKRYLOV_DECLARE_SITE(FermionSite, 1)
}  // namespace QKRYLOV_PRECISION_NAMESPACE
}  // namespace qkrylov
