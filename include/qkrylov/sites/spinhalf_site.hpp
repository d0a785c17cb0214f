// SpinHalfSite: Sz, Sp, Sm, Sx, Sy (spinhalf_site.cpp:18-121)
#pragma once

#include "qkrylov/sites/site.hpp"

namespace qkrylov {
namespace QKRYLOV_PRECISION_NAMESPACE {
QKRYLOV_DECLARE_SITE(SpinHalfSite, 0)
}  // namespace QKRYLOV_PRECISION_NAMESPACE
}  // namespace qkrylov
