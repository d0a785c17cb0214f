// TJSite: as Hubbard without Nupdn, creation forbidden on occupied sites (tj_site.cpp:47-113)
#pragma once

#include "qkrylov/sites/site.hpp"

namespace qkrylov {
namespace QKRYLOV_PRECISION_NAMESPACE {
QKRYLOV_DECLARE_SITE(TJSite, 3)
}  // namespace QKRYLOV_PRECISION_NAMESPACE
}  // namespace qkrylov
