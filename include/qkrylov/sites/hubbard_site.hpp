// HubbardSite: Nup, Ndn, Nupdn, CUp, CdagUp, CDn, CdagDn; up at bit 2i, down at 2i+1 (hubbard_site.cpp:15-125)
#pragma once

#include "qkrylov/sites/site.hpp"

namespace qkrylov {
namespace QKRYLOV_PRECISION_NAMESPACE {
QKRYLOV_DECLARE_SITE(HubbardSite, 2)
}  // namespace QKRYLOV_PRECISION_NAMESPACE
}  // namespace qkrylov
