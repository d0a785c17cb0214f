// Local site physics (qkrylov's include/qkrylov/sites/site.hpp:13-24).
// Site::apply keeps the reference contract.  The operator compiler reads
// family() to turn whole OpSums into device bit-mask tables; Site
// subclasses written outside this library report -1 and are rejected by
// MatrixFreeHamiltonian with std::invalid_argument.
#pragma once

#include <string>

#include "qkrylov/operators/local_action.hpp"

namespace qkrylov {
namespace QKRYLOV_PRECISION_NAMESPACE {

class Site {
 public:
  virtual ~Site() = default;
  virtual LocalAction apply(const std::string& op, int site, StateID state) const = 0;
  // 0 spin-1/2, 1 spinless fermion, 2 Hubbard, 3 t-J, -1 unknown
  virtual int family() const { return -1; }
};

namespace detail {
LocalAction site_apply(int family, const std::string& op, int site, StateID state);
}

#define QKRYLOV_DECLARE_SITE(NAME, FAMILY)                                           \
  class NAME : public Site {                                                         \
   public:                                                                           \
    LocalAction apply(const std::string& op, int site, StateID state) const override { \
      return detail::site_apply(FAMILY, op, site, state);                            \
    }                                                                                \
    int family() const override { return FAMILY; }                                   \
  };

}  // namespace QKRYLOV_PRECISION_NAMESPACE
}  // namespace qkrylov
