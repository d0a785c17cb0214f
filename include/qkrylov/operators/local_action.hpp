// Result of one site operator on one basis state (qkrylov's
// include/qkrylov/operators/local_action.hpp:9-16).
#pragma once

#include "qkrylov/core/types.hpp"

namespace qkrylov {
namespace QKRYLOV_PRECISION_NAMESPACE {

struct LocalAction {
  bool valid = false;
  StateID new_state = 0;
  Complex matrix_element = 0.0;
};

}  // namespace QKRYLOV_PRECISION_NAMESPACE
}  // namespace qkrylov
