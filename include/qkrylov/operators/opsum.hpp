// Ordered sum of operator terms (qkrylov's include/qkrylov/operators/opsum.hpp:13-48).
#pragma once

#include <vector>

#include "qkrylov/operators/local_op.hpp"
#include "qkrylov/operators/operator_term.hpp"

namespace qkrylov {
namespace QKRYLOV_PRECISION_NAMESPACE {

class OpSum {
 public:
  void add_term(const OperatorTerm& term) { terms_.push_back(term); }
  OpSum& operator+=(const OperatorTerm& term) { add_term(term); return *this; }
  OpSum& operator+=(const OpSumExpr& expr) {
    for (const auto& t : expr.terms) add_term(t);
    return *this;
  }
  void clear() { terms_.clear(); }
  std::size_t size() const { return terms_.size(); }
  const OperatorTerm& operator[](std::size_t i) const { return terms_[i]; }
  const std::vector<OperatorTerm>& terms() const { return terms_; }

 private:
  std::vector<OperatorTerm> terms_;
};

}  // namespace QKRYLOV_PRECISION_NAMESPACE
}  // namespace qkrylov
