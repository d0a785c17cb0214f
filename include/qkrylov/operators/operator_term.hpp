// Operator terms and the algebraic builder syntax
// (qkrylov's include/qkrylov/operators/operator_term.hpp:13-114):
//   1.0 * Sz(i) * Sz(j) + 0.5 * Sp(i) * Sm(j) - ...
// A term's factors act on a ket in list order (factors[0] first).
#pragma once

#include <initializer_list>
#include <string>
#include <utility>
#include <vector>

#include "qkrylov/core/types.hpp"

namespace qkrylov {
namespace QKRYLOV_PRECISION_NAMESPACE {

struct OperatorFactor {
  std::string op;
  int site = 0;
  OperatorFactor() = default;
  OperatorFactor(std::string op_, int site_) : op(std::move(op_)), site(site_) {}
};

struct OperatorTerm {
  Complex coeff;
  std::vector<OperatorFactor> factors;
  OperatorTerm() = default;
  OperatorTerm(Complex c, std::initializer_list<OperatorFactor> f) : coeff(c), factors(f) {}
};

struct LocalOp {
  std::string name;
  int site = 0;
  LocalOp() = default;
  LocalOp(std::string name_, int site_) : name(std::move(name_)), site(site_) {}
};

inline OperatorTerm operator*(Complex coeff, const LocalOp& op) {
  OperatorTerm t;
  t.coeff = coeff;
  t.factors.push_back({op.name, op.site});
  return t;
}
inline OperatorTerm operator*(Real coeff, const LocalOp& op) { return Complex(coeff, 0.0) * op; }
inline OperatorTerm operator*(const LocalOp& a, const LocalOp& b) {
  OperatorTerm t;
  t.coeff = 1.0;
  t.factors.push_back({a.name, a.site});
  t.factors.push_back({b.name, b.site});
  return t;
}
inline OperatorTerm operator*(OperatorTerm term, const LocalOp& op) {
  term.factors.push_back({op.name, op.site});
  return term;
}
inline OperatorTerm operator*(OperatorTerm a, const OperatorTerm& b) {
  a.coeff *= b.coeff;
  a.factors.insert(a.factors.end(), b.factors.begin(), b.factors.end());
  return a;
}

struct OpSumExpr {
  std::vector<OperatorTerm> terms;
  OpSumExpr(const OperatorTerm& t) : terms({t}) {}
  OpSumExpr(const std::vector<OperatorTerm>& ts) : terms(ts) {}
};

inline OpSumExpr operator+(const OperatorTerm& a, const OperatorTerm& b) { return OpSumExpr({a, b}); }
inline OpSumExpr operator+(OpSumExpr e, const OperatorTerm& t) { e.terms.push_back(t); return e; }
inline OpSumExpr operator+(const OperatorTerm& t, OpSumExpr e) { e.terms.insert(e.terms.begin(), t); return e; }
inline OpSumExpr operator+(OpSumExpr a, const OpSumExpr& b) {
  a.terms.insert(a.terms.end(), b.terms.begin(), b.terms.end());
  return a;
}
inline OpSumExpr operator-(const OperatorTerm& a, OperatorTerm b) { b.coeff = -b.coeff; return OpSumExpr({a, b}); }
inline OpSumExpr operator-(OpSumExpr e, OperatorTerm t) { t.coeff = -t.coeff; e.terms.push_back(t); return e; }

}  // namespace QKRYLOV_PRECISION_NAMESPACE
}  // namespace qkrylov
