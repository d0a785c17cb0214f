#include "operator.hpp"

namespace qkb {

Operator::Operator(Family site_family, std::shared_ptr<const SectorTable> basis,
                   const std::vector<TermIn>& terms, int device)
    : basis_(std::move(basis)), device_(device) {
  op_ = compile_opsum(site_family, *basis_, terms);
  Context::get(device_);
  static_assert(sizeof(CTerm) == sizeof(qk_term_t), "term layout");
  static_assert(sizeof(CGroup) == sizeof(qk_group_t), "group layout");
  qk_plan_desc d{};
  d.nbits = basis_->nbits;
  d.L = basis_->L;
  d.dim = basis_->dim;
  d.A = basis_->A.data(); d.nA = basis_->A.size();
  d.B = basis_->B.data(); d.nB = basis_->B.size();
  d.llist = basis_->llist.data(); d.nllist = basis_->llist.size();
  d.key_off = basis_->key_off.data(); d.nkeys = uint32_t(basis_->key_off.size() - 1);
  d.terms = reinterpret_cast<const qk_term_t*>(op_.terms.data());
  d.nterms = uint32_t(op_.terms.size());
  d.groups = reinterpret_cast<const qk_group_t*>(op_.groups.data());
  d.ngroups = uint32_t(op_.groups.size());
  d.has_diag = op_.has_diag;
  d.all_real = op_.all_real;
  d.pair_sites = is_pair(basis_->family) ? 1 : 0;
  qkd_check(qkd_plan_create(&d, device_, &plan_), "operator upload");
}

Operator::~Operator() { qkd_plan_destroy(plan_); }

void Operator::apply(qk_dtype t, const void* x, void* y) const {
  qkd_check(qkd_apply(plan_, t, x, y, ctx().stream), "H.x");
}

void Operator::apply_dot(qk_dtype t, const void* x, void* y, double* dot_dev) const {
  Context& c = ctx();
  qkd_check(qkd_apply_dot(plan_, c.ws, t, x, y, dot_dev, c.stream), "H.x");
}

void Operator::diagonal(qk_dtype t, void* d) const {
  qkd_check(qkd_diagonal(plan_, t, d, ctx().stream), "diagonal");
}

}  // namespace qkb
