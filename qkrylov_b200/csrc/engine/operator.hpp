// A compiled operator resident on one GPU: sector tables + compiled term
// groups uploaded once, applied any number of times by the H.x kernels.
// This is what the reference's MatrixFreeHamiltonian constructor builds
// (src/hamiltonian/matrix_free_hamiltonian.cpp:12-135), without the CSR.
#pragma once

#include <memory>
#include <vector>

#include "compile.hpp"
#include "runtime.hpp"
#include "sector.hpp"

namespace qkb {

class Operator {
 public:
  Operator(Family site_family, std::shared_ptr<const SectorTable> basis,
           const std::vector<TermIn>& terms, int device);
  ~Operator();
  Operator(const Operator&) = delete;
  Operator& operator=(const Operator&) = delete;

  uint64_t dim() const { return basis_->dim; }
  bool all_real() const { return op_.all_real; }
  int device() const { return device_; }
  const CompiledOp& compiled() const { return op_; }
  const SectorTable& basis() const { return *basis_; }
  std::shared_ptr<const SectorTable> basis_ptr() const { return basis_; }
  const qk_plan* plan() const { return plan_; }
  Context& ctx() const { return Context::get(device_); }

  // Device pointers, issued on the context stream (no host sync).
  void apply(qk_dtype t, const void* x, void* y) const;
  void apply_dot(qk_dtype t, const void* x, void* y, double* dot_dev) const;
  void diagonal(qk_dtype t, void* d) const;

 private:
  std::shared_ptr<const SectorTable> basis_;
  CompiledOp op_;
  qk_plan* plan_ = nullptr;
  int device_;
};

}  // namespace qkb
