// Matrix-free Hamiltonian (qkrylov's
// include/qkrylov/hamiltonian/matrix_free_hamiltonian.hpp:24-77, same
// constructor and methods).
//
// The constructor compiles the OpSum once into device tables (bit masks,
// Jordan-Wigner parity masks and coefficients per term, grouped by target)
// and uploads the basis' sector tables; apply() then generates every
// matrix element on the fly on the GPU.  Nothing of size nnz is stored.
#pragma once

#include <memory>
#include <mutex>

#include "qkrylov/basis/basis.hpp"
#include "qkrylov/core/device.hpp"
#include "qkrylov/core/kokkos_types.hpp"
#include "qkrylov/operators/opsum.hpp"
#include "qkrylov/sites/site.hpp"

namespace qkb { class Operator; }

namespace qkrylov {
namespace QKRYLOV_PRECISION_NAMESPACE {

template <typename ExecSpace>
class MatrixFreeHamiltonian {
 public:
  MatrixFreeHamiltonian(std::shared_ptr<Basis> basis, std::shared_ptr<Site> site, const OpSum& ops,
                        Device device = Device());
  ~MatrixFreeHamiltonian();

  /// y = H x on device-resident vectors (no host copies).
  void apply(const VectorView<ExecSpace>& x, VectorView<ExecSpace>& y) const;
  /// y = H x on host arrays of dimension() complex numbers.
  void apply(const Complex* x, Complex* y) const;
  const VectorView<ExecSpace>& diagonal() const { return diagonal_; }
  HostVector diagonal_host() const;
  Index dimension() const { return dim_; }
  const Device& device() const { return device_; }

  /// The compiled device operator (for the extended solvers and C ABI).
  const qkb::Operator& op() const { return *op_; }
  std::shared_ptr<const qkb::Operator> op_ptr() const { return op_; }

 private:
  Device device_;
  Index dim_ = 0;
  std::shared_ptr<qkb::Operator> op_;
  VectorView<ExecSpace> diagonal_;
  std::shared_ptr<Basis> basis_;
  std::shared_ptr<Site> site_;
  OpSum ops_;
  mutable std::mutex host_mu_;
  mutable VectorView<ExecSpace> hx_, hy_;  // staging for the host-pointer apply
};

}  // namespace QKRYLOV_PRECISION_NAMESPACE
}  // namespace qkrylov
