// Lowest eigenpairs by Davidson with the diagonal preconditioner
// (qkrylov's include/qkrylov/solvers/davidson.hpp:13-27).
#pragma once

#include <vector>

#include "qkrylov/hamiltonian/matrix_free_hamiltonian.hpp"
#include "qkrylov/linalg/vector_ops.hpp"

namespace qkrylov {
namespace QKRYLOV_PRECISION_NAMESPACE {

struct DavidsonResult {
  std::vector<Real> eigenvalues;
  std::vector<HostVector> eigenvectors;
  int iterations = 0;
  bool converged = false;
};

template <typename ExecSpace>
DavidsonResult davidson_lowest(const MatrixFreeHamiltonian<ExecSpace>& H, int n_eig = 1,
                               int max_subspace = 20, Real tol = 1.0e-8);

}  // namespace QKRYLOV_PRECISION_NAMESPACE
}  // namespace qkrylov
