// Ground state by Lanczos with full reorthogonalisation
// (qkrylov's include/qkrylov/solvers/lanczos.hpp:11-25).
#pragma once

#include "qkrylov/hamiltonian/matrix_free_hamiltonian.hpp"
#include "qkrylov/linalg/vector_ops.hpp"

namespace qkrylov {
namespace QKRYLOV_PRECISION_NAMESPACE {

struct LanczosResult {
  Real energy = 0.0;
  int iterations = 0;
  bool converged = false;
  HostVector eigenvector;
};

template <typename ExecSpace>
LanczosResult lanczos_ground_state(const MatrixFreeHamiltonian<ExecSpace>& H, int maxiter = 200,
                                   Real tol = 1.0e-12);

}  // namespace QKRYLOV_PRECISION_NAMESPACE
}  // namespace qkrylov
