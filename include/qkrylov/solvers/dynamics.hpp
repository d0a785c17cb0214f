// Continued-fraction dynamics (qkrylov's include/qkrylov/solvers/dynamics.hpp:13-38).
#pragma once

#include <vector>

#include "qkrylov/hamiltonian/matrix_free_hamiltonian.hpp"
#include "qkrylov/linalg/vector_ops.hpp"

namespace qkrylov {
namespace QKRYLOV_PRECISION_NAMESPACE {

struct DynamicsResult {
  std::vector<Real> alphas;
  std::vector<Real> betas;
  Real norm_phi0 = 0;
};

template <typename ExecSpace>
DynamicsResult continued_fraction_coeffs(const MatrixFreeHamiltonian<ExecSpace>& H, const HostVector& phi0,
                                         int n_iter = 100);

// S(omega) = -1/pi Im <phi0| (omega + E0 + i eta - H)^-1 |phi0>
Real evaluate_spectral_function(const Real* alphas, const Real* betas, size_t n, Real norm_phi0, Real omega,
                                Real E0, Real eta = 0.1);

}  // namespace QKRYLOV_PRECISION_NAMESPACE
}  // namespace qkrylov
