// Finite-temperature Lanczos (qkrylov's include/qkrylov/solvers/ftlm.hpp:12-27),
// plus ftlm_sweep: the same estimator for many inverse temperatures from one
// set of random-vector tridiagonals (each entry equals a separate ftlm call).
#pragma once

#include <vector>

#include "qkrylov/hamiltonian/matrix_free_hamiltonian.hpp"

namespace qkrylov {
namespace QKRYLOV_PRECISION_NAMESPACE {

struct FTLMResult {
  Real beta;
  Real partition_function = 0.0;
  Real internal_energy = 0.0;
  Real specific_heat = 0.0;
};

template <typename ExecSpace>
FTLMResult ftlm(const MatrixFreeHamiltonian<ExecSpace>& H, Real beta, int n_random = 50, int n_steps = 100);

template <typename ExecSpace>
std::vector<FTLMResult> ftlm_sweep(const MatrixFreeHamiltonian<ExecSpace>& H, const std::vector<Real>& betas,
                                   int n_random = 50, int n_steps = 100);

}  // namespace QKRYLOV_PRECISION_NAMESPACE
}  // namespace qkrylov
