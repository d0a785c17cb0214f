// Public solver entry points for one precision namespace (compiled for fp64
// and fp32); each forwards to the GPU engine in engine/solvers.cpp.
#include <stdexcept>

#include "engine/operator.hpp"
#include "engine/solvers.hpp"
#include "qkrylov/solvers/davidson.hpp"
#include "qkrylov/solvers/dynamics.hpp"
#include "qkrylov/solvers/ftlm.hpp"
#include "qkrylov/solvers/lanczos.hpp"

namespace qkrylov {
namespace QKRYLOV_PRECISION_NAMESPACE {

template <typename ExecSpace>
LanczosResult lanczos_ground_state(const MatrixFreeHamiltonian<ExecSpace>& H, int maxiter, Real tol) {
  LanczosResult res;
  if (H.dimension() == 0) return res;
  std::vector<Complex> ritz;
  auto r = qkb::lanczos<Real>(H.op(), maxiter, tol, nullptr, &ritz);
  res.energy = r.energy;
  res.iterations = r.iterations;
  res.converged = r.converged;
  res.eigenvector.assign(ritz.begin(), ritz.end());
  return res;
}

template <typename ExecSpace>
DavidsonResult davidson_lowest(const MatrixFreeHamiltonian<ExecSpace>& H, int n_eig, int max_subspace, Real tol) {
  DavidsonResult res;
  if (H.dimension() == 0) return res;
  auto r = qkb::davidson<Real>(H.op(), n_eig, max_subspace, tol);
  res.eigenvalues = r.eigenvalues;
  for (auto& v : r.eigenvectors) res.eigenvectors.emplace_back(v.begin(), v.end());
  res.iterations = r.iterations;
  res.converged = r.converged;
  return res;
}

template <typename ExecSpace>
DynamicsResult continued_fraction_coeffs(const MatrixFreeHamiltonian<ExecSpace>& H, const HostVector& phi0,
                                         int n_iter) {
  DynamicsResult res;
  if (H.dimension() == 0) return res;
  if (phi0.size() != H.dimension())
    throw std::invalid_argument("phi0 vector size does not match Hamiltonian dimension");
  auto r = qkb::continued_fraction<Real>(H.op(), phi0.data(), n_iter);
  res.alphas = r.alphas;
  res.betas = r.betas;
  res.norm_phi0 = r.norm_phi0;
  return res;
}

Real evaluate_spectral_function(const Real* alphas, const Real* betas, size_t n, Real norm_phi0, Real omega,
                                Real E0, Real eta) {
  return qkb::spectral_function<Real>(alphas, betas, n, norm_phi0, omega, E0, eta);
}

template <typename ExecSpace>
std::vector<FTLMResult> ftlm_sweep(const MatrixFreeHamiltonian<ExecSpace>& H, const std::vector<Real>& betas,
                                   int n_random, int n_steps) {
  std::vector<FTLMResult> out;
  if (H.dimension() == 0) {
    for (Real b : betas) { FTLMResult f; f.beta = b; out.push_back(f); }
    return out;
  }
  for (const auto& r : qkb::ftlm<Real>(H.op(), betas, n_random, n_steps)) {
    FTLMResult f;
    f.beta = r.beta;
    f.partition_function = r.Z;
    f.internal_energy = r.U;
    f.specific_heat = r.Cv;
    out.push_back(f);
  }
  return out;
}

template <typename ExecSpace>
FTLMResult ftlm(const MatrixFreeHamiltonian<ExecSpace>& H, Real beta, int n_random, int n_steps) {
  return ftlm_sweep(H, std::vector<Real>{beta}, n_random, n_steps)[0];
}

template LanczosResult lanczos_ground_state<CudaSpace>(const MatrixFreeHamiltonian<CudaSpace>&, int, Real);
template DavidsonResult davidson_lowest<CudaSpace>(const MatrixFreeHamiltonian<CudaSpace>&, int, int, Real);
template DynamicsResult continued_fraction_coeffs<CudaSpace>(const MatrixFreeHamiltonian<CudaSpace>&,
                                                             const HostVector&, int);
template FTLMResult ftlm<CudaSpace>(const MatrixFreeHamiltonian<CudaSpace>&, Real, int, int);
template std::vector<FTLMResult> ftlm_sweep<CudaSpace>(const MatrixFreeHamiltonian<CudaSpace>&,
                                                       const std::vector<Real>&, int, int);

}  // namespace QKRYLOV_PRECISION_NAMESPACE
}  // namespace qkrylov
