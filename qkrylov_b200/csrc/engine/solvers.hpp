// GPU Krylov solvers with the reference's semantics (same start vectors,
// same recurrences, same stopping rules), vectors resident in HBM, H.x and
// all vector passes on the device, only the O(n) scalars on the host.
//
// Real = double works on complex128 vectors (qkrylov's fp64 namespace),
// Real = float on complex64 vectors (its fp32 namespace, the C ABI).
#pragma once

#include <complex>
#include <vector>

#include "operator.hpp"

namespace qkb {

template <class Real> constexpr qk_dtype complex_dtype() {
  return sizeof(Real) == 8 ? QK_C128 : QK_C64;
}

template <class Real>
struct LanczosOut {
  Real energy = 0;
  int iterations = 0;
  bool converged = false;
  std::vector<Real> alphas, betas;
  int reorth_second_rounds = 0;
};

template <class Real>
struct CFOut {
  std::vector<Real> alphas, betas;
  Real norm_phi0 = 0;
};

template <class Real>
struct FTLMOut {
  Real beta = 0, Z = 0, U = 0, Cv = 0;
};

template <class Real>
struct DavidsonOut {
  std::vector<Real> eigenvalues;
  std::vector<std::vector<std::complex<Real>>> eigenvectors;
  int iterations = 0;
  bool converged = false;
};

// Reference random streams (libstdc++ mt19937 + distributions; the
// imaginary part is drawn before the real part, the order GCC evaluates the
// two arguments of KComplex(dist(rng), dist(rng))).
template <class Real> void reference_uniform_start(uint64_t dim, std::vector<std::complex<Real>>& v);

// src/solvers/lanczos.cpp:101-202.  start == nullptr uses the reference's
// start vector.  Full reorthogonalisation against every stored Krylov
// vector is classical Gram-Schmidt with a second pass when the first one
// removes more than 3/4 of the norm (the reference runs sequential
// modified Gram-Schmidt; both project onto the same complement).
template <class Real>
LanczosOut<Real> lanczos(const Operator& H, int maxiter, Real tol,
                         const std::complex<Real>* start, std::vector<std::complex<Real>>* ritz);

// src/solvers/dynamics.cpp:12-59
template <class Real>
CFOut<Real> continued_fraction(const Operator& H, const std::complex<Real>* phi0, int n_iter);

// src/solvers/ftlm.cpp:122-170, for several inverse temperatures at once:
// the R tridiagonals do not depend on beta (the generator is re-seeded on
// every call of the reference), so one set serves every beta exactly.
template <class Real>
std::vector<FTLMOut<Real>> ftlm(const Operator& H, const std::vector<Real>& betas, int n_random,
                                int n_steps);

// src/solvers/davidson.cpp:86-227
template <class Real>
DavidsonOut<Real> davidson(const Operator& H, int n_eig, int max_subspace, Real tol);

// src/solvers/dynamics.cpp:61-89 (host, O(n))
template <class Real>
Real spectral_function(const Real* alphas, const Real* betas, size_t n, Real norm_phi0,
                       Real omega, Real E0, Real eta);

}  // namespace qkb
