// GPU Krylov solvers with the reference's semantics (same start vectors,
// same recurrences, same stopping rules), vectors resident in HBM, H.x and
// all vector passes on the device, only the O(n) scalars on the host.
//
// Real = double works on complex128 vectors (qkrylov's fp64 namespace),
// Real = float on complex64 vectors (its fp32 namespace, the C ABI).
#pragma once

#include <complex>
#include <string>
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

// Lanczos with full reorthogonalisation on device vectors of any dtype,
// scalars (alpha, beta, reorthogonalisation coefficients, tridiagonal) in
// FP64 on the host.  `start` (dtype t, dim elements) is copied, not
// modified.  Stops when |E_k - E_{k-1}| < tol_dE |E_k|, when the residual estimate
// beta_k |z_k| falls below tol_res * |E_k|, at breakdown, or at maxiter.  If
// ritz is given it receives the normalised Ritz vector in dtype tout.
struct TraceEntry { int iteration; double energy; double seconds; double resid_est; };
struct CoreOut {
  double energy = 0, resid_est = 0;
  int iterations = 0;
  bool converged = false;
  std::vector<double> alphas, betas;
  std::vector<TraceEntry> trace;
};
CoreOut lanczos_core(const Operator& H, qk_dtype t, const void* start, int maxiter, double tol_dE,
                     double tol_res, qk_dtype tout, void* ritz, double t0_seconds);

// Mixed precision.  The iterate psi, its Rayleigh quotient E and the
// residual r = H psi - E psi are FP64 (one FP64 apply per outer step); each
// correction comes from a Lanczos pass on FP32 vectors (FP64 alpha, beta,
// reorthogonalisation coefficients and tridiagonal) over the Krylov space
// of r kept orthogonal to psi, followed by the Rayleigh-Ritz step on
// span{psi, v_1..v_m}.  A pass stops when its Ritz residual estimate falls
// below max(0.3 tol, 1e-6 |r|/|E|); the loop ends when the explicit FP64
// residual |r| / |E| <= tol_res.  A pass that fails to halve the residual
// switches the passes to FP64.  Real operators use float32 / float64
// vectors, complex ones complex64 / complex128.
// low_phase = false: plain FP64 Lanczos from the start (restarted from the
// Ritz vector, at most 8 times) with the same explicit-residual stopping
// rule.  start: device vector of the FP32 type (mixed) or FP64 type
// (plain); null: a device random start from seed.  maxiter <= 511 steps
// per pass.
struct MixedOut {
  double energy = 0, residual = 0;
  int iters_low = 0, iters_high = 0, restarts = 0;  // FP32 steps; FP64 steps and applies; outer steps
  bool converged = false;
  double seconds_low = 0, seconds_high = 0;         // wall time in FP32 passes / FP64 work
  std::vector<TraceEntry> trace;                    // every step, seconds from the start
};
// partial: partial reorthogonalisation inside the passes (the default);
// false: every pass step orthogonalised against all the pass's vectors.
MixedOut lanczos_mixed(const Operator& H, const void* start, uint64_t seed, int maxiter, double tol_res,
                       void* psi_out_high, bool low_phase = true, bool partial = true);

// Batched FTLM on R (32, 64, 128) Rademacher vectors as one row-interleaved
// block of dtype t, M Lanczos steps without reorthogonalisation (the
// reference's recurrence), optionally captured as one CUDA graph; and the
// same vectors run one at a time (ftlm_loop, the first nvec columns).
struct FtlmBlockOut {
  int R = 0, M = 0, lanes_per_row = 0;
  bool graph = false;
  double seconds = 0, seconds_device = 0, e_min = 0;
  std::vector<double> alphas, betas, norm2;  // [r][M]; betas[r][k] = beta_k (len - 1 used)
  std::vector<int> len;                      // tridiagonal length per vector (breakdown)
  std::vector<double> logZ, U, Cv;           // per temperature
};
FtlmBlockOut ftlm_block(const Operator& H, qk_dtype t, int R, int M, uint64_t seed, const std::vector<double>& temps,
                        bool use_graph);
FtlmBlockOut ftlm_loop(const Operator& H, qk_dtype t, int R, int M, uint64_t seed, const std::vector<double>& temps,
                       int nvec);
// Block continued fraction (dynamics.cpp:12-59 of qkrylov for R start
// vectors at once): the three-term recurrence without reorthogonalisation
// from each column of `start` (device, row-interleaved dim x R of dtype t,
// unnormalised; copied), M steps, a column stopping at beta < 1e-15.
// alphas / betas [r][M] of the normalised recurrences, len, norm2.
FtlmBlockOut cf_block(const Operator& H, qk_dtype t, int R, int M, const void* start, bool use_graph);

// Block Davidson (k eigenpairs, a block of corrections per iteration,
// diagonal preconditioner, bounded subspace, seeded random block start; the
// form used for Hubbard 4x4 with k = 4, block 8, subspace 64) for real
// operators on float32 / float64 vectors, storing only the basis.
struct DavidsonBlockOut {
  std::vector<double> eigenvalues, residuals;
  int iterations = 0, applies = 0, restarts = 0;
  bool converged = false;
  double seconds = 0;
  std::vector<TraceEntry> trace;  // (iteration, lowest Ritz value, seconds, worst residual of the k)
};
DavidsonBlockOut davidson_block(const Operator& H, qk_dtype t, int n_eig, int block, int max_subspace, double tol,
                                uint64_t seed, int maxiter, double* evecs_out);

// Batched coupling sweep (no counterpart in the reference): ground states
// of H0 + g H1 for up to 128 couplings g as one row-interleaved FP64 block,
// each column its own Lanczos recurrence kept semi-orthogonal by partial
// reorthogonalisation, restarted from its Ritz vector (passes of at most
// pass_len steps) until every explicit residual |H psi - E psi| / |E| <= tol.
struct SweepOut {
  std::vector<double> energies, residuals;
  std::vector<int> converged;
  int R = 0, steps = 0, passes = 0, applies = 0, reorths = 0, lanes_per_row = 0;
  double seconds = 0, seconds_inference = 0;
};
class WarmStartNet;
// net: NULL for seeded random starts, or a warm-start network on the same
// basis whose coupling input is g (its start vector at each coupling)
SweepOut lanczos_sweep(const Operator& H0, const Operator& H1, const std::vector<double>& couplings, int pass_len,
                       int max_passes, double tol, uint64_t seed, WarmStartNet* net);

// src/solvers/dynamics.cpp:12-59
template <class Real>
CFOut<Real> continued_fraction(const Operator& H, const std::complex<Real>* phi0, int n_iter);
// continued_fraction on complex128 vectors with a checkpoint: resumed from
// resume_dir (when not empty; phi0 is then ignored) and/or saved to
// save_dir (when not empty) as .npy files; n_iter counts all steps.
CFOut<double> continued_fraction_checkpointed(const Operator& H, const std::complex<double>* phi0,
                                              const std::string& resume_dir, int n_iter,
                                              const std::string& save_dir);

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
