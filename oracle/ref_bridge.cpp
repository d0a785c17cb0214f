// extern "C" bridge over the qkrylov reference's own C++ API in its fp64
// namespace, compiled together with the reference's unchanged src/*.cpp into
// oracle/_ref/liboracle_ref.so (see oracle/Makefile).  Test infrastructure:
// the parity tests and golden-fixture generator call it as the checker.
//
// Besides forwarding to the public API (bases, sites, MatrixFreeHamiltonian,
// lanczos_ground_state, davidson_lowest, continued_fraction_coeffs,
// evaluate_spectral_function, ftlm) it reads the private CSR arrays that the
// reference constructor builds (src/hamiltonian/matrix_free_hamiltonian.cpp:
// 45-94) so the matrix-element pattern, duplicates and zeros included, can be
// compared entry by entry.
#include <algorithm>
#include <complex>
#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include <Kokkos_Core.hpp>

#include "qkrylov/core/types.hpp"
#include "qkrylov/core/kokkos_types.hpp"
#include "qkrylov/core/device.hpp"
#include "qkrylov/symmetry/sector.hpp"
#include "qkrylov/operators/opsum.hpp"
#include "qkrylov/basis/spinhalf_basis.hpp"
#include "qkrylov/basis/fermion_basis.hpp"
#include "qkrylov/basis/hubbard_basis.hpp"
#include "qkrylov/basis/tj_basis.hpp"
#include "qkrylov/sites/spinhalf_site.hpp"
#include "qkrylov/sites/fermion_site.hpp"
#include "qkrylov/sites/hubbard_site.hpp"
#include "qkrylov/sites/tj_site.hpp"
#include "qkrylov/linalg/vector_ops.hpp"
#define private public
#include "qkrylov/hamiltonian/matrix_free_hamiltonian.hpp"
#undef private
#include "qkrylov/solvers/lanczos.hpp"
#include "qkrylov/solvers/davidson.hpp"
#include "qkrylov/solvers/dynamics.hpp"
#include "qkrylov/solvers/ftlm.hpp"

using namespace qkrylov;
using namespace qkrylov::fp64;
using HExec = Kokkos::DefaultExecutionSpace;
using Ham = MatrixFreeHamiltonian<HExec>;

namespace {
thread_local std::string g_err;
int fail(const std::exception& e) { g_err = e.what(); return -2; }

struct BasisBox { std::shared_ptr<Basis> b; };
struct HamBox { std::shared_ptr<Basis> b; std::shared_ptr<Site> s; std::unique_ptr<Ham> h; };

std::shared_ptr<Site> make_site(int kind) {
  switch (kind) {
    case 0: return std::make_shared<SpinHalfSite>();
    case 1: return std::make_shared<FermionSite>();
    case 2: return std::make_shared<HubbardSite>();
    case 3: return std::make_shared<TJSite>();
  }
  throw std::runtime_error("bad site kind");
}
}  // namespace

extern "C" {

const char* refb_last_error() { return g_err.c_str(); }

// kind: 0 spin-1/2, 1 spinless fermion, 2 Hubbard, 3 t-J.
// sec[10] = use_sz, sz2, use_nup, nup, use_ndn, ndn, use_n, n, use_nb, nb
void* refb_basis_create(int kind, int nsites, const int* sec) {
  try {
    Sector s;
    s.use_sz = sec[0]; s.sz2 = sec[1];
    s.use_nup = sec[2]; s.nup = sec[3];
    s.use_ndn = sec[4]; s.ndn = sec[5];
    s.use_n = sec[6]; s.n = sec[7];
    s.use_nb = sec[8]; s.nb = sec[9];
    auto box = new BasisBox;
    switch (kind) {
      case 0: box->b = std::make_shared<SpinHalfBasis>(nsites, s); break;
      case 1: box->b = std::make_shared<FermionBasis>(nsites, s); break;
      case 2: box->b = std::make_shared<HubbardBasis>(nsites, s); break;
      case 3: box->b = std::make_shared<TJBasis>(nsites, s); break;
      default: delete box; throw std::runtime_error("bad basis kind");
    }
    return box;
  } catch (const std::exception& e) { g_err = e.what(); return nullptr; }
}

void refb_basis_destroy(void* b) { delete static_cast<BasisBox*>(b); }
uint64_t refb_basis_dim(void* b) { return static_cast<BasisBox*>(b)->b->size(); }
void refb_basis_states(void* b, uint64_t* out) {
  auto& B = *static_cast<BasisBox*>(b)->b;
  for (Index i = 0; i < B.size(); ++i) out[i] = B.state(i);
}
int64_t refb_basis_index(void* b, uint64_t s) {
  auto& B = *static_cast<BasisBox*>(b)->b;
  if (!B.contains(s)) return -1;
  return static_cast<int64_t>(B.index(s));
}

int refb_site_apply(int kind, const char* op, int site, uint64_t state,
                    int* valid, uint64_t* new_state, double* me) {
  try {
    auto s = make_site(kind);
    auto a = s->apply(op, site, state);
    *valid = a.valid; *new_state = a.new_state;
    me[0] = a.matrix_element.real(); me[1] = a.matrix_element.imag();
    return 0;
  } catch (const std::exception& e) { return fail(e); }
}

// Terms: coef[2*t] + i coef[2*t+1]; factor counts nfac[t]; ops and sites
// flattened in term order.
void* refb_ham_create(void* basis, int site_kind, int nterms, const double* coef,
                      const int* nfac, const char* const* ops, const int* sites) {
  try {
    auto box = std::make_unique<HamBox>();
    box->b = static_cast<BasisBox*>(basis)->b;
    box->s = make_site(site_kind);
    OpSum os;
    int f = 0;
    for (int t = 0; t < nterms; ++t) {
      OperatorTerm term;
      term.coeff = Complex(coef[2 * t], coef[2 * t + 1]);
      for (int k = 0; k < nfac[t]; ++k, ++f) term.factors.push_back({std::string(ops[f]), sites[f]});
      os.add_term(term);
    }
    box->h = std::make_unique<Ham>(box->b, box->s, os, Device());
    return box.release();
  } catch (const std::exception& e) { g_err = e.what(); return nullptr; }
}

void refb_ham_destroy(void* h) { delete static_cast<HamBox*>(h); }
uint64_t refb_ham_dim(void* h) { return static_cast<HamBox*>(h)->h->dimension(); }
uint64_t refb_ham_nnz(void* h) { return static_cast<HamBox*>(h)->h->col_indices_.extent(0); }

void refb_ham_csr(void* h, int32_t* rowptr, int32_t* cols, double* vals) {
  auto& H = *static_cast<HamBox*>(h)->h;
  const std::size_t dim = H.dimension();
  const std::size_t nnz = H.col_indices_.extent(0);
  for (std::size_t i = 0; i <= dim; ++i) rowptr[i] = H.row_offsets_(i);
  for (std::size_t j = 0; j < nnz; ++j) {
    cols[j] = H.col_indices_(j);
    vals[2 * j] = H.values_(j).real();
    vals[2 * j + 1] = H.values_(j).imag();
  }
}

int refb_ham_apply(void* h, const double* x, double* y) {
  try {
    auto& H = *static_cast<HamBox*>(h)->h;
    H.apply(reinterpret_cast<const Complex*>(x), reinterpret_cast<Complex*>(y));
    return 0;
  } catch (const std::exception& e) { return fail(e); }
}

void refb_ham_diagonal(void* h, double* d) {
  auto v = static_cast<HamBox*>(h)->h->diagonal_host();
  std::memcpy(d, v.data(), v.size() * sizeof(Complex));
}

int refb_lanczos(void* h, int maxiter, double tol, double* energy, int* iters, int* conv,
                 double* evec) {
  try {
    auto r = lanczos_ground_state(*static_cast<HamBox*>(h)->h, maxiter, tol);
    *energy = r.energy; *iters = r.iterations; *conv = r.converged;
    if (evec && !r.eigenvector.empty())
      std::memcpy(evec, r.eigenvector.data(), r.eigenvector.size() * sizeof(Complex));
    return 0;
  } catch (const std::exception& e) { return fail(e); }
}

int refb_davidson(void* h, int n_eig, int max_subspace, double tol, double* evals,
                  double* evecs, int* n_out, int* iters, int* conv) {
  try {
    auto& H = *static_cast<HamBox*>(h)->h;
    auto r = davidson_lowest(H, n_eig, max_subspace, tol);
    *n_out = static_cast<int>(r.eigenvalues.size());
    *iters = r.iterations; *conv = r.converged;
    for (std::size_t k = 0; k < r.eigenvalues.size(); ++k) {
      evals[k] = r.eigenvalues[k];
      if (evecs)
        std::memcpy(evecs + 2 * k * H.dimension(), r.eigenvectors[k].data(),
                    r.eigenvectors[k].size() * sizeof(Complex));
    }
    return 0;
  } catch (const std::exception& e) { return fail(e); }
}

int refb_cf(void* h, const double* phi0, int n_iter, double* alphas, double* betas,
            double* norm_phi0, int* n_alpha, int* n_beta) {
  try {
    auto& H = *static_cast<HamBox*>(h)->h;
    HostVector p(reinterpret_cast<const Complex*>(phi0),
                 reinterpret_cast<const Complex*>(phi0) + H.dimension());
    auto r = continued_fraction_coeffs(H, p, n_iter);
    *norm_phi0 = r.norm_phi0;
    *n_alpha = static_cast<int>(r.alphas.size());
    *n_beta = static_cast<int>(r.betas.size());
    std::copy(r.alphas.begin(), r.alphas.end(), alphas);
    std::copy(r.betas.begin(), r.betas.end(), betas);
    return 0;
  } catch (const std::exception& e) { return fail(e); }
}

double refb_spectral(const double* alphas, const double* betas, std::size_t n, double norm_phi0,
                     double omega, double E0, double eta) {
  return evaluate_spectral_function(alphas, betas, n, norm_phi0, omega, E0, eta);
}

int refb_ftlm(void* h, double beta, int n_random, int n_steps, double* Z, double* U, double* Cv) {
  try {
    auto r = ftlm(*static_cast<HamBox*>(h)->h, beta, n_random, n_steps);
    *Z = r.partition_function; *U = r.internal_energy; *Cv = r.specific_heat;
    return 0;
  } catch (const std::exception& e) { return fail(e); }
}

}  // extern "C"
