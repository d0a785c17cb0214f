// qkrylov's C ABI (include/qkrylov/c_api.h, implementation src/c_api.cpp)
// on the B200 engine.  Argument checks, status codes, NULL/0/-1 sentinels
// and float conversions follow the reference entry by entry; solvers run in
// single precision (complex64 vectors, float scalars) as the reference C
// ABI does, with all vector work on the GPU.
#include <cstring>
#include <exception>

#include "api/handles.hpp"
#include "engine/solvers.hpp"
#include "qkrylov_c_api.h"

namespace qkapi {
namespace {
thread_local std::string g_last_error;
}
void set_error(const std::string& msg) { g_last_error = msg; }
const char* last_error() { return g_last_error.c_str(); }
}  // namespace qkapi

namespace {

template <class F>
int guarded(F&& f) {
  try {
    return f();
  } catch (const std::exception& e) {
    qkapi::set_error(e.what());
    return QKRYLOV_ERROR_EXCEPTION;
  } catch (...) {
    qkapi::set_error("unknown exception");
    return QKRYLOV_ERROR_EXCEPTION;
  }
}

qkrylov_basis_h make_basis(qkb::Family f, int n, qkrylov_sector_h sector) {
  try {
    auto h = std::make_unique<qkrylov_basis_t>();
    h->family = f;
    h->nsites = n;
    h->table = std::make_shared<const qkb::SectorTable>(f, n, sector ? sector->s : qkb::SectorSpec{});
    return h.release();
  } catch (const std::exception& e) {
    qkapi::set_error(e.what());
    return nullptr;
  }
}

qkrylov_site_h make_site(qkb::Family f) {
  try {
    return new qkrylov_site_t{f};
  } catch (...) {
    return nullptr;
  }
}

int add_term(qkrylov_opsum_h opsum, std::complex<double> c, int n, const char* const* ops, const int* sites) {
  qkb::TermIn t;
  t.coeff = c;
  for (int i = 0; i < n; ++i) {
    if (!ops[i]) return QKRYLOV_ERROR_INVALID_ARG;
    t.factors.push_back({std::string(ops[i]), sites[i]});
  }
  opsum->terms.push_back(std::move(t));
  return QKRYLOV_SUCCESS;
}

}  // namespace

extern "C" {

/* Sector (c_api.cpp:56-158) */
qkrylov_sector_h qkrylov_sector_create(void) {
  try { return new qkrylov_sector_t{}; } catch (...) { return nullptr; }
}
void qkrylov_sector_destroy(qkrylov_sector_h sector) { delete sector; }
int qkrylov_sector_set_sz(qkrylov_sector_h sector, int sz2) {
  if (!sector) return QKRYLOV_ERROR_INVALID_ARG;
  sector->s.use_sz = true; sector->s.sz2 = sz2;
  return QKRYLOV_SUCCESS;
}
int qkrylov_sector_set_hubbard_particles(qkrylov_sector_h sector, int nup, int ndn) {
  if (!sector) return QKRYLOV_ERROR_INVALID_ARG;
  sector->s.use_nup = true; sector->s.use_ndn = true; sector->s.nup = nup; sector->s.ndn = ndn;
  return QKRYLOV_SUCCESS;
}
int qkrylov_sector_set_n(qkrylov_sector_h sector, int n) {
  if (!sector) return QKRYLOV_ERROR_INVALID_ARG;
  sector->s.use_n = true; sector->s.n = n;
  return QKRYLOV_SUCCESS;
}
int qkrylov_sector_set_nb(qkrylov_sector_h sector, int nb) {
  if (!sector) return QKRYLOV_ERROR_INVALID_ARG;
  sector->s.use_nb = true; sector->s.nb = nb;
  return QKRYLOV_SUCCESS;
}
int qkrylov_sector_get_sz(qkrylov_sector_h sector, int* sz2_out, int* active_out) {
  if (!sector) return QKRYLOV_ERROR_INVALID_ARG;
  if (active_out) *active_out = sector->s.use_sz ? 1 : 0;
  if (sz2_out) *sz2_out = sector->s.sz2;
  return QKRYLOV_SUCCESS;
}
int qkrylov_sector_get_hubbard_particles(qkrylov_sector_h sector, int* nup_out, int* ndn_out, int* active_out) {
  if (!sector) return QKRYLOV_ERROR_INVALID_ARG;
  if (active_out) *active_out = (sector->s.use_nup && sector->s.use_ndn) ? 1 : 0;
  if (nup_out) *nup_out = sector->s.nup;
  if (ndn_out) *ndn_out = sector->s.ndn;
  return QKRYLOV_SUCCESS;
}
int qkrylov_sector_get_n(qkrylov_sector_h sector, int* n_out, int* active_out) {
  if (!sector) return QKRYLOV_ERROR_INVALID_ARG;
  if (active_out) *active_out = sector->s.use_n ? 1 : 0;
  if (n_out) *n_out = sector->s.n;
  return QKRYLOV_SUCCESS;
}
int qkrylov_sector_get_nb(qkrylov_sector_h sector, int* nb_out, int* active_out) {
  if (!sector) return QKRYLOV_ERROR_INVALID_ARG;
  if (active_out) *active_out = sector->s.use_nb ? 1 : 0;
  if (nb_out) *nb_out = sector->s.nb;
  return QKRYLOV_SUCCESS;
}

/* Basis (c_api.cpp:161-257) */
qkrylov_basis_h qkrylov_spinhalf_basis_create(int n, qkrylov_sector_h s) { return make_basis(qkb::Family::Spin, n, s); }
qkrylov_basis_h qkrylov_fermion_basis_create(int n, qkrylov_sector_h s) { return make_basis(qkb::Family::Fermion, n, s); }
qkrylov_basis_h qkrylov_hubbard_basis_create(int n, qkrylov_sector_h s) { return make_basis(qkb::Family::Hubbard, n, s); }
qkrylov_basis_h qkrylov_tj_basis_create(int n, qkrylov_sector_h s) { return make_basis(qkb::Family::TJ, n, s); }
void qkrylov_basis_destroy(qkrylov_basis_h basis) { delete basis; }
uint64_t qkrylov_basis_dimension(qkrylov_basis_h basis) {
  if (!basis || !basis->table) return 0;
  return basis->table->dim;
}
int qkrylov_basis_nsites(qkrylov_basis_h basis) {
  if (!basis || !basis->table) return 0;
  return basis->nsites;
}
uint64_t qkrylov_basis_state(qkrylov_basis_h basis, uint64_t index) {
  if (!basis || !basis->table) return 0;
  try { return basis->table->state(index); } catch (...) { return 0; }
}
int64_t qkrylov_basis_index(qkrylov_basis_h basis, uint64_t s) {
  if (!basis || !basis->table) return -1;
  return basis->table->index(s);
}
int qkrylov_basis_contains(qkrylov_basis_h basis, uint64_t s) {
  if (!basis || !basis->table) return 0;
  return basis->table->contains(s) ? 1 : 0;
}

/* Site (c_api.cpp:260-302) */
qkrylov_site_h qkrylov_spinhalf_site_create(void) { return make_site(qkb::Family::Spin); }
qkrylov_site_h qkrylov_fermion_site_create(void) { return make_site(qkb::Family::Fermion); }
qkrylov_site_h qkrylov_hubbard_site_create(void) { return make_site(qkb::Family::Hubbard); }
qkrylov_site_h qkrylov_tj_site_create(void) { return make_site(qkb::Family::TJ); }
void qkrylov_site_destroy(qkrylov_site_h site) { delete site; }

/* OpSum (c_api.cpp:305-373); float coefficients are stored exactly. */
qkrylov_opsum_h qkrylov_opsum_create(void) {
  try { return new qkrylov_opsum_t{}; } catch (...) { return nullptr; }
}
void qkrylov_opsum_destroy(qkrylov_opsum_h opsum) { delete opsum; }
int qkrylov_opsum_clear(qkrylov_opsum_h opsum) {
  if (!opsum) return QKRYLOV_ERROR_INVALID_ARG;
  opsum->terms.clear();
  return QKRYLOV_SUCCESS;
}
int qkrylov_opsum_add_term_1body(qkrylov_opsum_h opsum, float cr, float ci, const char* op1, int site1) {
  if (!opsum || !op1) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] { const char* o[1] = {op1}; const int s[1] = {site1}; return add_term(opsum, {cr, ci}, 1, o, s); });
}
int qkrylov_opsum_add_term_2body(qkrylov_opsum_h opsum, float cr, float ci, const char* op1, int site1,
                                 const char* op2, int site2) {
  if (!opsum || !op1 || !op2) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    const char* o[2] = {op1, op2};
    const int s[2] = {site1, site2};
    return add_term(opsum, {cr, ci}, 2, o, s);
  });
}
int qkrylov_opsum_add_term_nbody(qkrylov_opsum_h opsum, float cr, float ci, int n, const char** ops,
                                 const int* sites) {
  if (!opsum || !ops || !sites || n <= 0) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] { return add_term(opsum, {cr, ci}, n, ops, sites); });
}

/* Hamiltonian (c_api.cpp:376-471) */
qkrylov_hamiltonian_h qkrylov_hamiltonian_create(qkrylov_basis_h basis, qkrylov_site_h site,
                                                qkrylov_opsum_h opsum) {
  if (!basis || !basis->table || !site || !opsum) return nullptr;
  try {
    auto h = std::make_unique<qkrylov_hamiltonian_t>();
    h->op = std::make_shared<qkb::Operator>(site->family, basis->table, opsum->terms, 0);
    h->precision = 32;
    return h.release();
  } catch (const std::exception& e) {
    qkapi::set_error(e.what());
    return nullptr;
  }
}
void qkrylov_hamiltonian_destroy(qkrylov_hamiltonian_h h) { delete h; }
uint64_t qkrylov_hamiltonian_dimension(qkrylov_hamiltonian_h h) {
  if (!h || !h->op) return 0;
  return h->op->dim();
}

namespace {
// Host complex-float apply through the handle's device staging buffers.
int apply_c64(qkrylov_hamiltonian_h h, const std::complex<float>* x, std::complex<float>* y) {
  const uint64_t dim = h->op->dim();
  if (dim == 0) return QKRYLOV_SUCCESS;
  auto& c = h->op->ctx();
  std::lock_guard<std::mutex> lk(h->mu);
  h->stage(QK_C64);
  qkb::cuda_check(cudaMemcpyAsync(h->sx.data(), x, dim * 8, cudaMemcpyHostToDevice, c.stream), "H2D");
  h->op->apply(QK_C64, h->sx.data(), h->sy.data());
  qkb::cuda_check(cudaMemcpyAsync(y, h->sy.data(), dim * 8, cudaMemcpyDeviceToHost, c.stream), "D2H");
  c.sync();
  return QKRYLOV_SUCCESS;
}
}  // namespace

int qkrylov_hamiltonian_apply(qkrylov_hamiltonian_h h, const float* x_real, const float* x_imag, float* y_real,
                              float* y_imag) {
  if (!h || !h->op || !x_real || !y_real) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    const uint64_t dim = h->op->dim();
    std::vector<std::complex<float>> x(dim), y(dim);
    for (uint64_t i = 0; i < dim; ++i) x[i] = {x_real[i], x_imag ? x_imag[i] : 0.0f};
    int rc = apply_c64(h, x.data(), y.data());
    if (rc) return rc;
    for (uint64_t i = 0; i < dim; ++i) {
      y_real[i] = y[i].real();
      if (y_imag) y_imag[i] = y[i].imag();
    }
    return QKRYLOV_SUCCESS;
  });
}

int qkrylov_hamiltonian_apply_complex(qkrylov_hamiltonian_h h, const float* x_complex, float* y_complex) {
  if (!h || !h->op || !x_complex || !y_complex) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    return apply_c64(h, reinterpret_cast<const std::complex<float>*>(x_complex),
                     reinterpret_cast<std::complex<float>*>(y_complex));
  });
}

int qkrylov_hamiltonian_diagonal(qkrylov_hamiltonian_h h, float* diag_out) {
  if (!h || !h->op || !diag_out) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    const uint64_t dim = h->op->dim();
    if (dim == 0) return QKRYLOV_SUCCESS;
    qkb::DevVec d(dim, QK_C64, h->op->device(), false);
    h->op->diagonal(QK_C64, d.data());
    std::vector<std::complex<float>> hd(dim);
    auto& c = h->op->ctx();
    qkb::cuda_check(cudaMemcpyAsync(hd.data(), d.data(), dim * 8, cudaMemcpyDeviceToHost, c.stream), "D2H");
    c.sync();
    for (uint64_t i = 0; i < dim; ++i) diag_out[i] = hd[i].real();
    return QKRYLOV_SUCCESS;
  });
}

/* Solvers (c_api.cpp:474-624), single precision like the reference ABI. */
int qkrylov_lanczos_ground_state(qkrylov_hamiltonian_h h, int maxiter, float tol, qkrylov_lanczos_result_c_t* result) {
  return qkrylov_lanczos_ground_state_complex(h, maxiter, tol, result, nullptr);
}

int qkrylov_lanczos_ground_state_complex(qkrylov_hamiltonian_h h, int maxiter, float tol,
                                         qkrylov_lanczos_result_c_t* result, float* eigenvector_complex) {
  if (!h || !h->op || !result) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    std::vector<std::complex<float>> ritz;
    auto r = qkb::lanczos<float>(*h->op, maxiter, tol, nullptr, eigenvector_complex ? &ritz : nullptr);
    result->energy = r.energy;
    result->iterations = r.iterations;
    result->converged = r.converged ? 1 : 0;
    if (eigenvector_complex && !ritz.empty()) std::memcpy(eigenvector_complex, ritz.data(), ritz.size() * 8);
    return QKRYLOV_SUCCESS;
  });
}

int qkrylov_davidson_lowest_complex(qkrylov_hamiltonian_h h, int n_eig, int max_subspace, float tol,
                                    float* eigenvalues_out, float* eigenvectors_complex_out,
                                    qkrylov_davidson_result_c_t* result_info) {
  if (!h || !h->op || !eigenvalues_out || n_eig <= 0) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    auto r = qkb::davidson<float>(*h->op, n_eig, max_subspace, tol);
    const size_t k = std::min(size_t(n_eig), r.eigenvalues.size());
    for (size_t i = 0; i < k; ++i) eigenvalues_out[i] = r.eigenvalues[i];
    if (result_info) { result_info->iterations = r.iterations; result_info->converged = r.converged ? 1 : 0; }
    if (eigenvectors_complex_out) {
      const uint64_t dim = h->op->dim();
      for (size_t q = 0; q < k; ++q)
        std::memcpy(eigenvectors_complex_out + 2 * q * dim, r.eigenvectors[q].data(),
                    std::min<size_t>(dim, r.eigenvectors[q].size()) * 8);
    }
    return QKRYLOV_SUCCESS;
  });
}

int qkrylov_continued_fraction_coeffs_complex(qkrylov_hamiltonian_h h, const float* phi0_complex, int n_iter,
                                              float* alphas_out, float* betas_out, float* norm_phi0_out,
                                              int* num_coeffs_out) {
  if (!h || !h->op || !phi0_complex || !alphas_out || !betas_out || !norm_phi0_out || n_iter <= 0)
    return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    auto r = qkb::continued_fraction<float>(*h->op, reinterpret_cast<const std::complex<float>*>(phi0_complex), n_iter);
    *norm_phi0_out = r.norm_phi0;
    for (size_t i = 0; i < r.alphas.size() && i < size_t(n_iter); ++i) alphas_out[i] = r.alphas[i];
    for (size_t i = 0; i < r.betas.size() && i < size_t(n_iter); ++i) betas_out[i] = r.betas[i];
    if (num_coeffs_out) *num_coeffs_out = int(r.alphas.size());
    return QKRYLOV_SUCCESS;
  });
}

float qkrylov_evaluate_spectral_function(const float* alphas, const float* betas, size_t n, float norm_phi0,
                                         float omega, float E0, float eta) {
  if (!alphas || !betas || n == 0) return 0.0f;
  try {
    std::vector<float> b(n, 0.0f);
    for (size_t i = 0; i + 1 < n; ++i) b[i] = betas[i];
    return qkb::spectral_function<float>(alphas, b.data(), n, norm_phi0, omega, E0, eta);
  } catch (...) {
    return 0.0f;
  }
}

int qkrylov_ftlm(qkrylov_hamiltonian_h h, float beta, int n_random, int n_steps, qkrylov_ftlm_result_c_t* result) {
  if (!h || !h->op || !result) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    auto r = qkb::ftlm<float>(*h->op, std::vector<float>{beta}, n_random, n_steps)[0];
    result->beta = r.beta;
    result->partition_function = r.Z;
    result->internal_energy = r.U;
    result->specific_heat = r.Cv;
    return QKRYLOV_SUCCESS;
  });
}

}  // extern "C"
