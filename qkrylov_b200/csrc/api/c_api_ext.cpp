// Extended C ABI (include/qkrylov_b200.h): double precision, device
// pointers, multi-temperature FTLM, compiler inspection, diagnostics.
#include <chrono>
#include <cstring>
#include <exception>
#include <memory>

#include "api/handles.hpp"
#include "engine/solvers.hpp"
#include "engine/warmstart.hpp"
#include "qkrylov_b200.h"

namespace qkapi {
const char* last_error();
}

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
bool valid_dtype(int t) { return t >= QKRYLOV_DTYPE_C128 && t <= QKRYLOV_DTYPE_F32; }
}  // namespace

extern "C" {

const char* qkrylov_b200_last_error(void) { return qkapi::last_error(); }
uint64_t qkrylov_b200_launch_count(void) { return qkd_launch_count(); }
int qkrylov_b200_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) { (void)cudaGetLastError(); return 0; }
  return n;
}

int qkrylov_b200_set_kernel_policy(int policy) {
  // 0 auto (the specialised kernels where the operator has their tables),
  // 1 the generic term-walk kernel only, 2 auto without per-die work queues,
  // 3 auto without the spin-product path of Hubbard-type operators
  if (policy < 0 || policy > 3) return QKRYLOV_ERROR_INVALID_ARG;
  qkd_set_kernel_policy(policy);
  return QKRYLOV_SUCCESS;
}

int qkrylov_b200_die_count(int* sms_die0, int* sms_die1) { return qkd_die_count(sms_die0, sms_die1); }

int qkrylov_hamiltonian_kernel(qkrylov_hamiltonian_h h) { return (h && h->op) ? qkd_plan_kernel(h->op->plan()) : 0; }

int qkrylov_b200_sector_set_species(qkrylov_sector_h sector, int use_nup, int use_ndn) {
  if (!sector) return QKRYLOV_ERROR_INVALID_ARG;
  sector->s.use_nup = use_nup != 0;
  sector->s.use_ndn = use_ndn != 0;
  return QKRYLOV_SUCCESS;
}

int qkrylov_b200_site_apply(qkrylov_site_h site, const char* op, int site_index, uint64_t state, int* valid,
                            uint64_t* new_state, double* me) {
  if (!site || !op || !valid || !new_state || !me) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    const auto a = qkb::apply_factor(site->family, op, site_index, state);
    *valid = a.valid;
    *new_state = a.new_state;
    me[0] = a.me.real();
    me[1] = a.me.imag();
    return QKRYLOV_SUCCESS;
  });
}

int qkrylov_basis_states(qkrylov_basis_h basis, uint64_t first, uint64_t count, uint64_t* out) {
  if (!basis || !basis->table || (count && !out)) return QKRYLOV_ERROR_INVALID_ARG;
  if (first > basis->table->dim || count > basis->table->dim - first) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    for (uint64_t i = 0; i < count; ++i) out[i] = basis->table->state(first + i);
    return QKRYLOV_SUCCESS;
  });
}

int qkrylov_basis_index_many(qkrylov_basis_h basis, const uint64_t* states, uint64_t n, int64_t* out) {
  if (!basis || !basis->table || (n && (!states || !out))) return QKRYLOV_ERROR_INVALID_ARG;
  for (uint64_t i = 0; i < n; ++i) out[i] = basis->table->index(states[i]);
  return QKRYLOV_SUCCESS;
}

int qkrylov_opsum_add_term_nbody_f64(qkrylov_opsum_h opsum, double cr, double ci, int n, const char** ops,
                                     const int* sites) {
  if (!opsum || !ops || !sites || n <= 0) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    qkb::TermIn t;
    t.coeff = {cr, ci};
    for (int i = 0; i < n; ++i) {
      if (!ops[i]) return QKRYLOV_ERROR_INVALID_ARG;
      t.factors.push_back({std::string(ops[i]), sites[i]});
    }
    opsum->terms.push_back(std::move(t));
    return QKRYLOV_SUCCESS;
  });
}

uint64_t qkrylov_opsum_size(qkrylov_opsum_h opsum) { return opsum ? opsum->terms.size() : 0; }

int qkrylov_opsum_compile(qkrylov_basis_h basis, qkrylov_site_h site, qkrylov_opsum_h opsum, int* n_terms,
                          int* n_groups, int* has_diag, int* all_real, uint64_t* mask, double* coef,
                          uint64_t* flip, uint32_t* first, uint32_t* count, uint32_t* check) {
  if (!basis || !basis->table || !site || !opsum) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    const auto op = qkb::compile_opsum(site->family, *basis->table, opsum->terms);
    if (n_terms) *n_terms = int(op.terms.size());
    if (n_groups) *n_groups = int(op.groups.size());
    if (has_diag) *has_diag = op.has_diag;
    if (all_real) *all_real = op.all_real;
    for (size_t t = 0; t < op.terms.size(); ++t) {
      if (mask) { mask[3 * t] = op.terms[t].cmask; mask[3 * t + 1] = op.terms[t].cval; mask[3 * t + 2] = op.terms[t].smask; }
      if (coef) { coef[2 * t] = op.terms[t].wre; coef[2 * t + 1] = op.terms[t].wim; }
    }
    for (size_t g = 0; g < op.groups.size(); ++g) {
      if (flip) flip[g] = op.groups[g].flip;
      if (first) first[g] = op.groups[g].first;
      if (count) count[g] = op.groups[g].count;
      if (check) check[g] = op.groups[g].check;
    }
    return QKRYLOV_SUCCESS;
  });
}

qkrylov_hamiltonian_h qkrylov_hamiltonian_create_ex(qkrylov_basis_h basis, qkrylov_site_h site,
                                                   qkrylov_opsum_h opsum, int precision, int device) {
  if (!basis || !basis->table || !site || !opsum || (precision != 32 && precision != 64) || device < 0) {
    qkapi::set_error("invalid argument");
    return nullptr;
  }
  try {
    auto h = std::make_unique<qkrylov_hamiltonian_t>();
    h->op = std::make_shared<qkb::Operator>(site->family, basis->table, opsum->terms, device);
    h->precision = precision;
    return h.release();
  } catch (const std::exception& e) {
    qkapi::set_error(e.what());
    return nullptr;
  }
}

int qkrylov_hamiltonian_precision(qkrylov_hamiltonian_h h) { return (h && h->op) ? h->precision : 0; }
int qkrylov_hamiltonian_all_real(qkrylov_hamiltonian_h h) { return (h && h->op) ? int(h->op->all_real()) : 0; }
uint64_t qkrylov_hamiltonian_device_bytes(qkrylov_hamiltonian_h h) {
  return (h && h->op) ? qkd_plan_device_bytes(h->op->plan()) : 0;
}
void* qkrylov_hamiltonian_stream(qkrylov_hamiltonian_h h) {
  if (!h || !h->op) return nullptr;
  try { return h->op->ctx().stream; } catch (...) { return nullptr; }
}

int qkrylov_hamiltonian_apply_complex_f64(qkrylov_hamiltonian_h h, const double* x, double* y) {
  if (!h || !h->op || !x || !y) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    const uint64_t dim = h->op->dim();
    if (dim == 0) return QKRYLOV_SUCCESS;
    auto& c = h->op->ctx();
    std::lock_guard<std::mutex> lk(h->mu);
    h->stage(QK_C128);
    qkb::cuda_check(cudaMemcpyAsync(h->sx.data(), x, dim * 16, cudaMemcpyHostToDevice, c.stream), "H2D");
    h->op->apply(QK_C128, h->sx.data(), h->sy.data());
    qkb::cuda_check(cudaMemcpyAsync(y, h->sy.data(), dim * 16, cudaMemcpyDeviceToHost, c.stream), "D2H");
    c.sync();
    return QKRYLOV_SUCCESS;
  });
}

int qkrylov_hamiltonian_diagonal_complex_f64(qkrylov_hamiltonian_h h, double* d) {
  if (!h || !h->op || !d) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    const uint64_t dim = h->op->dim();
    if (dim == 0) return QKRYLOV_SUCCESS;
    auto& c = h->op->ctx();
    qkb::DevVec dd(dim, QK_C128, h->op->device(), false);
    h->op->diagonal(QK_C128, dd.data());
    qkb::cuda_check(cudaMemcpyAsync(d, dd.data(), dim * 16, cudaMemcpyDeviceToHost, c.stream), "D2H");
    c.sync();
    return QKRYLOV_SUCCESS;
  });
}

int qkrylov_hamiltonian_apply_device(qkrylov_hamiltonian_h h, int dtype, const void* x, void* y, void* stream) {
  if (!h || !h->op || !x || !y || !valid_dtype(dtype)) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    auto& c = h->op->ctx();
    const int rc = qkd_apply(h->op->plan(), qk_dtype(dtype), x, y, stream ? cudaStream_t(stream) : c.stream);
    if (rc == QKD_EINVAL) { qkapi::set_error("invalid dtype for this operator or aliased x/y"); return QKRYLOV_ERROR_INVALID_ARG; }
    qkb::qkd_check(rc, "H.x");
    return QKRYLOV_SUCCESS;
  });
}

int qkrylov_b200_basis_shard_bounds(qkrylov_basis_h basis, int nshards, uint64_t* bounds_out) {
  if (!basis || !basis->table || nshards < 1 || !bounds_out) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    const std::vector<uint64_t> b = basis->table->shard_bounds(nshards);
    std::copy(b.begin(), b.end(), bounds_out);
    return QKRYLOV_SUCCESS;
  });
}

int qkrylov_hamiltonian_apply_range_device(qkrylov_hamiltonian_h h, int dtype, const void* x, void* y,
                                           uint64_t row_lo, uint64_t row_hi, void* stream) {
  if (!h || !h->op || !x || !y || !valid_dtype(dtype) || row_lo > row_hi || row_hi > h->op->dim())
    return QKRYLOV_ERROR_INVALID_ARG;
  if (!h->op->basis().is_block_start(row_lo) || !h->op->basis().is_block_start(row_hi)) {
    qkapi::set_error("apply_range: the row bounds are not sector-block boundaries (qkrylov_b200_basis_shard_bounds)");
    return QKRYLOV_ERROR_INVALID_ARG;
  }
  return guarded([&] {
    auto& c = h->op->ctx();
    const int rc = qkd_apply_range(h->op->plan(), qk_dtype(dtype), x, y, row_lo, row_hi,
                                   stream ? cudaStream_t(stream) : c.stream);
    if (rc == QKD_EINVAL) { qkapi::set_error("invalid dtype for this operator or aliased x/y"); return QKRYLOV_ERROR_INVALID_ARG; }
    qkb::qkd_check(rc, "H.x rows");
    return QKRYLOV_SUCCESS;
  });
}

int qkrylov_b200_apply_block_device(qkrylov_hamiltonian_h h, int dtype, int R, int lanes_per_row, const void* X,
                                    void* Y, double* dots_out, void* stream) {
  if (!h || !h->op || !X || !Y || X == Y || !valid_dtype(dtype) || (R != 32 && R != 64 && R != 128) ||
      (lanes_per_row != 0 && lanes_per_row != 8 && lanes_per_row != 16 && lanes_per_row != 32) ||
      (lanes_per_row != 0 && R / lanes_per_row > 8))
    return QKRYLOV_ERROR_INVALID_ARG;
  if ((reinterpret_cast<uintptr_t>(X) | reinterpret_cast<uintptr_t>(Y)) & 15u) {
    qkapi::set_error("apply_block: X and Y must be 16-byte aligned");
    return QKRYLOV_ERROR_INVALID_ARG;
  }
  return guarded([&] {
    auto& c = h->op->ctx();
    c.activate();
    const cudaStream_t s = stream ? cudaStream_t(stream) : c.stream;
    qk_plan* plan = const_cast<qk_plan*>(h->op->plan());
    const qk_dtype t = qk_dtype(dtype);
    if (lanes_per_row == 0 && !qkd_rows_shape(plan, t, R)) {  // first call: tune the shape on these blocks
      int chosen = 0;
      const int rc = qkd_tune_rows(plan, c.ws, t, R, X, Y, nullptr, s, &chosen);
      if (rc == QKD_EINVAL) { qkapi::set_error("apply_block: invalid dtype for this operator"); return QKRYLOV_ERROR_INVALID_ARG; }
      qkb::qkd_check(rc, "block shape tuning");
    }
    double* dd = dots_out ? c.dres(0) : nullptr;
    const int rc = qkd_apply_rows(plan, c.ws, t, R, lanes_per_row, X, Y, nullptr, dd, s);
    if (rc == QKD_EINVAL) { qkapi::set_error("apply_block: invalid dtype for this operator"); return QKRYLOV_ERROR_INVALID_ARG; }
    qkb::qkd_check(rc, "block H.X");
    if (dots_out) {
      if (s != c.stream) qkb::cuda_check(cudaStreamSynchronize(s), "block H.X");
      const double* v = c.fetch(dd, 2 * R);
      for (int i = 0; i < 2 * R; ++i) dots_out[i] = v[i];
    }
    return QKRYLOV_SUCCESS;
  });
}

int qkrylov_b200_block_shape_timings(qkrylov_hamiltonian_h h, int dtype, int R, double* ms9) {
  if (!h || !h->op || !ms9 || !valid_dtype(dtype)) return QKRYLOV_ERROR_INVALID_ARG;
  float f[9];
  if (qkd_rows_timings(h->op->plan(), qk_dtype(dtype), R, f) != QKD_OK) return QKRYLOV_ERROR_INVALID_ARG;
  for (int i = 0; i < 9; ++i) ms9[i] = f[i];
  return QKRYLOV_SUCCESS;
}

int qkrylov_hamiltonian_diagonal_device(qkrylov_hamiltonian_h h, int dtype, void* d, void* stream) {
  if (!h || !h->op || !d || !valid_dtype(dtype)) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    auto& c = h->op->ctx();
    const int rc = qkd_diagonal(h->op->plan(), qk_dtype(dtype), d, stream ? cudaStream_t(stream) : c.stream);
    if (rc == QKD_EINVAL) return QKRYLOV_ERROR_INVALID_ARG;
    qkb::qkd_check(rc, "diagonal");
    return QKRYLOV_SUCCESS;
  });
}

int qkrylov_b200_spectral_function_batch(int device, int ncols, int ld, const double* alphas, const double* betas,
                                         const int* lengths, const double* norm_phi0, size_t n_omega,
                                         const double* omegas, double E0, double eta, double* out) {
  if (device < 0 || ncols < 0 || ld < 0 || (ncols > 0 && n_omega > 0 && (!alphas || !betas || !omegas || !out)) ||
      ncols > 65535)
    return QKRYLOV_ERROR_INVALID_ARG;
  if (lengths)
    for (int c = 0; c < ncols; ++c)
      if (lengths[c] < 0 || lengths[c] > ld) return QKRYLOV_ERROR_INVALID_ARG;
  if (ncols == 0 || n_omega == 0) return QKRYLOV_SUCCESS;
  return guarded([&] {
    auto& c = qkb::Context::get(device);
    c.activate();
    const size_t nc = size_t(ncols) * size_t(ld);
    const size_t bytes = (2 * nc + size_t(ncols) + n_omega + size_t(ncols) * n_omega) * sizeof(double) +
                         size_t(ncols) * sizeof(int);
    char* buf = static_cast<char*>(c.alloc(bytes));
    double* da = reinterpret_cast<double*>(buf);
    double* db = da + nc;
    double* dn = db + nc;
    double* dw = dn + ncols;
    double* dout = dw + n_omega;
    int* dl = reinterpret_cast<int*>(dout + size_t(ncols) * n_omega);
    int rc = QKD_OK;
    try {
      auto h2d = [&](void* d, const void* h, size_t b) {
        if (b) qkb::cuda_check(cudaMemcpyAsync(d, h, b, cudaMemcpyHostToDevice, c.stream), "H2D");
      };
      h2d(da, alphas, nc * sizeof(double));
      h2d(db, betas, nc * sizeof(double));
      if (norm_phi0) h2d(dn, norm_phi0, size_t(ncols) * sizeof(double));
      if (lengths) h2d(dl, lengths, size_t(ncols) * sizeof(int));
      h2d(dw, omegas, n_omega * sizeof(double));
      rc = qkd_spectral_batch(da, db, lengths ? dl : nullptr, ncols, ld, norm_phi0 ? dn : nullptr, dw, n_omega, E0,
                              eta, dout, c.stream);
      if (rc == QKD_OK)
        qkb::cuda_check(cudaMemcpyAsync(out, dout, size_t(ncols) * n_omega * sizeof(double), cudaMemcpyDeviceToHost,
                                        c.stream), "D2H");
      c.sync();
    } catch (...) {
      c.release(buf);
      throw;
    }
    c.release(buf);
    qkb::qkd_check(rc, "spectral function batch");
    return QKRYLOV_SUCCESS;
  });
}

int qkrylov_b200_apply_operator(qkrylov_basis_h basis, qkrylov_site_h site, qkrylov_opsum_h opsum, int device,
                                int dtype, const void* x, void* y, double* expectation) {
  if (!basis || !basis->table || !site || !opsum || device < 0 || !valid_dtype(dtype) || !x || !y || x == y)
    return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    qkb::Operator op(site->family, basis->table, opsum->terms, device);
    const qk_dtype t = qk_dtype(dtype);
    if (!qk_dtype_complex(t) && !op.all_real()) {
      qkapi::set_error("apply_operator: a complex operator needs complex vectors");
      return QKRYLOV_ERROR_INVALID_ARG;
    }
    auto& c = op.ctx();
    if (expectation) {
      op.apply_dot(t, x, y, c.dres(0));
      const double* v = c.fetch(c.dres(0), 2);
      expectation[0] = v[0];
      expectation[1] = v[1];
    } else {
      op.apply(t, x, y);
      c.sync();
    }
    return QKRYLOV_SUCCESS;
  });
}

int qkrylov_b200_multi_dot(int device, int dtype, size_t n, int k, const void* const* V, const void* x,
                           double* out) {
  if (device < 0 || !valid_dtype(dtype) || k <= 0 || !V || !x || !out) return QKRYLOV_ERROR_INVALID_ARG;
  for (int j = 0; j < k; ++j)
    if (!V[j]) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    auto& c = qkb::Context::get(device);
    qkb::PtrArray P(size_t(k), device);
    for (int j = 0; j < k; ++j) P.set(size_t(j), V[j], c.stream);
    qkb::DevVec res(2 * size_t(k), QK_F64, device, false);
    constexpr int kChunk = 511;
    for (int j0 = 0; j0 < k; j0 += kChunk) {
      const int kk = std::min(kChunk, k - j0);
      qkb::qkd_check(qkd_update_mdot(c.ws, qk_dtype(dtype), n, 0, nullptr, nullptr, kk, P.at(j0),
                                     const_cast<void*>(x), static_cast<double*>(res.data()) + 2 * j0, c.stream),
                     "multi-dot");
    }
    qkb::cuda_check(cudaMemcpyAsync(out, res.data(), sizeof(double) * 2 * k, cudaMemcpyDeviceToHost, c.stream), "D2H");
    c.sync();
    return QKRYLOV_SUCCESS;
  });
}

int qkrylov_lanczos_ground_state_f64(qkrylov_hamiltonian_h h, int maxiter, double tol, const double* start,
                                     qkrylov_lanczos_result_f64_t* result, double* evec, double* alphas,
                                     double* betas) {
  if (!h || !h->op || !result) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    std::vector<std::complex<double>> ritz;
    auto r = qkb::lanczos<double>(*h->op, maxiter, tol, reinterpret_cast<const std::complex<double>*>(start),
                                  evec ? &ritz : nullptr);
    result->energy = r.energy;
    result->iterations = r.iterations;
    result->converged = r.converged;
    result->n_alpha = int(r.alphas.size());
    result->n_beta = int(r.betas.size());
    if (evec && !ritz.empty()) std::memcpy(evec, ritz.data(), ritz.size() * 16);
    if (alphas) std::copy(r.alphas.begin(), r.alphas.end(), alphas);
    if (betas) std::copy(r.betas.begin(), r.betas.end(), betas);
    return QKRYLOV_SUCCESS;
  });
}

static int lanczos_two_phase(qkrylov_hamiltonian_h h, bool low_phase, uint64_t seed, const void* start,
                             int start_on_device, int maxiter, double tol, qkrylov_b200_mixed_result_t* result,
                             void* psi_out, int trace_cap, int* trace_iteration, double* trace_energy,
                             double* trace_seconds, bool partial = true) {
  if (!h || !h->op || !result || maxiter < 1 || maxiter > 511 || !(tol > 0) || trace_cap < 0)
    return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    const qkb::Operator& H = *h->op;
    const uint64_t dim = H.dim();
    const bool real = H.all_real();
    const qk_dtype st = low_phase ? (real ? QK_F32 : QK_C64) : (real ? QK_F64 : QK_C128);
    const qk_dtype hi = real ? QK_F64 : QK_C128;
    std::unique_ptr<qkb::DevVec> sdev, pdev;
    const void* sptr = start;
    if (start && !start_on_device) {
      sdev = std::make_unique<qkb::DevVec>(dim, st, H.device(), false);
      qkb::cuda_check(cudaMemcpyAsync(sdev->data(), start, dim * qk_dtype_size(st), cudaMemcpyHostToDevice,
                                      H.ctx().stream), "H2D");
      sptr = sdev->data();
    }
    if (psi_out) pdev = std::make_unique<qkb::DevVec>(dim, hi, H.device(), false);
    auto r = qkb::lanczos_mixed(H, sptr, seed, maxiter, tol, pdev ? pdev->data() : nullptr, low_phase, partial);
    if (psi_out) {
      qkb::cuda_check(cudaMemcpyAsync(psi_out, pdev->data(), dim * qk_dtype_size(hi), cudaMemcpyDeviceToHost,
                                      H.ctx().stream), "D2H");
      H.ctx().sync();
    }
    result->energy = r.energy;
    result->residual = r.residual;
    result->seconds_low = r.seconds_low;
    result->seconds_high = r.seconds_high;
    result->iterations_low = r.iters_low;
    result->iterations_high = r.iters_high;
    result->restarts = r.restarts;
    result->converged = r.converged;
    const int n = int(std::min<size_t>(size_t(trace_cap), r.trace.size()));
    for (int i = 0; i < n; ++i) {
      if (trace_iteration) trace_iteration[i] = r.trace[i].iteration;
      if (trace_energy) trace_energy[i] = r.trace[i].energy;
      if (trace_seconds) trace_seconds[i] = r.trace[i].seconds;
    }
    result->trace_len = n;
    return QKRYLOV_SUCCESS;
  });
}

int qkrylov_b200_lanczos_mixed(qkrylov_hamiltonian_h h, uint64_t seed, const void* start, int start_on_device,
                               int maxiter, double tol, qkrylov_b200_mixed_result_t* result, void* psi_out,
                               int trace_cap, int* trace_iteration, double* trace_energy, double* trace_seconds) {
  return lanczos_two_phase(h, true, seed, start, start_on_device, maxiter, tol, result, psi_out, trace_cap,
                           trace_iteration, trace_energy, trace_seconds);
}

int qkrylov_b200_lanczos_mixed_full(qkrylov_hamiltonian_h h, uint64_t seed, const void* start, int start_on_device,
                                    int maxiter, double tol, qkrylov_b200_mixed_result_t* result, void* psi_out,
                                    int trace_cap, int* trace_iteration, double* trace_energy,
                                    double* trace_seconds) {
  return lanczos_two_phase(h, true, seed, start, start_on_device, maxiter, tol, result, psi_out, trace_cap,
                           trace_iteration, trace_energy, trace_seconds, false);
}

int qkrylov_b200_lanczos_fp64(qkrylov_hamiltonian_h h, uint64_t seed, const void* start, int start_on_device,
                              int maxiter, double tol, qkrylov_b200_mixed_result_t* result, void* psi_out,
                              int trace_cap, int* trace_iteration, double* trace_energy, double* trace_seconds) {
  return lanczos_two_phase(h, false, seed, start, start_on_device, maxiter, tol, result, psi_out, trace_cap,
                           trace_iteration, trace_energy, trace_seconds);
}

static int ftlm_common(qkrylov_hamiltonian_h h, bool block, int precision, int n_random, int n_steps, uint64_t seed,
                       int n_vectors, int n_temps, const double* temps, double* logZ, double* U, double* Cv,
                       int use_graph, qkrylov_b200_ftlm_info_t* info) {
  if (!h || !h->op || (precision != 32 && precision != 64) || n_temps < 0 || (n_temps > 0 && !temps))
    return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    const qkb::Operator& H = *h->op;
    const bool real = H.all_real();
    const qk_dtype t = precision == 32 ? (real ? QK_F32 : QK_C64) : (real ? QK_F64 : QK_C128);
    const std::vector<double> T(temps, temps + n_temps);
    auto r = block ? qkb::ftlm_block(H, t, n_random, n_steps, seed, T, use_graph != 0)
                   : qkb::ftlm_loop(H, t, n_random, n_steps, seed, T, n_vectors);
    for (int q = 0; q < n_temps; ++q) {
      if (logZ) logZ[q] = r.logZ[q];
      if (U) U[q] = r.U[q];
      if (Cv) Cv[q] = r.Cv[q];
    }
    if (info) {
      info->seconds = r.seconds;
      info->seconds_device = r.seconds_device;
      info->e_min = r.e_min;
      info->lanes_per_row = r.lanes_per_row;
      info->graph = r.graph;
      info->vectors = r.R;
      info->steps = r.M;
    }
    return QKRYLOV_SUCCESS;
  });
}

int qkrylov_b200_ftlm_block(qkrylov_hamiltonian_h h, int precision, int n_random, int n_steps, uint64_t seed,
                            int n_temps, const double* temps, double* logZ, double* U, double* Cv, int use_graph,
                            qkrylov_b200_ftlm_info_t* info) {
  return ftlm_common(h, true, precision, n_random, n_steps, seed, 0, n_temps, temps, logZ, U, Cv, use_graph, info);
}

int qkrylov_b200_cf_block(qkrylov_hamiltonian_h h, int precision, int complex_vectors, int n_vectors, int n_steps,
                          const void* start, int start_on_device, int use_graph, double* alphas, double* betas,
                          double* norms, int* lengths, qkrylov_b200_ftlm_info_t* info) {
  if (!h || !h->op || (precision != 32 && precision != 64) || !start || !alphas || !betas ||
      (n_vectors != 32 && n_vectors != 64 && n_vectors != 128) || n_steps < 1 || n_steps > 1000)
    return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    const qkb::Operator& H = *h->op;
    const bool real = H.all_real() && !complex_vectors;
    const qk_dtype t = precision == 32 ? (real ? QK_F32 : QK_C64) : (real ? QK_F64 : QK_C128);
    const size_t count = size_t(H.dim()) * n_vectors;
    qkb::DevVec staged;
    const void* dstart = start;
    if (!start_on_device) {
      qkb::Context& c = H.ctx();
      c.activate();
      staged = qkb::DevVec(count, t, H.device(), false);
      qkb::cuda_check(cudaMemcpyAsync(staged.data(), start, staged.bytes(), cudaMemcpyHostToDevice, c.stream), "H2D");
      dstart = staged.data();
    }
    auto r = qkb::cf_block(H, t, n_vectors, n_steps, dstart, use_graph != 0);
    std::copy(r.alphas.begin(), r.alphas.end(), alphas);
    std::copy(r.betas.begin(), r.betas.end(), betas);
    for (int q = 0; q < n_vectors; ++q) {
      if (norms) norms[q] = std::sqrt(r.norm2[q]);
      if (lengths) lengths[q] = r.len[q];
    }
    if (info) {
      info->seconds = r.seconds;
      info->seconds_device = r.seconds_device;
      info->e_min = 0.0;
      info->lanes_per_row = r.lanes_per_row;
      info->graph = r.graph;
      info->vectors = r.R;
      info->steps = r.M;
    }
    return QKRYLOV_SUCCESS;
  });
}

int qkrylov_b200_ftlm_loop(qkrylov_hamiltonian_h h, int precision, int n_random, int n_steps, uint64_t seed,
                           int n_vectors, int n_temps, const double* temps, double* logZ, double* U, double* Cv,
                           qkrylov_b200_ftlm_info_t* info) {
  return ftlm_common(h, false, precision, n_random, n_steps, seed, n_vectors, n_temps, temps, logZ, U, Cv, 0, info);
}

struct qkrylov_b200_mlp_t {
  std::unique_ptr<qkb::WarmStartNet> net;
};

qkrylov_b200_mlp_h qkrylov_b200_mlp_create(qkrylov_basis_h basis, int device, uint64_t seed) {
  if (!basis || !basis->table) return nullptr;
  try {
    auto* h = new qkrylov_b200_mlp_t;
    h->net = std::make_unique<qkb::WarmStartNet>(basis->table, device, seed);
    return h;
  } catch (const std::exception& e) {
    qkapi::set_error(e.what());
    return nullptr;
  }
}

void qkrylov_b200_mlp_destroy(qkrylov_b200_mlp_h h) { delete h; }

size_t qkrylov_b200_mlp_num_params(qkrylov_b200_mlp_h h) { return h ? h->net->num_params() : 0; }

int qkrylov_b200_mlp_get_params(qkrylov_b200_mlp_h h, float* out) {
  if (!h || !out) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    const auto p = h->net->params();
    std::copy(p.begin(), p.end(), out);
    return QKRYLOV_SUCCESS;
  });
}

int qkrylov_b200_mlp_set_params(qkrylov_b200_mlp_h h, const float* in) {
  if (!h || !in) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    h->net->set_params(std::vector<float>(in, in + h->net->num_params()));
    return QKRYLOV_SUCCESS;
  });
}

int qkrylov_b200_mlp_set_tensor_cores(qkrylov_b200_mlp_h h, int on) {
  if (!h) return QKRYLOV_ERROR_INVALID_ARG;
  h->net->set_tensor_cores(on != 0);
  return QKRYLOV_SUCCESS;
}

int qkrylov_b200_mlp_add_target(qkrylov_b200_mlp_h h, double j2, const double* psi) {
  if (!h || !psi) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    h->net->add_target(j2, psi);
    return QKRYLOV_SUCCESS;
  });
}

int qkrylov_b200_mlp_train(qkrylov_b200_mlp_h h, int steps, int batch, double lr, uint64_t seed, double c_sign,
                           double* loss_out) {
  if (!h || steps < 0 || batch < 1 || !(lr > 0)) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    const auto l = h->net->train(steps, batch, lr, seed, c_sign);
    if (loss_out) std::copy(l.begin(), l.end(), loss_out);
    return QKRYLOV_SUCCESS;
  });
}

int qkrylov_b200_mlp_start_vector(qkrylov_b200_mlp_h h, double j2, float* out, int out_on_device) {
  if (!h || !out) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    const uint64_t dim = h->net->dim();
    if (out_on_device) {
      h->net->start_vector(j2, out);
      return QKRYLOV_SUCCESS;
    }
    qkb::Context& c = qkb::Context::get(h->net->device());
    qkb::DevVec d(dim, QK_F32, h->net->device(), false);
    h->net->start_vector(j2, static_cast<float*>(d.data()));
    // the start vector is written on the context's (non-blocking) stream
    qkb::cuda_check(cudaMemcpyAsync(out, d.data(), dim * 4, cudaMemcpyDeviceToHost, c.stream), "D2H");
    c.sync();
    return QKRYLOV_SUCCESS;
  });
}

int qkrylov_b200_mlp_loss_grad(qkrylov_b200_mlp_h h, int n, const uint64_t* states, const double* j2,
                               const float* targets, double c_sign, float* grad_out, double* loss_out) {
  if (!h || n < 1 || !states || !j2 || !targets) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    std::vector<float> g;
    const double l = h->net->loss_grad(n, states, j2, targets, c_sign, grad_out ? &g : nullptr);
    if (grad_out) std::copy(g.begin(), g.end(), grad_out);
    if (loss_out) *loss_out = l;
    return QKRYLOV_SUCCESS;
  });
}

int qkrylov_b200_lanczos_warm(qkrylov_hamiltonian_h h, qkrylov_b200_mlp_h net, double j2, int maxiter, double tol,
                              qkrylov_b200_mixed_result_t* result, double* seconds_inference) {
  if (!h || !h->op || !net || !result || maxiter < 1 || maxiter > 511 || !(tol > 0)) return QKRYLOV_ERROR_INVALID_ARG;
  if (!h->op->all_real() || h->op->dim() != net->net->dim()) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    const qkb::Operator& H = *h->op;
    const auto t0 = std::chrono::steady_clock::now();
    qkb::DevVec start(H.dim(), QK_F32, H.device(), false);
    net->net->start_vector(j2, static_cast<float*>(start.data()));
    H.ctx().sync();
    const double tinf = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    auto r = qkb::lanczos_mixed(H, start.data(), 0, maxiter, tol, nullptr, true);
    result->energy = r.energy;
    result->residual = r.residual;
    result->seconds_low = r.seconds_low + tinf;
    result->seconds_high = r.seconds_high;
    result->iterations_low = r.iters_low;
    result->iterations_high = r.iters_high;
    result->restarts = r.restarts;
    result->converged = r.converged;
    result->trace_len = 0;
    if (seconds_inference) *seconds_inference = tinf;
    return QKRYLOV_SUCCESS;
  });
}

int qkrylov_b200_davidson_block(qkrylov_hamiltonian_h h, int precision, int n_eig, int block, int max_subspace,
                                double tol, uint64_t seed, int maxiter, double* evals, double* residuals,
                                double* evecs, qkrylov_b200_davidson_info_t* info) {
  if (!h || !h->op || !evals || (precision != 32 && precision != 64) || !(tol > 0)) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    auto r = qkb::davidson_block(*h->op, precision == 32 ? QK_F32 : QK_F64, n_eig, block, max_subspace, tol, seed,
                                 maxiter, evecs);
    for (int a = 0; a < n_eig && a < int(r.eigenvalues.size()); ++a) evals[a] = r.eigenvalues[a];
    if (residuals)
      for (int a = 0; a < n_eig && a < int(r.residuals.size()); ++a) residuals[a] = r.residuals[a];
    if (info) {
      info->iterations = r.iterations;
      info->applies = r.applies;
      info->restarts = r.restarts;
      info->converged = r.converged;
      info->seconds = r.seconds;
    }
    return QKRYLOV_SUCCESS;
  });
}

int qkrylov_b200_lanczos_sweep(qkrylov_hamiltonian_h h0, qkrylov_hamiltonian_h h1, int n_couplings,
                               const double* couplings, int pass_len, int max_passes, double tol, uint64_t seed,
                               qkrylov_b200_mlp_h net, double* energies, double* residuals, int* converged,
                               qkrylov_b200_sweep_info_t* info) {
  if (!h0 || !h0->op || !h1 || !h1->op || !couplings || !energies || n_couplings < 1 || n_couplings > 128 ||
      pass_len < 2 || pass_len > 128 || max_passes < 1 || max_passes > 64 || !(tol > 0))
    return QKRYLOV_ERROR_INVALID_ARG;
  if (h0->op->dim() != h1->op->dim() || !h0->op->all_real() || !h1->op->all_real()) return QKRYLOV_ERROR_INVALID_ARG;
  if (net && (!net->net || net->net->dim() != h0->op->dim())) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    const std::vector<double> g(couplings, couplings + n_couplings);
    auto r = qkb::lanczos_sweep(*h0->op, *h1->op, g, pass_len, max_passes, tol, seed, net ? net->net.get() : nullptr);
    for (int q = 0; q < n_couplings; ++q) {
      energies[q] = r.energies[q];
      if (residuals) residuals[q] = r.residuals[q];
      if (converged) converged[q] = r.converged[q];
    }
    if (info) {
      info->block = r.R;
      info->steps = r.steps;
      info->passes = r.passes;
      info->applies = r.applies;
      info->lanes_per_row = r.lanes_per_row;
      info->seconds = r.seconds;
      info->seconds_inference = r.seconds_inference;
    }
    return QKRYLOV_SUCCESS;
  });
}

int qkrylov_davidson_lowest_f64(qkrylov_hamiltonian_h h, int n_eig, int max_subspace, double tol, double* evals,
                                double* evecs, qkrylov_davidson_result_c_t* info) {
  if (!h || !h->op || !evals || n_eig <= 0) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    auto r = qkb::davidson<double>(*h->op, n_eig, max_subspace, tol);
    const size_t k = std::min(size_t(n_eig), r.eigenvalues.size());
    for (size_t i = 0; i < k; ++i) evals[i] = r.eigenvalues[i];
    if (info) { info->iterations = r.iterations; info->converged = r.converged; }
    if (evecs) {
      const uint64_t dim = h->op->dim();
      for (size_t q = 0; q < k; ++q) std::memcpy(evecs + 2 * q * dim, r.eigenvectors[q].data(), dim * 16);
    }
    return QKRYLOV_SUCCESS;
  });
}

int qkrylov_continued_fraction_coeffs_f64(qkrylov_hamiltonian_h h, const double* phi0, int n_iter,
                                          double* alphas, double* betas, double* norm_phi0, int* na, int* nb) {
  if (!h || !h->op || !phi0 || !alphas || !betas || !norm_phi0 || n_iter <= 0) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    auto r = qkb::continued_fraction<double>(*h->op, reinterpret_cast<const std::complex<double>*>(phi0), n_iter);
    *norm_phi0 = r.norm_phi0;
    std::copy(r.alphas.begin(), r.alphas.end(), alphas);
    std::copy(r.betas.begin(), r.betas.end(), betas);
    if (na) *na = int(r.alphas.size());
    if (nb) *nb = int(r.betas.size());
    return QKRYLOV_SUCCESS;
  });
}

int qkrylov_b200_cf_checkpointed(qkrylov_hamiltonian_h h, const double* phi0, const char* resume_dir, int n_iter,
                                 const char* save_dir, double* alphas, double* betas, double* norm_phi0, int* na,
                                 int* nb) {
  if (!h || !h->op || (!phi0 && !resume_dir) || !alphas || !betas || !norm_phi0 || n_iter <= 0)
    return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    auto r = qkb::continued_fraction_checkpointed(*h->op, resume_dir ? nullptr : reinterpret_cast<const std::complex<double>*>(phi0),
                                                  resume_dir ? resume_dir : "", n_iter, save_dir ? save_dir : "");
    if (int(r.alphas.size()) > n_iter) {  // a checkpoint longer than the requested run
      qkapi::set_error("cf_checkpointed: the checkpoint holds more steps than n_iter");
      return QKRYLOV_ERROR_INVALID_ARG;
    }
    *norm_phi0 = r.norm_phi0;
    std::copy(r.alphas.begin(), r.alphas.end(), alphas);
    std::copy(r.betas.begin(), r.betas.end(), betas);
    if (na) *na = int(r.alphas.size());
    if (nb) *nb = int(r.betas.size());
    return QKRYLOV_SUCCESS;
  });
}

double qkrylov_evaluate_spectral_function_f64(const double* alphas, const double* betas, size_t n,
                                              double norm_phi0, double omega, double E0, double eta) {
  if (!alphas || n == 0 || (n > 1 && !betas)) return 0.0;
  std::vector<double> b(n, 0.0);
  for (size_t i = 0; i + 1 < n; ++i) b[i] = betas[i];
  return qkb::spectral_function<double>(alphas, b.data(), n, norm_phi0, omega, E0, eta);
}

int qkrylov_ftlm_sweep_f64(qkrylov_hamiltonian_h h, int n_beta, const double* betas, int n_random, int n_steps,
                           double* Z, double* U, double* Cv) {
  if (!h || !h->op || n_beta <= 0 || !betas || !Z || !U || !Cv) return QKRYLOV_ERROR_INVALID_ARG;
  return guarded([&] {
    auto r = qkb::ftlm<double>(*h->op, std::vector<double>(betas, betas + n_beta), n_random, n_steps);
    for (int q = 0; q < n_beta; ++q) { Z[q] = r[q].Z; U[q] = r[q].U; Cv[q] = r[q].Cv; }
    return QKRYLOV_SUCCESS;
  });
}

}  // extern "C"
