// Public C++ API objects for one precision namespace (this file is compiled
// twice: with QKRYLOV_DOUBLE_PRECISION for fp64 and without for fp32).
#include <cuda_runtime.h>

#include <stdexcept>

#include "engine/compile.hpp"
#include "engine/operator.hpp"
#include "engine/runtime.hpp"
#include "engine/sector.hpp"
#include "qkrylov/basis/basis.hpp"
#include "qkrylov/hamiltonian/matrix_free_hamiltonian.hpp"
#include "qkrylov/linalg/vector_ops.hpp"
#include "qkrylov/sites/site.hpp"

namespace qkrylov {
namespace QKRYLOV_PRECISION_NAMESPACE {

namespace {
constexpr qk_dtype kVecType = sizeof(Real) == 8 ? QK_C128 : QK_C64;
qkb::Family fam(int f) {
  if (f < 0 || f > 3) throw std::invalid_argument("qkrylov_b200: unsupported site/basis family");
  return static_cast<qkb::Family>(f);
}
}  // namespace

namespace detail {

LocalAction site_apply(int family, const std::string& op, int site, StateID state) {
  const auto a = qkb::apply_factor(fam(family), op, site, state);
  LocalAction r;
  r.valid = a.valid;
  r.new_state = a.new_state;
  r.matrix_element = Complex(Real(a.me.real()), Real(a.me.imag()));
  return r;
}

std::shared_ptr<const qkb::SectorTable> make_table(int family, int N, const Sector& s) {
  qkb::SectorSpec spec;
  spec.use_sz = s.use_sz; spec.sz2 = s.sz2;
  spec.use_nup = s.use_nup; spec.use_ndn = s.use_ndn; spec.nup = s.nup; spec.ndn = s.ndn;
  spec.use_n = s.use_n; spec.n = s.n; spec.use_nb = s.use_nb; spec.nb = s.nb;
  return std::make_shared<const qkb::SectorTable>(fam(family), N, spec);
}
Index table_size(const qkb::SectorTable& t) { return Index(t.dim); }
StateID table_state(const qkb::SectorTable& t, Index i) { return t.state(i); }
long long table_index(const qkb::SectorTable& t, StateID s) { return t.index(s); }

KComplex vec_dot(const KComplex* x, const KComplex* y, std::size_t n, int device) {
  auto& c = qkb::Context::get(device);
  qkb::qkd_check(qkd_dot(c.ws, kVecType, n, x, y, c.dres(0), c.stream), "dot");
  const double* r = c.fetch(c.dres(0), 2);
  return KComplex(Real(r[0]), Real(r[1]));
}
void vec_scal(KComplex a, KComplex* x, std::size_t n, int device) {
  auto& c = qkb::Context::get(device);
  qkb::qkd_check(qkd_scal(kVecType, n, a.real(), a.imag(), x, c.stream), "scal");
}
void vec_axpy(KComplex a, const KComplex* x, KComplex* y, std::size_t n, int device) {
  auto& c = qkb::Context::get(device);
  qkb::qkd_check(qkd_axpy(kVecType, n, a.real(), a.imag(), x, y, c.stream), "axpy");
}
void vec_fill(KComplex v, KComplex* x, std::size_t n, int device) {
  auto& c = qkb::Context::get(device);
  qkb::qkd_check(qkd_fill(kVecType, n, x, v.real(), v.imag(), c.stream), "fill");
}
void vec_copy(KComplex* dst, const KComplex* src, std::size_t n, int device) {
  auto& c = qkb::Context::get(device);
  qkb::qkd_check(qkd_copy(kVecType, n, src, dst, c.stream), "copy");
}
void vec_h2d(const KComplex* h, KComplex* d, std::size_t n, int device) {
  auto& c = qkb::Context::get(device);
  qkb::cuda_check(cudaMemcpyAsync(d, h, n * sizeof(KComplex), cudaMemcpyHostToDevice, c.stream), "H2D");
  c.sync();
}
void vec_d2h(const KComplex* d, KComplex* h, std::size_t n, int device) {
  auto& c = qkb::Context::get(device);
  qkb::cuda_check(cudaMemcpyAsync(h, d, n * sizeof(KComplex), cudaMemcpyDeviceToHost, c.stream), "D2H");
  c.sync();
}

}  // namespace detail

template <typename ExecSpace>
MatrixFreeHamiltonian<ExecSpace>::MatrixFreeHamiltonian(std::shared_ptr<Basis> basis,
                                                        std::shared_ptr<Site> site, const OpSum& ops,
                                                        Device device)
    : device_(device), basis_(std::move(basis)), site_(std::move(site)), ops_(ops) {
  if (!basis_ || !site_) throw std::invalid_argument("qkrylov_b200: null basis or site");
  auto table = basis_->table();
  if (!table) throw std::invalid_argument("qkrylov_b200: basis type is not supported (use this library's bases)");
  if (site_->family() < 0) throw std::invalid_argument("qkrylov_b200: site type is not supported (use this library's sites)");
  detail::initialize_kokkos(device_);
  std::vector<qkb::TermIn> terms;
  terms.reserve(ops_.size());
  for (const auto& t : ops_.terms()) {
    qkb::TermIn ti;
    ti.coeff = std::complex<double>(double(t.coeff.real()), double(t.coeff.imag()));
    for (const auto& f : t.factors) ti.factors.push_back({f.op, f.site});
    terms.push_back(std::move(ti));
  }
  op_ = std::make_shared<qkb::Operator>(static_cast<qkb::Family>(site_->family()), table, terms, device_.id);
  dim_ = Index(op_->dim());
  diagonal_ = VectorView<ExecSpace>("qkrylov::diagonal", dim_, device_.id);
  op_->diagonal(kVecType, diagonal_.data());
  op_->ctx().sync();
}

template <typename ExecSpace>
MatrixFreeHamiltonian<ExecSpace>::~MatrixFreeHamiltonian() = default;

template <typename ExecSpace>
void MatrixFreeHamiltonian<ExecSpace>::apply(const VectorView<ExecSpace>& x, VectorView<ExecSpace>& y) const {
  if (x.extent(0) != dim_ || y.extent(0) != dim_)
    throw std::invalid_argument("qkrylov_b200: vector size does not match the Hamiltonian dimension");
  if (dim_ == 0) return;
  op_->apply(kVecType, x.data(), y.data());
  op_->ctx().sync();
}

template <typename ExecSpace>
void MatrixFreeHamiltonian<ExecSpace>::apply(const Complex* x, Complex* y) const {
  if (dim_ == 0) return;
  std::lock_guard<std::mutex> lk(host_mu_);
  if (hx_.extent(0) != dim_) {
    hx_ = VectorView<ExecSpace>("x_temp", dim_, device_.id);
    hy_ = VectorView<ExecSpace>("y_temp", dim_, device_.id);
  }
  auto& c = op_->ctx();
  qkb::cuda_check(cudaMemcpyAsync(hx_.data(), x, dim_ * sizeof(Complex), cudaMemcpyHostToDevice, c.stream), "H2D");
  op_->apply(kVecType, hx_.data(), hy_.data());
  qkb::cuda_check(cudaMemcpyAsync(y, hy_.data(), dim_ * sizeof(Complex), cudaMemcpyDeviceToHost, c.stream), "D2H");
  c.sync();
}

template <typename ExecSpace>
HostVector MatrixFreeHamiltonian<ExecSpace>::diagonal_host() const {
  HostVector h;
  copy_device_to_host(diagonal_, h);
  return h;
}

template class MatrixFreeHamiltonian<CudaSpace>;

}  // namespace QKRYLOV_PRECISION_NAMESPACE
}  // namespace qkrylov
