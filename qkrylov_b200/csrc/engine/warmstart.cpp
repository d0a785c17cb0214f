#include "warmstart.hpp"

#include <cmath>
#include <random>
#include <stdexcept>

#include "kernels/dev_api.h"

extern "C" {
int qkd_mlp_gemm(int M, int N, int K, int a_bf16, const void* A, int lda, int trans_a, int b_bf16, const void* B,
                 int ldb, int trans_b, const float* bias, float* C, int ldc, float* Z, int gelu_ep, cudaStream_t s);
int qkd_mlp_inputs(int n, int nsites, const uint64_t* states, const uint32_t* idx, const float* j2, float j2_all,
                   float* X, int ldx, cudaStream_t s);
int qkd_mlp_gelu_bwd(size_t n, const float* dH, const float* Z, float* dZ, cudaStream_t s);
int qkd_mlp_colsum(int M, int N, const float* D, float* db, cudaStream_t s);
int qkd_mlp_loss(qk_workspace* w, int n, const float* O, const float* tgt, float c_sign, float* dO, double* loss,
                 cudaStream_t s);
int qkd_mlp_adam(size_t n, float* p, const float* g, float* m, float* v, float lr, float b1, float b2, int t,
                 float eps, void* pb, size_t nw, cudaStream_t s);
int qkd_mlp_tobf16(size_t n, const float* p, void* pb, cudaStream_t s);
int qkd_mlp_startvec(int n, const uint64_t* states, uint64_t marshall, const float* O, float shift, float* out,
                     cudaStream_t s);
int qkd_cdf(qk_dtype t, size_t n, const void* psi, double* cdf, double* bsum, cudaStream_t s);
int qkd_sample(qk_dtype t, int m, size_t n, const double* cdf, const void* psi, const uint64_t* states,
               uint64_t marshall, double log_max, uint64_t seed, uint32_t* idx, float* tgt, cudaStream_t s);
int qkd_max_f32(qk_workspace* w, size_t n, const float* x, int stride, float* out, cudaStream_t s);
int qkd_mlp_forward_tc(int n, int nsites, const uint64_t* states, float j2, const void* w1, const void* w2,
                       const void* w3, const float* b1, const float* b2, const float* b3, float* out, int* err,
                       cudaStream_t s);
}

namespace qkb {

namespace {
template <class T> void dalloc(T** p, size_t n) {
  cuda_check(cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(n, 1) * sizeof(T)), "device allocation");
}
template <class T> void dfree(T*& p) { if (p) cudaFree(p); p = nullptr; }
constexpr int H_ = WarmStartNet::kHidden;
constexpr int kChunk = 65536;  // inference rows per pass
}  // namespace

WarmStartNet::WarmStartNet(std::shared_ptr<const SectorTable> basis, int device, uint64_t seed)
    : basis_(std::move(basis)), dev_(device) {
  if (!basis_ || basis_->family != Family::Spin) throw std::invalid_argument("qkrylov_b200: warm start needs a spin-1/2 basis");
  nsites_ = basis_->nsites;
  if (nsites_ < 2 || nsites_ > 62) throw std::invalid_argument("qkrylov_b200: warm start needs 2..62 sites");
  ki_ = nsites_ + 1;
  dim_ = basis_->dim;
  if (dim_ == 0 || dim_ >= (1ull << 31)) throw std::invalid_argument("qkrylov_b200: warm start basis size");
  marshall_ = 0;
  for (int b = 1; b < nsites_; b += 2) marshall_ |= 1ull << b;  // odd sublattice
  nw_ = size_t(H_) * ki_ + size_t(H_) * H_ + 2 * size_t(H_);
  off_w2_ = size_t(H_) * ki_;
  off_w3_ = off_w2_ + size_t(H_) * H_;
  off_b1_ = nw_;
  off_b2_ = off_b1_ + H_;
  off_b3_ = off_b2_ + H_;
  np_ = off_b3_ + 2;
  Context& c = Context::get(dev_);
  c.activate();
  dalloc(&p_, np_); dalloc(&g_, np_); dalloc(&m_, np_); dalloc(&v_, np_);
  cuda_check(cudaMalloc(&pb_, nw_ * 2), "device allocation");
  cuda_check(cudaMemset(m_, 0, np_ * 4), "memset");
  cuda_check(cudaMemset(v_, 0, np_ * 4), "memset");
  // states of the basis, in index order
  std::vector<uint64_t> st(dim_);
  for (uint64_t i = 0; i < dim_; ++i) st[i] = basis_->state(i);
  dalloc(&states_, dim_);
  cuda_check(cudaMemcpy(states_, st.data(), dim_ * 8, cudaMemcpyHostToDevice), "H2D");
  // He-style uniform initialisation, biases 0
  std::mt19937_64 rng(seed);
  std::vector<float> p(np_, 0.f);
  auto fill = [&](size_t off, size_t n, int fan_in) {
    std::uniform_real_distribution<float> u(-1.f, 1.f);
    const float a = std::sqrt(3.f / float(fan_in));
    for (size_t i = 0; i < n; ++i) p[off + i] = a * u(rng);
  };
  fill(0, size_t(H_) * ki_, ki_);
  fill(off_w2_, size_t(H_) * H_, H_);
  fill(off_w3_, 2 * size_t(H_), H_);
  set_params(p);
}

WarmStartNet::~WarmStartNet() {
  cudaSetDevice(dev_);
  dfree(p_); dfree(g_); dfree(m_); dfree(v_);
  if (pb_) cudaFree(pb_);
  dfree(states_);
  dfree(X_); dfree(Z1_); dfree(H1_); dfree(Z2_); dfree(H2_); dfree(O_); dfree(dO_); dfree(dH_); dfree(dZ_);
  dfree(tgt_); dfree(j2_); dfree(idx_);
  dfree(err_);
}

std::vector<float> WarmStartNet::params() const {
  std::vector<float> p(np_);
  Context::get(dev_).activate();
  cuda_check(cudaMemcpy(p.data(), p_, np_ * 4, cudaMemcpyDeviceToHost), "D2H");
  return p;
}

void WarmStartNet::set_params(const std::vector<float>& p) {
  if (p.size() != np_) throw std::invalid_argument("qkrylov_b200: parameter vector has the wrong size");
  Context& c = Context::get(dev_);
  c.activate();
  cuda_check(cudaMemcpy(p_, p.data(), np_ * 4, cudaMemcpyHostToDevice), "H2D");
  qkd_check(qkd_mlp_tobf16(nw_, p_, pb_, c.stream), "bf16");
  c.sync();
}

void WarmStartNet::add_target(double j2, const double* psi) {
  Context& c = Context::get(dev_);
  c.activate();
  Target t{j2, 0.0, DevVec(dim_, QK_F64, dev_, false), DevVec(dim_, QK_F64, dev_, false),
           DevVec((dim_ + 1023) / 1024 + 1, QK_F64, dev_, false)};
  double mx = 0.0;
  for (uint64_t i = 0; i < dim_; ++i) mx = std::max(mx, std::abs(psi[i]));
  if (!(mx > 0)) throw std::invalid_argument("qkrylov_b200: zero target state");
  t.log_max = std::log(mx);
  cuda_check(cudaMemcpyAsync(t.psi.data(), psi, dim_ * 8, cudaMemcpyHostToDevice, c.stream), "H2D");
  qkd_check(qkd_cdf(QK_F64, dim_, t.psi.data(), static_cast<double*>(t.cdf.data()),
                    static_cast<double*>(t.bsum.data()), c.stream), "cdf");
  c.sync();
  targets_.push_back(std::move(t));
}

void WarmStartNet::ensure_batch(int n) {
  if (n <= cap_) return;
  dfree(X_); dfree(Z1_); dfree(H1_); dfree(Z2_); dfree(H2_); dfree(O_); dfree(dO_); dfree(dH_); dfree(dZ_);
  dfree(tgt_); dfree(j2_); dfree(idx_);
  const size_t m = size_t(n);
  dalloc(&X_, m * ki_); dalloc(&Z1_, m * H_); dalloc(&H1_, m * H_); dalloc(&Z2_, m * H_); dalloc(&H2_, m * H_);
  dalloc(&O_, m * 2); dalloc(&dO_, m * 2); dalloc(&dH_, m * H_); dalloc(&dZ_, m * H_);
  dalloc(&tgt_, m * 3); dalloc(&j2_, m); dalloc(&idx_, m);
  cap_ = n;
}

// X -> Z1, H1 -> Z2, H2 -> O for n samples (idx into states, or states
// 0..n-1 of the given array); BF16 weights, FP32 accumulation.
void WarmStartNet::forward(int n, const uint32_t* idx, const uint64_t* states, const float* j2, float j2_all) {
  Context& c = Context::get(dev_);
  const auto* pb = static_cast<const uint16_t*>(pb_);
  qkd_check(qkd_mlp_inputs(n, nsites_, states, idx, j2, j2_all, X_, ki_, c.stream), "inputs");
  qkd_check(qkd_mlp_gemm(n, H_, ki_, 0, X_, ki_, 0, 1, pb, ki_, 1, p_ + off_b1_, H1_, H_, Z1_, 1, c.stream), "layer 1");
  qkd_check(qkd_mlp_gemm(n, H_, H_, 0, H1_, H_, 0, 1, pb + off_w2_, H_, 1, p_ + off_b2_, H2_, H_, Z2_, 1, c.stream),
            "layer 2");
  qkd_check(qkd_mlp_gemm(n, 2, H_, 0, H2_, H_, 0, 1, pb + off_w3_, H_, 1, p_ + off_b3_, O_, 2, nullptr, 0, c.stream),
            "layer 3");
}

// Loss on the current forward pass and gradient (FP32) into g_.
double WarmStartNet::backward(int n, const float* tgt, double c_sign) {
  Context& c = Context::get(dev_);
  const auto* pb = static_cast<const uint16_t*>(pb_);
  double* loss = c.dres(0);
  qkd_check(qkd_mlp_loss(c.ws, n, O_, tgt, float(c_sign), dO_, loss, c.stream), "loss");
  // layer 3: dW3 = dO^T H2, db3 = sum dO, dH2 = dO W3
  qkd_check(qkd_mlp_gemm(2, H_, n, 0, dO_, 2, 1, 0, H2_, H_, 0, nullptr, g_ + off_w3_, H_, nullptr, 0, c.stream), "dW3");
  qkd_check(qkd_mlp_colsum(n, 2, dO_, g_ + off_b3_, c.stream), "db3");
  qkd_check(qkd_mlp_gemm(n, H_, 2, 0, dO_, 2, 0, 1, pb + off_w3_, H_, 0, nullptr, dH_, H_, nullptr, 0, c.stream), "dH2");
  qkd_check(qkd_mlp_gelu_bwd(size_t(n) * H_, dH_, Z2_, dZ_, c.stream), "gelu'");
  // layer 2: dW2 = dZ2^T H1, db2, dH1 = dZ2 W2
  qkd_check(qkd_mlp_gemm(H_, H_, n, 0, dZ_, H_, 1, 0, H1_, H_, 0, nullptr, g_ + off_w2_, H_, nullptr, 0, c.stream), "dW2");
  qkd_check(qkd_mlp_colsum(n, H_, dZ_, g_ + off_b2_, c.stream), "db2");
  qkd_check(qkd_mlp_gemm(n, H_, H_, 0, dZ_, H_, 0, 1, pb + off_w2_, H_, 0, nullptr, dH_, H_, nullptr, 0, c.stream), "dH1");
  qkd_check(qkd_mlp_gelu_bwd(size_t(n) * H_, dH_, Z1_, dZ_, c.stream), "gelu'");
  // layer 1: dW1 = dZ1^T X, db1
  qkd_check(qkd_mlp_gemm(H_, ki_, n, 0, dZ_, H_, 1, 0, X_, ki_, 0, nullptr, g_, ki_, nullptr, 0, c.stream), "dW1");
  qkd_check(qkd_mlp_colsum(n, H_, dZ_, g_ + off_b1_, c.stream), "db1");
  return c.fetch(loss, 1)[0];
}

std::vector<double> WarmStartNet::train(int steps, int batch, double lr, uint64_t seed, double c_sign) {
  if (targets_.empty()) throw std::invalid_argument("qkrylov_b200: no training targets");
  const int T = int(targets_.size());
  const int per = std::max(1, batch / T);
  const int n = per * T;
  Context& c = Context::get(dev_);
  c.activate();
  ensure_batch(n);
  std::vector<double> hist;
  hist.reserve(steps);
  for (int s = 0; s < steps; ++s) {
    for (int k = 0; k < T; ++k) {
      const Target& t = targets_[k];
      qkd_check(qkd_sample(QK_F64, per, dim_, static_cast<const double*>(t.cdf.data()), t.psi.data(), states_,
                           marshall_, t.log_max, seed * 1000003ull + uint64_t(s) * 4099ull + uint64_t(k),
                           idx_ + size_t(k) * per, tgt_ + size_t(k) * per * 3, c.stream), "sample");
      qkd_check(qkd_fill(QK_F32, per, j2_ + size_t(k) * per, t.j2, 0.0, c.stream), "fill");
    }
    forward(n, idx_, states_, j2_, 0.f);
    hist.push_back(backward(n, tgt_, c_sign));
    // cosine decay from lr to lr/20
    const double f = 0.05 + 0.95 * 0.5 * (1.0 + std::cos(M_PI * double(s) / std::max(1, steps - 1)));
    qkd_check(qkd_mlp_adam(np_, p_, g_, m_, v_, float(lr * f), 0.9f, 0.999f, ++adam_t_, 1e-8f, pb_, nw_, c.stream),
              "adam");
  }
  c.sync();
  return hist;
}

void WarmStartNet::start_vector(double j2, float* out) {
  Context& c = Context::get(dev_);
  c.activate();
  ensure_batch(kChunk);
  DevVec O(2 * dim_, QK_F32, dev_, false);
  float* Oall = static_cast<float*>(O.data());
  if (tc_) {
    if (!err_) dalloc(&err_, 1);
    cuda_check(cudaMemsetAsync(err_, 0, sizeof(int), c.stream), "memset");
    const auto* pb = static_cast<const uint16_t*>(pb_);
    qkd_check(qkd_mlp_forward_tc(int(dim_), nsites_, states_, float(j2), pb, pb + off_w2_, pb + off_w3_,
                                 p_ + off_b1_, p_ + off_b2_, p_ + off_b3_, Oall, err_, c.stream), "tensor-core forward");
    int e = 0;
    cuda_check(cudaMemcpyAsync(&e, err_, sizeof(int), cudaMemcpyDeviceToHost, c.stream), "D2H");
    c.sync();
    if (e) throw DeviceError("qkrylov_b200: tensor-core forward: an MMA completion wait expired");
  } else {
    for (uint64_t r0 = 0; r0 < dim_; r0 += kChunk) {
      const int n = int(std::min<uint64_t>(kChunk, dim_ - r0));
      forward(n, nullptr, states_ + r0, nullptr, float(j2));
      cuda_check(cudaMemcpyAsync(Oall + 2 * r0, O_, size_t(n) * 2 * 4, cudaMemcpyDeviceToDevice, c.stream), "copy");
    }
  }
  // shift by the largest log-amplitude so that exp() cannot overflow
  float* mx = reinterpret_cast<float*>(c.dres(0));
  qkd_check(qkd_max_f32(c.ws, dim_, Oall, 2, mx, c.stream), "max");
  const float shift = *reinterpret_cast<const float*>(c.fetch(c.dres(0), 1));
  qkd_check(qkd_mlp_startvec(int(dim_), states_, marshall_, Oall, shift, out, c.stream), "start vector");
}

double WarmStartNet::loss_grad(int n, const uint64_t* states, const double* j2, const float* targets, double c_sign,
                               std::vector<float>* grad) {
  if (n <= 0) throw std::invalid_argument("qkrylov_b200: empty sample set");
  Context& c = Context::get(dev_);
  c.activate();
  ensure_batch(n);
  uint64_t* st = nullptr;
  dalloc(&st, size_t(n));
  std::vector<float> jf(j2, j2 + n);
  try {
    cuda_check(cudaMemcpyAsync(st, states, size_t(n) * 8, cudaMemcpyHostToDevice, c.stream), "H2D");
    cuda_check(cudaMemcpyAsync(j2_, jf.data(), size_t(n) * 4, cudaMemcpyHostToDevice, c.stream), "H2D");
    cuda_check(cudaMemcpyAsync(tgt_, targets, size_t(n) * 12, cudaMemcpyHostToDevice, c.stream), "H2D");
    forward(n, nullptr, st, j2_, 0.f);
    const double l = backward(n, tgt_, c_sign);
    if (grad) {
      grad->resize(np_);
      cuda_check(cudaMemcpy(grad->data(), g_, np_ * 4, cudaMemcpyDeviceToHost), "D2H");
    }
    dfree(st);
    return l;
  } catch (...) {
    dfree(st);
    throw;
  }
}

}  // namespace qkb
