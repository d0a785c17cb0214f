// Learned warm start: an MLP over spin configurations and the coupling J2,
// in 25 (spins as +-1, J2) -> 128 -> 128 -> 2 (log-amplitude, sign logit),
// GELU, BF16 weights with FP32 accumulation, trained on the GPU by the
// project's own kernels on ground states from plain Lanczos at a few
// couplings, and evaluated at new couplings as the Lanczos start vector
//   phi(s) = M(s) exp(o0(s)) tanh(o1(s)),  M(s) = (-1)^popcount(s & marshall)
// where M is Marshall's sign rule for the bipartite chain (the network
// learns the deviation from it in o1).
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include "runtime.hpp"
#include "sector.hpp"

namespace qkb {

class WarmStartNet {
 public:
  static constexpr int kHidden = 128;
  WarmStartNet(std::shared_ptr<const SectorTable> basis, int device, uint64_t seed);
  ~WarmStartNet();
  WarmStartNet(const WarmStartNet&) = delete;
  WarmStartNet& operator=(const WarmStartNet&) = delete;

  int nsites() const { return nsites_; }
  uint64_t dim() const { return dim_; }
  int device() const { return dev_; }
  size_t num_params() const { return np_; }
  size_t num_weights() const { return nw_; }
  // Parameters in FP32: W1 [128][nsites+1], W2 [128][128], W3 [2][128], b1, b2, b3.
  std::vector<float> params() const;
  void set_params(const std::vector<float>& p);
  // A training ground state (real, FP64, host memory, dim entries).
  void add_target(double j2, const double* psi);
  int num_targets() const { return int(targets_.size()); }
  // Adam steps on minibatches of `batch` samples drawn by |psi|^2, split
  // evenly over the targets; returns the loss of every step.
  std::vector<double> train(int steps, int batch, double lr, uint64_t seed, double c_sign);
  // Start vector at coupling j2 over the whole basis, FP32, into device
  // memory `out` (dim floats), not normalised.
  void start_vector(double j2, float* out);
  // Inference on the tensor cores (tcgen05, BF16 activations; default) or
  // on the CUDA cores (FP32 activations, the training forward).
  void set_tensor_cores(bool on) { tc_ = on; }
  bool tensor_cores() const { return tc_; }
  // Loss and gradient (FP32, layout of params()) on explicit samples.
  double loss_grad(int n, const uint64_t* states, const double* j2, const float* targets, double c_sign,
                   std::vector<float>* grad);

 private:
  void ensure_batch(int n);
  void forward(int n, const uint32_t* idx, const uint64_t* states, const float* j2, float j2_all);
  double backward(int n, const float* tgt, double c_sign);  // loss; gradient into grad_

  std::shared_ptr<const SectorTable> basis_;
  int dev_, nsites_, ki_;
  uint64_t dim_, marshall_;
  size_t np_, nw_;
  size_t off_w2_, off_w3_, off_b1_, off_b2_, off_b3_;
  float *p_ = nullptr, *g_ = nullptr, *m_ = nullptr, *v_ = nullptr;
  void* pb_ = nullptr;                     // BF16 weights
  uint64_t* states_ = nullptr;             // all basis states on the device
  int adam_t_ = 0;
  struct Target { double j2, log_max; DevVec psi, cdf, bsum; };
  std::vector<Target> targets_;
  int cap_ = 0;                            // batch scratch capacity
  float *X_ = nullptr, *Z1_ = nullptr, *H1_ = nullptr, *Z2_ = nullptr, *H2_ = nullptr, *O_ = nullptr,
        *dO_ = nullptr, *dH_ = nullptr, *dZ_ = nullptr, *tgt_ = nullptr, *j2_ = nullptr;
  uint32_t* idx_ = nullptr;
  bool tc_ = true;
  int* err_ = nullptr;  // device flag of the tensor-core kernel
};

}  // namespace qkb
