// Streaming kernels on row-interleaved blocks of R vectors (element (i, r)
// at i*R + r), the vector side of the batched Lanczos recurrences: per
// column coefficient updates with fused FP64 column norms, column scaling
// with breakdown bookkeeping, and column extraction.  Coefficients are read
// from device memory, so a whole Lanczos step runs without a host round
// trip and can be captured in a CUDA graph.
#include <algorithm>

#include "reduce.cuh"

namespace qkd {
namespace {

constexpr int kBT = 256;

inline unsigned block_grid(size_t n) {
  int dev = 0;
  cudaGetDevice(&dev);
  const size_t need = (n + kBT - 1) / kBT;
  return unsigned(std::max<size_t>(1, std::min<size_t>(need, std::min<size_t>(size_t(sm_count(dev)) * 4, kMaxG))));
}

// The grid stride (gridDim * 256) is a multiple of R, so every thread stays
// on one column c = (global thread index) % R.
template <int DT>
__global__ void __launch_bounds__(kBT)
k_block_update(size_t n, int R, const void* __restrict__ V, const double* __restrict__ a,
               const void* __restrict__ Vp, const double* __restrict__ b, void* W, double* partials,
               unsigned* ticket, double* nrm2) {
  using T = VT<DT>;
  using R_ = typename T::R;
  const size_t total = n * size_t(R);
  const size_t g0 = size_t(blockIdx.x) * kBT + threadIdx.x;
  const int c = int(g0 % size_t(R));
  const double ar = V ? a[2 * c] : 0.0, ai = V ? a[2 * c + 1] : 0.0;
  const double br = Vp ? b[c] : 0.0;
  double acc = 0.0;
  for (size_t f = g0; f < total; f += size_t(gridDim.x) * kBT) {
    R_ wr, wi;
    T::ld_plain(W, f, wr, wi);
    double xr = wr, xi = wi;
    if (V) {
      R_ vr, vi;
      T::ld(V, f, vr, vi);
      xr -= ar * double(vr) - ai * double(vi);
      xi -= ar * double(vi) + ai * double(vr);
    }
    if (Vp) {
      R_ pr, pi;
      T::ld(Vp, f, pr, pi);
      xr -= br * double(pr);
      xi -= br * double(pi);
    }
    const R_ sr = R_(xr), si = R_(xi);
    if (V || Vp) T::st(W, f, sr, si);
    acc += double(sr) * double(sr) + double(si) * double(si);
  }
  // column sums: threads t, t + R, t + 2R, ... of the block share a column
  __shared__ double red[kBT];
  red[threadIdx.x] = acc;
  __syncthreads();
  const int cb = int((size_t(blockIdx.x) * kBT) % size_t(R));  // column of thread 0
  for (int j = threadIdx.x; j < R; j += kBT) {
    double sum = 0.0;
    // thread t holds column (cb + t) % R
    const int t0 = (j - cb + R) % R;
    for (int t = t0; t < kBT; t += R) sum += red[t];
    partials[(size_t(j) * gridDim.x + blockIdx.x) * 2] = sum;
    partials[(size_t(j) * gridDim.x + blockIdx.x) * 2 + 1] = 0.0;
  }
  grid_finish(partials, ticket, R, nrm2);
}

template <int DT>
__global__ void k_block_scale(size_t n, int R, const double* __restrict__ nrm2, void* W, double* beta_out,
                              int* len, int step) {
  using T = VT<DT>;
  using R_ = typename T::R;
  const size_t total = n * size_t(R);
  for (size_t f = size_t(blockIdx.x) * blockDim.x + threadIdx.x; f < total; f += size_t(gridDim.x) * blockDim.x) {
    const int c = int(f % size_t(R));
    const double beta = sqrt(nrm2[2 * c]);
    const double sc = beta < 1e-15 ? 0.0 : 1.0 / beta;
    R_ wr, wi;
    T::ld_plain(W, f, wr, wi);
    T::st(W, f, R_(double(wr) * sc), R_(double(wi) * sc));
    if (f < size_t(R)) {
      beta_out[c] = beta;
      if (beta < 1e-15 && len[c] > step + 1) len[c] = step + 1;
    }
  }
}

template <int DT>
__global__ void k_block_column(size_t n, int R, const void* __restrict__ X, int c, void* out) {
  using T = VT<DT>;
  using R_ = typename T::R;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
    R_ re, im;
    T::ld(X, i * size_t(R) + c, re, im);
    T::st(out, i, re, im);
  }
}

}  // namespace
}  // namespace qkd

using namespace qkd;

extern "C" {

int qkd_block_update(qk_workspace* w, qk_dtype t, size_t n, int R, const void* V, const double* a, const void* Vp,
                     const double* b, void* W, double* nrm2, cudaStream_t s) {
  if (!w || !W || !nrm2 || R <= 0 || R > kMaxK || kBT % R != 0 || (V && !a) || (Vp && !b)) return QKD_EINVAL;
  if (n == 0) return QKD_OK;
  QKD_DISPATCH(t, k_block_update<DT><<<block_grid(n * size_t(R)), kBT, 0, s>>>(n, R, V, a, Vp, b, W, w->partials,
                                                                               w->ticket, nrm2));
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

int qkd_block_scale(qk_dtype t, size_t n, int R, const double* nrm2, void* W, double* beta_out, int* len, int step,
                    cudaStream_t s) {
  if (!nrm2 || !W || !beta_out || !len || R <= 0) return QKD_EINVAL;
  if (n == 0) return QKD_OK;
  QKD_DISPATCH(t, k_block_scale<DT><<<block_grid(n * size_t(R)), kBT, 0, s>>>(n, R, nrm2, W, beta_out, len, step));
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

int qkd_block_column(qk_dtype t, size_t n, int R, const void* X, int c, void* out, cudaStream_t s) {
  if (!X || !out || R <= 0 || c < 0 || c >= R) return QKD_EINVAL;
  if (n == 0) return QKD_OK;
  QKD_DISPATCH(t, k_block_column<DT><<<block_grid(n), kBT, 0, s>>>(n, R, X, c, out));
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

}  // extern "C"
