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

// The block size (256) and the grid stride are multiples of R, so each
// thread keeps one column and computes its scale once.
template <int DT>
__global__ void __launch_bounds__(kBT)
k_block_scale(size_t n, int R, const double* __restrict__ nrm2, void* W, double* beta_out, int* len, int step) {
  using T = VT<DT>;
  using R_ = typename T::R;
  const size_t total = n * size_t(R);
  const size_t g0 = size_t(blockIdx.x) * kBT + threadIdx.x;
  const int c = int(threadIdx.x) % R;
  const double beta = sqrt(nrm2[2 * c]);
  const double sc = beta < 1e-15 ? 0.0 : 1.0 / beta;
  if (g0 < size_t(R)) {
    beta_out[c] = beta;
    if (beta < 1e-15 && len[c] > step + 1) len[c] = step + 1;
  }
  for (size_t f = g0; f < total; f += size_t(gridDim.x) * kBT) {
    R_ wr, wi;
    T::ld_plain(W, f, wr, wi);
    T::st(W, f, R_(double(wr) * sc), R_(double(wi) * sc));
  }
}

// 16-byte packs of consecutive columns of one row.
template <int DT> struct BPk;
template <> struct BPk<QK_C128> {
  using V = double2; static constexpr int W = 1;
  __device__ static void un(const V& v, double* re, double* im) { re[0] = v.x; im[0] = v.y; }
  __device__ static V pk(const double* re, const double* im) { return make_double2(re[0], im[0]); }
};
template <> struct BPk<QK_C64> {
  using V = float4; static constexpr int W = 2;
  __device__ static void un(const V& v, double* re, double* im) { re[0] = v.x; im[0] = v.y; re[1] = v.z; im[1] = v.w; }
  __device__ static V pk(const double* re, const double* im) {
    return make_float4(float(re[0]), float(im[0]), float(re[1]), float(im[1]));
  }
};
template <> struct BPk<QK_F64> {
  using V = double2; static constexpr int W = 2;
  __device__ static void un(const V& v, double* re, double* im) { re[0] = v.x; re[1] = v.y; im[0] = im[1] = 0.0; }
  __device__ static V pk(const double* re, const double*) { return make_double2(re[0], re[1]); }
};
template <> struct BPk<QK_F32> {
  using V = float4; static constexpr int W = 4;
  __device__ static void un(const V& v, double* re, double* im) {
    re[0] = v.x; re[1] = v.y; re[2] = v.z; re[3] = v.w; im[0] = im[1] = im[2] = im[3] = 0.0;
  }
  __device__ static V pk(const double* re, const double*) {
    return make_float4(float(re[0]), float(re[1]), float(re[2]), float(re[3]));
  }
};

// One Lanczos step of R recurrences on unnormalised vectors (v_k = s_k U_k),
// 16-byte packs; the grid stride in elements is a multiple of R, so each
// thread keeps the same W columns and reads their coefficients once.  The
// last block to finish turns the column norms into beta, s_{k+1} and the
// breakdown lengths.
template <int DT>
__global__ void __launch_bounds__(kBT)
k_block_lanczos(size_t n, int R, const void* __restrict__ Uk, const void* __restrict__ Ukm1,
                const double* __restrict__ dots, const double* __restrict__ beta_prev,
                const double* __restrict__ s_prev, const double* __restrict__ s_k, double* s_next, void* Y,
                double* alpha_out, double* beta_out, int* len, int step, double* partials, unsigned* ticket) {
  using P = BPk<DT>;
  using PV = typename P::V;
  constexpr int W = P::W;
  const size_t nq = n * size_t(R) / W;
  const size_t g = size_t(blockIdx.x) * kBT + threadIdx.x;
  const int c0 = int((g * W) % size_t(R));
  double cy[W], cu[W], cp[W];
  #pragma unroll
  for (int w = 0; w < W; ++w) {
    const int c = c0 + w;
    const double sk = s_k[c];
    cy[w] = sk;
    cu[w] = sk * sk * dots[2 * c] * sk;
    cp[w] = Ukm1 ? beta_prev[c] * s_prev[c] : 0.0;
  }
  double acc[W];
  #pragma unroll
  for (int w = 0; w < W; ++w) acc[w] = 0.0;
  for (size_t q = g; q < nq; q += size_t(gridDim.x) * kBT) {
    double yr[W], yi[W], ur[W], ui[W];
    P::un(reinterpret_cast<const PV*>(Y)[q], yr, yi);
    P::un(__ldg(reinterpret_cast<const PV*>(Uk) + q), ur, ui);
    #pragma unroll
    for (int w = 0; w < W; ++w) { yr[w] = cy[w] * yr[w] - cu[w] * ur[w]; yi[w] = cy[w] * yi[w] - cu[w] * ui[w]; }
    if (Ukm1) {
      P::un(__ldg(reinterpret_cast<const PV*>(Ukm1) + q), ur, ui);
      #pragma unroll
      for (int w = 0; w < W; ++w) { yr[w] -= cp[w] * ur[w]; yi[w] -= cp[w] * ui[w]; }
    }
    const PV o = P::pk(yr, yi);
    reinterpret_cast<PV*>(Y)[q] = o;
    P::un(o, yr, yi);
    #pragma unroll
    for (int w = 0; w < W; ++w) acc[w] += yr[w] * yr[w] + yi[w] * yi[w];
  }
  // per-column block sums: slot t*W + w holds column (t*W + w) % R
  __shared__ double red[kBT * W];
  #pragma unroll
  for (int w = 0; w < W; ++w) red[threadIdx.x * W + w] = acc[w];
  __syncthreads();
  for (int j = threadIdx.x; j < R; j += kBT) {
    double sum = 0.0;
    for (int i = j; i < kBT * W; i += R) sum += red[i];
    partials[size_t(j) * gridDim.x + blockIdx.x] = sum;
  }
  __shared__ unsigned s_ticket;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_ticket = atomicAdd(ticket, 1u);
  __syncthreads();
  if (s_ticket != gridDim.x - 1) return;
  __threadfence();
  for (int j = threadIdx.x; j < R; j += kBT) {
    double nrm = 0.0;
    for (unsigned b = 0; b < gridDim.x; ++b) nrm += __ldcg(partials + size_t(j) * gridDim.x + b);
    const double beta = sqrt(nrm), sk = s_k[j];
    alpha_out[j] = sk * sk * dots[2 * j];
    beta_out[j] = beta;
    s_next[j] = beta < 1e-15 ? 0.0 : 1.0 / beta;
    if (beta < 1e-15 && len[j] > step + 1) len[j] = step + 1;
  }
  if (threadIdx.x == 0) *ticket = 0u;
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

// Column-wise kernels of the batched coupling sweep (real vectors, element
// type E): every thread keeps one column c = threadIdx.x % R, because the
// block size and the grid stride are multiples of R.  Column sums go to
// per-CTA partials partials[o * G + b] and a second launch reduces them in a
// fixed order (deterministic results).
constexpr int kSweepJ = 16;      // blocks combined per pass over the rows
constexpr int kSweepMaxV = 192;  // blocks per call

// sum over the threads of this CTA that hold column threadIdx.x % R,
// written by the first R threads to partials[o * G + blockIdx.x]
__device__ __forceinline__ void column_partial(double v, int R, size_t o_base, double* red, double* partials) {
  red[threadIdx.x] = v;
  __syncthreads();
  if (threadIdx.x < unsigned(R)) {
    double s = 0.0;
    for (int t = threadIdx.x; t < kBT; t += R) s += red[t];
    partials[(o_base + threadIdx.x) * gridDim.x + blockIdx.x] = s;
  }
  __syncthreads();
}

// out[2 (j R + c)] = <V_j[:, c], W[:, c]> for j < nv (partials only; see k_sweep_reduce)
template <class E>
__global__ void __launch_bounds__(kBT)
k_block_mdot(size_t n, int R, int nv, const void* const* __restrict__ V, const E* __restrict__ W,
             double* __restrict__ partials) {
  __shared__ const E* sV[kSweepMaxV];
  __shared__ double red[kBT];
  for (int j = threadIdx.x; j < nv; j += kBT) sV[j] = static_cast<const E*>(V[j]);
  __syncthreads();
  const size_t total = n * size_t(R), stride = size_t(gridDim.x) * kBT;
  const size_t g0 = size_t(blockIdx.x) * kBT + threadIdx.x;
  for (int j0 = 0; j0 < nv; j0 += kSweepJ) {
    double acc[kSweepJ];
    #pragma unroll
    for (int u = 0; u < kSweepJ; ++u) acc[u] = 0.0;
    for (size_t f = g0; f < total; f += stride) {
      const double w = double(W[f]);
      #pragma unroll
      for (int u = 0; u < kSweepJ; ++u)
        if (j0 + u < nv) acc[u] += double(__ldg(sV[j0 + u] + f)) * w;
    }
    #pragma unroll
    for (int u = 0; u < kSweepJ; ++u)  // the condition is the same for the whole CTA
      if (j0 + u < nv) column_partial(acc[u], R, size_t(j0 + u) * R, red, partials);
  }
}

// W[:, c] = (keep ? W[:, c] : 0) - sum_j coef[2 (j R + c)] V_j[:, c], in j
// order; partials of |W[:, c]|^2 (after rounding to E) when partials != NULL
template <class E>
__global__ void __launch_bounds__(kBT)
k_block_mcomb(size_t n, int R, int nv, const void* const* __restrict__ V, const double* __restrict__ coef, int keep,
              E* W, double* __restrict__ partials) {
  __shared__ const E* sV[kSweepMaxV];
  __shared__ double red[kBT];
  for (int j = threadIdx.x; j < nv; j += kBT) sV[j] = static_cast<const E*>(V[j]);
  __syncthreads();
  const size_t total = n * size_t(R), stride = size_t(gridDim.x) * kBT;
  const size_t g0 = size_t(blockIdx.x) * kBT + threadIdx.x;
  const int c = int(threadIdx.x) % R;
  double acc = 0.0;
  for (int j0 = 0; j0 < nv; j0 += kSweepJ) {
    double cf[kSweepJ];
    #pragma unroll
    for (int u = 0; u < kSweepJ; ++u) cf[u] = j0 + u < nv ? coef[2 * (size_t(j0 + u) * R + c)] : 0.0;
    const bool zero = j0 == 0 && !keep, last = j0 + kSweepJ >= nv;
    for (size_t f = g0; f < total; f += stride) {
      double x = zero ? 0.0 : double(W[f]);
      #pragma unroll
      for (int u = 0; u < kSweepJ; ++u)
        if (j0 + u < nv) x -= cf[u] * double(__ldg(sV[j0 + u] + f));
      const E xe = E(x);
      W[f] = xe;
      if (last) acc += double(xe) * double(xe);
    }
  }
  if (partials) column_partial(acc, R, 0, red, partials);
}

// Y0[:, c] += g[c] Y1[:, c]; partials of <X[:, c], Y0[:, c]>
template <class E>
__global__ void __launch_bounds__(kBT)
k_block_axpy_cols(size_t n, int R, const double* __restrict__ g, const E* __restrict__ Y1, E* Y0,
                  const E* __restrict__ X, double* __restrict__ partials) {
  __shared__ double red[kBT];
  const size_t total = n * size_t(R), stride = size_t(gridDim.x) * kBT;
  const double gc = g[int(threadIdx.x) % R];
  double acc = 0.0;
  for (size_t f = size_t(blockIdx.x) * kBT + threadIdx.x; f < total; f += stride) {
    const E y = E(double(Y0[f]) + gc * double(Y1[f]));
    Y0[f] = y;
    acc += double(X[f]) * double(y);
  }
  column_partial(acc, R, 0, red, partials);
}

// column c of a row-interleaved block (element type Ed) from a vector of
// n elements (type Es)
template <class Es, class Ed>
__global__ void k_block_put_column(size_t n, int R, const Es* __restrict__ src, int c, Ed* dst) {
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    dst[i * size_t(R) + c] = Ed(src[i]);
}

// out[2 o] = sum_b partials[o * G + b] (lanes stride over b, then a warp
// sum), out[2 o + 1] = 0; one warp per output
__global__ void k_sweep_reduce(const double* __restrict__ partials, int G, int nout, double* out) {
  const int o = blockIdx.x * (kBT / 32) + int(threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (o >= nout) return;
  double s = 0.0;
  for (int b = lane; b < G; b += 32) s += partials[size_t(o) * G + b];
  s = warp_sum(s);
  if (lane == 0) { out[2 * o] = s; out[2 * o + 1] = 0.0; }
}

inline int sweep_finish(const double* partials, unsigned G, int nout, double* out, cudaStream_t s) {
  k_sweep_reduce<<<unsigned((nout + kBT / 32 - 1) / (kBT / 32)), kBT, 0, s>>>(partials, int(G), nout, out);
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

}  // namespace
}  // namespace qkd

using namespace qkd;

extern "C" {

int qkd_block_partials_grid(size_t n, int R) { return int(block_grid(n * size_t(R))); }

#define QKD_REAL_DISPATCH(t, ...)                          \
  do {                                                     \
    if ((t) == QK_F64) { using E = double; __VA_ARGS__; }  \
    else if ((t) == QK_F32) { using E = float; __VA_ARGS__; } \
    else return QKD_EINVAL;                                \
  } while (0)

int qkd_block_mdot(qk_dtype t, size_t n, int R, int nv, const void* const* V, const void* W, double* partials,
                   size_t partials_cap, double* out, cudaStream_t s) {
  if (!V || !W || !partials || !out || R <= 0 || kBT % R != 0 || nv < 1 || nv > kSweepMaxV) return QKD_EINVAL;
  if (n == 0) return QKD_OK;
  const unsigned G = block_grid(n * size_t(R));
  if (size_t(nv) * R * G > partials_cap) return QKD_EINVAL;
  QKD_REAL_DISPATCH(t, (k_block_mdot<E><<<G, kBT, 0, s>>>(n, R, nv, V, static_cast<const E*>(W), partials)));
  QKD_LAUNCH_CHECK();
  return sweep_finish(partials, G, nv * R, out, s);
}

int qkd_block_mcomb(qk_dtype t, size_t n, int R, int nv, const void* const* V, const double* coef, int keep, void* W,
                    double* partials, size_t partials_cap, double* nrm2, cudaStream_t s) {
  if (!V || !coef || !W || R <= 0 || kBT % R != 0 || nv < 1 || nv > kSweepMaxV || (nrm2 && !partials))
    return QKD_EINVAL;
  if (n == 0) return QKD_OK;
  const unsigned G = block_grid(n * size_t(R));
  if (nrm2 && size_t(R) * G > partials_cap) return QKD_EINVAL;
  QKD_REAL_DISPATCH(t, (k_block_mcomb<E><<<G, kBT, 0, s>>>(n, R, nv, V, coef, keep, static_cast<E*>(W),
                                                            nrm2 ? partials : nullptr)));
  QKD_LAUNCH_CHECK();
  return nrm2 ? sweep_finish(partials, G, R, nrm2, s) : QKD_OK;
}

int qkd_block_axpy_cols(qk_dtype t, size_t n, int R, const double* g, const void* Y1, void* Y0, const void* X,
                        double* partials, size_t partials_cap, double* dots, cudaStream_t s) {
  if (!g || !Y1 || !Y0 || !X || !partials || !dots || R <= 0 || kBT % R != 0) return QKD_EINVAL;
  if (n == 0) return QKD_OK;
  const unsigned G = block_grid(n * size_t(R));
  if (size_t(R) * G > partials_cap) return QKD_EINVAL;
  QKD_REAL_DISPATCH(t, (k_block_axpy_cols<E><<<G, kBT, 0, s>>>(n, R, g, static_cast<const E*>(Y1), static_cast<E*>(Y0),
                                                                static_cast<const E*>(X), partials)));
  QKD_LAUNCH_CHECK();
  return sweep_finish(partials, G, R, dots, s);
}

int qkd_block_put_column(qk_dtype ts, const void* src, size_t n, int R, int c, qk_dtype td, void* dst,
                         cudaStream_t s) {
  if (!src || !dst || R <= 0 || c < 0 || c >= R) return QKD_EINVAL;
  if (n == 0) return QKD_OK;
  const unsigned G = block_grid(n);
  if (ts == QK_F32 && td == QK_F64)
    k_block_put_column<float, double><<<G, kBT, 0, s>>>(n, R, static_cast<const float*>(src), c, static_cast<double*>(dst));
  else if (ts == QK_F64 && td == QK_F64)
    k_block_put_column<double, double><<<G, kBT, 0, s>>>(n, R, static_cast<const double*>(src), c, static_cast<double*>(dst));
  else if (ts == QK_F32 && td == QK_F32)
    k_block_put_column<float, float><<<G, kBT, 0, s>>>(n, R, static_cast<const float*>(src), c, static_cast<float*>(dst));
  else
    return QKD_EINVAL;
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

#undef QKD_REAL_DISPATCH

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
  if (!nrm2 || !W || !beta_out || !len || R <= 0 || kBT % R != 0) return QKD_EINVAL;
  if (n == 0) return QKD_OK;
  QKD_DISPATCH(t, k_block_scale<DT><<<block_grid(n * size_t(R)), kBT, 0, s>>>(n, R, nrm2, W, beta_out, len, step));
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

int qkd_block_lanczos(qk_workspace* w, qk_dtype t, size_t n, int R, const void* Uk, const void* Ukm1,
                      const double* dots, const double* beta_prev, const double* s_prev, const double* s_k,
                      double* s_next, void* Y, double* alpha_out, double* beta_out, int* len, int step,
                      cudaStream_t s) {
  if (!w || !Uk || !Y || !dots || !s_k || !s_next || !alpha_out || !beta_out || !len || R < 32 || R > kMaxK ||
      kBT % R != 0 || (Ukm1 && (!beta_prev || !s_prev)))
    return QKD_EINVAL;
  const uintptr_t al = reinterpret_cast<uintptr_t>(Uk) | reinterpret_cast<uintptr_t>(Y) |
                       reinterpret_cast<uintptr_t>(Ukm1);
  if (al & 15) return QKD_EINVAL;  // 16-byte packs
  if (n == 0) return QKD_OK;
  const unsigned G = block_grid(n * size_t(R) / 4);
  QKD_DISPATCH(t, k_block_lanczos<DT><<<G, kBT, 0, s>>>(n, R, Uk, Ukm1, dots, beta_prev, s_prev, s_k, s_next, Y,
                                                        alpha_out, beta_out, len, step, w->partials, w->ticket));
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
