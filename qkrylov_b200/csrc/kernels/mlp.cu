// Kernels of the learned warm start: a 25 -> 128 -> 128 -> 2 MLP (GELU)
// over spin configurations, BF16 weights with FP32 accumulation, and its
// training (forward, loss, backward, Adam) on minibatches sampled from
// ground states by |psi|^2.
//
// Layout: activations row-major [batch][features] in FP32; weights row-major
// [out][in] (BF16 for the products, FP32 master copy for the optimizer).
// The products go through one tiled GEMM kernel, C = A op(B) (+ bias,
// + GELU), with 64x64 output tiles, 16-wide K slices in shared memory and a
// 4x4 register block per thread; every reduction is over a fixed order, so
// results are deterministic.
#include <cuda_bf16.h>

#include <algorithm>

#include "reduce.cuh"

namespace qkd {
namespace {

constexpr int kGT = 64, kGK = 16;  // GEMM tile and K slice

template <class T> __device__ __forceinline__ float tof(T v);
template <> __device__ __forceinline__ float tof<float>(float v) { return v; }
template <> __device__ __forceinline__ float tof<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }

// The network's activation: the tanh form of GELU (Hendrycks & Gimpel,
// "Gaussian Error Linear Units", 2016), 0.5 z (1 + tanh(c (z + k z^3)))
// with c = sqrt(2/pi), k = 0.044715, and its derivative.  Training uses the
// accurate tanhf; the tensor-core inference kernel uses the hardware
// approximation, whose error is below the BF16 rounding of its activations.
constexpr float kGeluC = 0.79788456080286536f, kGeluK = 0.044715f;
__device__ __forceinline__ float gelu(float z) {
  return 0.5f * z * (1.f + tanhf(kGeluC * z * fmaf(kGeluK * z, z, 1.f)));
}
__device__ __forceinline__ float gelu_d(float z) {
  const float t = tanhf(kGeluC * z * fmaf(kGeluK * z, z, 1.f));
  return 0.5f * (1.f + t) + 0.5f * z * (1.f - t * t) * kGeluC * fmaf(3.f * kGeluK * z, z, 1.f);
}

// C[M][N] = sum_k A[m][k] * B'(k, n) (+ bias[n]); B'(k, n) = B[n*ldb + k]
// when TB (B stored [N][K], the weight layout) else B[k*ldb + n].
// A(m, k) = A[m*lda + k] when !TA else A[k*lda + m].  Epilogue 1: store Z
// and GELU(Z) (Zout may be null); 0: store C.
template <class TAe, class TBe, bool TA, bool TB>
__global__ void __launch_bounds__(256)
k_gemm(int M, int N, int K, const TAe* __restrict__ A, int lda, const TBe* __restrict__ B, int ldb,
       const float* __restrict__ bias, float* __restrict__ C, int ldc, float* __restrict__ Zout, int gelu_ep) {
  __shared__ float sa[kGK][kGT + 1], sb[kGK][kGT + 1];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int m0 = blockIdx.y * kGT, n0 = blockIdx.x * kGT;
  float acc[4][4] = {};
  for (int k0 = 0; k0 < K; k0 += kGK) {
    for (int i = threadIdx.x; i < kGK * kGT; i += 256) {
      const int kk = i % kGK, mm = i / kGK;
      const int m = m0 + mm, k = k0 + kk;
      sa[kk][mm] = (m < M && k < K) ? tof(TA ? A[size_t(k) * lda + m] : A[size_t(m) * lda + k]) : 0.f;
      const int n = n0 + mm;
      sb[kk][mm] = (n < N && k < K) ? tof(TB ? B[size_t(n) * ldb + k] : B[size_t(k) * ldb + n]) : 0.f;
    }
    __syncthreads();
    #pragma unroll
    for (int kk = 0; kk < kGK; ++kk) {
      float a[4], b[4];
      #pragma unroll
      for (int i = 0; i < 4; ++i) { a[i] = sa[kk][ty + 16 * i]; b[i] = sb[kk][tx + 16 * i]; }
      #pragma unroll
      for (int i = 0; i < 4; ++i)
        #pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
  #pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + ty + 16 * i;
    if (m >= M) continue;
    #pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int n = n0 + tx + 16 * j;
      if (n >= N) continue;
      float z = acc[i][j] + (bias ? bias[n] : 0.f);
      if (gelu_ep) {
        if (Zout) Zout[size_t(m) * ldc + n] = z;
        z = gelu(z);
      }
      C[size_t(m) * ldc + n] = z;
    }
  }
}

// Input features of each sample: 24 spins as +-1 (bit set = up = +1) and
// the coupling J2; idx selects basis states (null: states 0..n-1).
__global__ void k_inputs(int n, int nsites, const uint64_t* __restrict__ states, const uint32_t* __restrict__ idx,
                         const float* __restrict__ j2, float j2_all, float* X, int ldx) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint64_t s = states[idx ? idx[i] : uint32_t(i)];
    float* x = X + size_t(i) * ldx;
    for (int b = 0; b < nsites; ++b) x[b] = ((s >> b) & 1ull) ? 1.f : -1.f;
    x[nsites] = j2 ? j2[i] : j2_all;
  }
}

// dZ = dH * GELU'(Z), elementwise
__global__ void k_gelu_bwd(size_t n, const float* __restrict__ dH, const float* __restrict__ Z, float* dZ) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    dZ[i] = dH[i] * gelu_d(Z[i]);
}

// db[j] = sum_i D[i][j]: one block per column, fixed order
__global__ void k_colsum(int M, int N, const float* __restrict__ D, float* db) {
  __shared__ float red[256];
  const int j = blockIdx.x;
  float s = 0.f;
  for (int i = threadIdx.x; i < M; i += 256) s += D[size_t(i) * N + j];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) db[j] = red[0];
}

// Loss per sample i with output o = (o0, o1), target log-amplitude a_i,
// residual sign y_i = +-1 and weight w_i:
//   l_i = w_i [ (o0 - a_i)^2 + c_sign softplus(-y_i o1) ]
// dO = dl/do / n; loss partials per block (FP64) summed in block order.
__global__ void k_loss(int n, const float* __restrict__ O, const float* __restrict__ tgt, float c_sign, float* dO,
                       double* partials, unsigned* ticket, double* loss) {
  double acc = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float o0 = O[2 * i], o1 = O[2 * i + 1];
    const float a = tgt[3 * i], y = tgt[3 * i + 1], w = tgt[3 * i + 2];
    const float e = o0 - a, m = -y * o1;
    const float sp = m > 20.f ? m : log1pf(expf(m));
    const float sg = 1.f / (1.f + expf(-m));  // d softplus(m)/dm
    acc += double(w) * (double(e) * e + double(c_sign) * sp);
    dO[2 * i] = w * 2.f * e / n;
    dO[2 * i + 1] = w * c_sign * sg * (-y) / n;
  }
  double im = 0.0;
  __shared__ double sbuf[16];
  block_sum2(acc, im, sbuf);
  if (threadIdx.x == 0) { partials[2 * blockIdx.x] = acc / n; partials[2 * blockIdx.x + 1] = 0.0; }
  grid_finish(partials, ticket, 1, loss);
}

// Adam on the FP32 master parameters, BF16 copy of the weights refreshed.
__global__ void k_adam(size_t n, float* p, const float* __restrict__ g, float* m, float* v, float lr, float b1,
                       float b2, float c1, float c2, float eps, __nv_bfloat16* pb, size_t nw) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi; v[i] = vi;
    const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] = pi;
    if (i < nw) pb[i] = __float2bfloat16(pi);
  }
}

__global__ void k_tobf16(size_t n, const float* __restrict__ p, __nv_bfloat16* pb) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    pb[i] = __float2bfloat16(p[i]);
}

// Start vector from the outputs: phi_i = M(s_i) exp(o0_i - shift) tanh(o1_i),
// M(s) = (-1)^popcount(s & marshall) the fixed sign prior.
__global__ void k_startvec(int n, const uint64_t* __restrict__ states, uint64_t marshall, const float* __restrict__ O,
                           float shift, float* out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float m = (__popcll(states[i] & marshall) & 1) ? -1.f : 1.f;
    out[i] = m * expf(O[2 * i] - shift) * tanhf(O[2 * i + 1]);
  }
}

// Inclusive prefix sums of |psi|^2 (FP64) in chunks: per-block scan, then
// block offsets added by a second pass (offsets scanned by one block).
template <class VTp>
__global__ void k_scan1(size_t n, const VTp* __restrict__ psi, double* cdf, double* bsum) {
  __shared__ double s[1024];
  const size_t i = blockIdx.x * size_t(1024) + threadIdx.x;
  const double v = i < n ? double(psi[i]) * double(psi[i]) : 0.0;
  s[threadIdx.x] = v;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    const double t = threadIdx.x >= off ? s[threadIdx.x - off] : 0.0;
    __syncthreads();
    s[threadIdx.x] += t;
    __syncthreads();
  }
  if (i < n) cdf[i] = s[threadIdx.x];
  if (threadIdx.x == 1023) bsum[blockIdx.x] = s[1023];
}

__global__ void k_scan_offsets(int nb, double* bsum) {  // one thread: exclusive scan of block sums
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double run = 0.0;
    for (int b = 0; b < nb; ++b) { const double t = bsum[b]; bsum[b] = run; run += t; }
    bsum[nb] = run;
  }
}

__global__ void k_scan2(size_t n, double* cdf, const double* __restrict__ bsum) {
  const size_t i = blockIdx.x * size_t(1024) + threadIdx.x;
  if (i < n) cdf[i] += bsum[blockIdx.x];
}

__device__ __forceinline__ uint64_t smix(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Draw m indices with probability |psi_i|^2 / sum (inverse CDF, binary
// search) and write (log|psi_i| - log_max, residual sign, 1) targets.
template <class VTp>
__global__ void k_sample(int m, size_t n, const double* __restrict__ cdf, const VTp* __restrict__ psi,
                         const uint64_t* __restrict__ states, uint64_t marshall, double log_max, uint64_t seed,
                         uint32_t* idx, float* tgt) {
  const double total = cdf[n - 1];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
    const double u = (double(smix(seed * 0x632BE59BD9B4E019ull + k) >> 11) + 0.5) * (1.0 / 9007199254740992.0) * total;
    size_t lo = 0, hi = n - 1;
    while (lo < hi) {  // first i with cdf[i] >= u
      const size_t mid = (lo + hi) / 2;
      if (cdf[mid] < u) lo = mid + 1; else hi = mid;
    }
    idx[k] = uint32_t(lo);
    const double p = double(psi[lo]);
    const double ms = (__popcll(states[lo] & marshall) & 1) ? -1.0 : 1.0;
    tgt[3 * k] = float(log(fabs(p) + 1e-300) - log_max);
    tgt[3 * k + 1] = (p * ms >= 0.0) ? 1.f : -1.f;
    tgt[3 * k + 2] = 1.f;
  }
}

// out[0] = max_i x[i * stride]; float bits compared as ordered integers
__global__ void k_max_f32(size_t n, const float* __restrict__ x, int stride, float* partials, unsigned* ticket,
                          float* out) {
  float m = -INFINITY;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    m = fmaxf(m, x[i * stride]);
  __shared__ float red[256];
  red[threadIdx.x] = m;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] = fmaxf(red[threadIdx.x], red[threadIdx.x + w]);
    __syncthreads();
  }
  __shared__ unsigned s_ticket;
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = red[0];
    __threadfence();
    s_ticket = atomicAdd(ticket, 1u);
  }
  __syncthreads();
  if (s_ticket != gridDim.x - 1 || threadIdx.x != 0) return;
  __threadfence();
  float r = -INFINITY;
  for (unsigned b = 0; b < gridDim.x; ++b) r = fmaxf(r, __ldcg(partials + b));
  *out = r;
  *ticket = 0u;
}

inline unsigned grid_for(size_t n, int t = 256) {
  return unsigned(std::max<size_t>(1, std::min<size_t>((n + t - 1) / t, 4096)));
}

}  // namespace
}  // namespace qkd

using namespace qkd;

extern "C" {

int qkd_mlp_gemm(int M, int N, int K, int a_bf16, const void* A, int lda, int trans_a, int b_bf16, const void* B,
                 int ldb, int trans_b, const float* bias, float* C, int ldc, float* Z, int gelu_ep, cudaStream_t s) {
  if (M <= 0 || N <= 0 || K <= 0 || !A || !B || !C || (gelu_ep && false)) return M == 0 || N == 0 ? QKD_OK : QKD_EINVAL;
  const dim3 grid((N + kGT - 1) / kGT, (M + kGT - 1) / kGT);
#define QKD_G(TA_, TB_, tA, tB) \
  k_gemm<TA_, TB_, tA, tB><<<grid, 256, 0, s>>>(M, N, K, static_cast<const TA_*>(A), lda, static_cast<const TB_*>(B), \
                                                ldb, bias, C, ldc, Z, gelu_ep)
  if (!a_bf16 && b_bf16) {
    if (!trans_a && trans_b) QKD_G(float, __nv_bfloat16, false, true);
    else if (!trans_a && !trans_b) QKD_G(float, __nv_bfloat16, false, false);
    else return QKD_EINVAL;
  } else if (!a_bf16 && !b_bf16) {
    if (trans_a && !trans_b) QKD_G(float, float, true, false);
    else if (!trans_a && trans_b) QKD_G(float, float, false, true);
    else if (!trans_a && !trans_b) QKD_G(float, float, false, false);
    else QKD_G(float, float, true, true);
  } else {
    return QKD_EINVAL;
  }
#undef QKD_G
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

int qkd_mlp_inputs(int n, int nsites, const uint64_t* states, const uint32_t* idx, const float* j2, float j2_all,
                   float* X, int ldx, cudaStream_t s) {
  if (n <= 0) return QKD_OK;
  if (!states || !X || nsites < 1 || ldx < nsites + 1) return QKD_EINVAL;
  k_inputs<<<grid_for(n), 256, 0, s>>>(n, nsites, states, idx, j2, j2_all, X, ldx);
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

int qkd_mlp_gelu_bwd(size_t n, const float* dH, const float* Z, float* dZ, cudaStream_t s) {
  if (n == 0) return QKD_OK;
  k_gelu_bwd<<<grid_for(n), 256, 0, s>>>(n, dH, Z, dZ);
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

int qkd_mlp_colsum(int M, int N, const float* D, float* db, cudaStream_t s) {
  if (N <= 0) return QKD_OK;
  k_colsum<<<N, 256, 0, s>>>(M, N, D, db);
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

int qkd_mlp_loss(qk_workspace* w, int n, const float* O, const float* tgt, float c_sign, float* dO, double* loss,
                 cudaStream_t s) {
  if (!w || n <= 0) return QKD_EINVAL;
  const unsigned g = std::min<unsigned>(grid_for(n), kMaxG);
  k_loss<<<g, 256, 0, s>>>(n, O, tgt, c_sign, dO, w->partials, w->ticket, loss);
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

int qkd_mlp_adam(size_t n, float* p, const float* g, float* m, float* v, float lr, float b1, float b2, int t,
                 float eps, void* pb, size_t nw, cudaStream_t s) {
  if (n == 0) return QKD_OK;
  const float c1 = 1.f - powf(b1, float(t)), c2 = 1.f - powf(b2, float(t));
  k_adam<<<grid_for(n), 256, 0, s>>>(n, p, g, m, v, lr, b1, b2, c1, c2, eps, static_cast<__nv_bfloat16*>(pb), nw);
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

int qkd_mlp_tobf16(size_t n, const float* p, void* pb, cudaStream_t s) {
  if (n == 0) return QKD_OK;
  k_tobf16<<<grid_for(n), 256, 0, s>>>(n, p, static_cast<__nv_bfloat16*>(pb));
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

int qkd_max_f32(qk_workspace* w, size_t n, const float* x, int stride, float* out, cudaStream_t s) {
  if (!w || !x || !out || n == 0 || stride < 1) return QKD_EINVAL;
  const unsigned g = std::min<unsigned>(grid_for(n), kMaxG);
  k_max_f32<<<g, 256, 0, s>>>(n, x, stride, reinterpret_cast<float*>(w->partials), w->ticket, out);
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

int qkd_mlp_startvec(int n, const uint64_t* states, uint64_t marshall, const float* O, float shift, float* out,
                     cudaStream_t s) {
  if (n <= 0) return QKD_OK;
  k_startvec<<<grid_for(n), 256, 0, s>>>(n, states, marshall, O, shift, out);
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

int qkd_cdf(qk_dtype t, size_t n, const void* psi, double* cdf, double* bsum, cudaStream_t s) {
  if (n == 0) return QKD_OK;
  if (t != QK_F64 && t != QK_F32) return QKD_EINVAL;
  const unsigned nb = unsigned((n + 1023) / 1024);
  if (t == QK_F64) k_scan1<double><<<nb, 1024, 0, s>>>(n, static_cast<const double*>(psi), cdf, bsum);
  else k_scan1<float><<<nb, 1024, 0, s>>>(n, static_cast<const float*>(psi), cdf, bsum);
  k_scan_offsets<<<1, 32, 0, s>>>(int(nb), bsum);
  k_scan2<<<nb, 1024, 0, s>>>(n, cdf, bsum);
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

int qkd_sample(qk_dtype t, int m, size_t n, const double* cdf, const void* psi, const uint64_t* states,
               uint64_t marshall, double log_max, uint64_t seed, uint32_t* idx, float* tgt, cudaStream_t s) {
  if (m <= 0) return QKD_OK;
  if (n == 0 || (t != QK_F64 && t != QK_F32)) return QKD_EINVAL;
  if (t == QK_F64)
    k_sample<double><<<grid_for(m), 256, 0, s>>>(m, n, cdf, static_cast<const double*>(psi), states, marshall,
                                                 log_max, seed, idx, tgt);
  else
    k_sample<float><<<grid_for(m), 256, 0, s>>>(m, n, cdf, static_cast<const float*>(psi), states, marshall, log_max,
                                                seed, idx, tgt);
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

}  // extern "C"
