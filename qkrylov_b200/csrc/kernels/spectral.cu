// Spectral functions of many continued fractions on many frequencies at once.
//
// The reference evaluates one frequency per call on the host
// (src/solvers/dynamics.cpp:61-89): z = omega + E0 + i eta,
// f = 1 / (z - a_{n-1}), then f = 1 / (z - a_i - b_i^2 f) down to i = 0,
// S = -(1/pi) Im(|phi0|^2 f).  Here one thread evaluates one (fraction,
// frequency) pair with the same backward recurrence in FP64; the complex
// reciprocal uses Smith's scaling (R. L. Smith, "Algorithm 116: Complex
// division", CACM 5 (1962) 435) so no intermediate overflows.  The
// coefficients of a fraction are read by all threads of a warp at the same
// index (one broadcast load), so the kernel runs at the issue rate.
#include "common.cuh"

namespace qkd {
namespace {

__device__ __forceinline__ void crecip(double a, double b, double& re, double& im) {
  // 1 / (a + i b)
  if (fabs(a) >= fabs(b)) {
    const double r = b / a, d = a + b * r;
    re = 1.0 / d;
    im = -r / d;
  } else {
    const double r = a / b, d = b + a * r;
    re = r / d;
    im = -1.0 / d;
  }
}

// grid: x over frequencies, y over fractions
__global__ void __launch_bounds__(256) k_spectral(const double* __restrict__ alphas, const double* __restrict__ betas,
                                                  const int* __restrict__ len, int ld,
                                                  const double* __restrict__ nrm, const double* __restrict__ omega,
                                                  uint32_t nw, double E0, double eta, double* __restrict__ out) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (k >= nw) return;
  const int n = len ? len[c] : ld;
  double s = 0.0;
  if (n > 0) {
    const double* a = alphas + size_t(c) * ld;
    const double* b = betas + size_t(c) * ld;
    const double zr = omega[k] + E0, zi = eta;
    double fr, fi;
    crecip(zr - a[n - 1], zi, fr, fi);
    for (int i = n - 2; i >= 0; --i) {
      const double b2 = b[i] * b[i];
      crecip(zr - a[i] - b2 * fr, zi - b2 * fi, fr, fi);
    }
    const double w = nrm ? nrm[c] : 1.0;
    s = -(w * w * fi) / 3.14159265358979323846;
  }
  out[size_t(c) * nw + k] = s;
}

}  // namespace
}  // namespace qkd

extern "C" int qkd_spectral_batch(const double* alphas, const double* betas, const int* len, int ncols, int ld,
                                  const double* nrm, const double* omega, size_t nw, double E0, double eta,
                                  double* out, cudaStream_t s) {
  if (ncols <= 0 || nw == 0) return QKD_OK;
  if (!alphas || !betas || !omega || !out || ld < 0 || ncols > 65535 || nw > (size_t(1) << 31)) return QKD_EINVAL;
  const dim3 grid(unsigned((nw + 255) / 256), unsigned(ncols));
  qkd::k_spectral<<<grid, 256, 0, s>>>(alphas, betas, len, ld, nrm, omega, uint32_t(nw), E0, eta, out);
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}
