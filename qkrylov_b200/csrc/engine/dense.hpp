// Small dense eigensolvers that run on the host, in the solver's precision.
//
// The Lanczos / FTLM convergence decisions compare successive Ritz values
// against a tolerance, so the tridiagonal eigensolver follows the same
// sweep sequence as the reference's (implicit-shift QL with the deflation
// test |e_i| < 1e-14 (|d_i| + |d_i+1|), at most 1000 sweeps;
// src/solvers/lanczos.cpp:25-98, src/solvers/ftlm.cpp:61-119), and the
// Davidson projection uses the same cyclic-by-largest Jacobi rotations
// (src/solvers/davidson.cpp:22-82).  Eigenvalues of the QL sweeps do not
// depend on whether eigenvectors are accumulated, so the per-iteration
// convergence check runs without them (O(n) per sweep instead of O(n^2)).
#pragma once

#include <algorithm>
#include <cmath>
#include <complex>
#include <numeric>
#include <vector>

namespace qkb {

// d <- eigenvalues of the n x n symmetric tridiagonal (alpha, beta); when z
// is given it receives the eigenvector matrix, z[j*n + i] = component j of
// eigenvector i, for the first zrows components (all n when zrows < 0).
// Each rotation acts on every row of z independently, so the first rows
// come out identical whether or not the others are accumulated.
template <class Real>
void tridiag_ql(const std::vector<Real>& alpha, const std::vector<Real>& beta, int n,
                std::vector<Real>& d, std::vector<Real>* z, int zrows = -1) {
  d.assign(alpha.begin(), alpha.begin() + n);
  std::vector<Real> e(beta.begin(), beta.begin() + std::min<size_t>(beta.size(), size_t(n)));
  e.resize(n, Real(0));
  const int zr = (zrows < 0 || zrows > n) ? n : zrows;
  if (z) {
    z->assign(size_t(zr) * n, Real(0));
    for (int i = 0; i < zr; ++i) (*z)[size_t(i) * n + i] = Real(1);
  }
  for (int iter = 0; iter < 1000; ++iter) {
    for (int i = 0; i < n - 1; ++i)
      if (std::abs(e[i]) < Real(1e-14) * (std::abs(d[i]) + std::abs(d[i + 1]))) e[i] = Real(0);
    int m = n - 1;
    while (m > 0 && e[m - 1] == Real(0)) m--;
    if (m == 0) break;
    int l = m - 1;
    while (l > 0 && e[l - 1] != Real(0)) l--;
    const Real b = (d[m - 1] - d[m]) / Real(2);
    const Real c = e[m - 1] * e[m - 1];
    const Real s = std::sqrt(b * b + c);
    const Real shift = (b > 0) ? d[m] - c / (b + s) : d[m] - c / (b - s);
    Real p = d[l] - shift, g = e[l];
    for (int i = l; i < m; ++i) {
      const Real r = std::hypot(p, g);
      const Real ct = p / r, st = g / r;
      if (i > l) e[i - 1] = r;
      const Real f = ct * d[i] + st * e[i];
      const Real gn = ct * e[i] + st * d[i + 1];
      const Real h = st * d[i] - ct * e[i];
      const Real k = st * e[i] - ct * d[i + 1];
      d[i] = ct * f + st * gn;
      e[i] = ct * h + st * k;
      d[i + 1] = st * h - ct * k;
      if (z) {
        Real* Z = z->data();
        for (int j = 0; j < zr; ++j) {
          const Real z1 = Z[size_t(j) * n + i], z2 = Z[size_t(j) * n + i + 1];
          Z[size_t(j) * n + i] = ct * z1 + st * z2;
          Z[size_t(j) * n + i + 1] = st * z1 - ct * z2;
        }
      }
      if (i < m - 1) { p = e[i]; g = st * e[i + 1]; e[i + 1] = -ct * e[i + 1]; }
    }
  }
}

// Lowest Ritz value (first index on ties) and, optionally, its eigenvector.
template <class Real>
Real tridiag_ground(const std::vector<Real>& alpha, const std::vector<Real>& beta, int n,
                    std::vector<Real>* vec) {
  if (n == 0) { if (vec) vec->clear(); return Real(0); }
  if (n == 1) { if (vec) vec->assign(1, Real(1)); return alpha[0]; }
  std::vector<Real> d, z;
  tridiag_ql(alpha, beta, n, d, vec ? &z : nullptr);
  int mi = 0;
  for (int i = 1; i < n; ++i) if (d[i] < d[mi]) mi = i;
  if (vec) {
    vec->resize(n);
    for (int i = 0; i < n; ++i) (*vec)[i] = z[size_t(i) * n + mi];
  }
  return d[mi];
}

// All Ritz values and the first component of each Ritz vector.
template <class Real>
void tridiag_first(const std::vector<Real>& alpha, const std::vector<Real>& beta,
                   std::vector<Real>& evals, std::vector<Real>& first) {
  const int n = int(alpha.size());
  evals.clear(); first.clear();
  if (n == 0) return;
  if (n == 1) { evals = {alpha[0]}; first = {Real(1)}; return; }
  std::vector<Real> d, z;
  tridiag_ql(alpha, beta, n, d, &z, 1);  // the first components only
  evals = d;
  first.assign(z.begin(), z.begin() + n);
}

// Cyclic Jacobi eigen-decomposition of a real symmetric n x n matrix A
// (row major, overwritten): sweeps over all pairs (p, q) until the
// off-diagonal Frobenius norm falls below 1e-15 of the total (at most 60
// sweeps).  evals ascending; evecs row major with eigenvector k in column k.
inline void jacobi_symmetric(std::vector<double> A, int n, std::vector<double>& evals,
                             std::vector<double>& evecs) {
  std::vector<double> V(size_t(n) * n, 0.0);
  for (int i = 0; i < n; ++i) V[size_t(i) * n + i] = 1.0;
  auto a = [&](int i, int j) -> double& { return A[size_t(i) * n + j]; };
  double total = 0.0;
  for (double x : A) total += x * x;
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j) off += 2.0 * a(i, j) * a(i, j);
    if (off <= 1e-30 * total || off == 0.0) break;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = a(p, q);
        if (apq == 0.0) continue;
        const double theta = (a(q, q) - a(p, p)) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::abs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {  // columns p, q
          const double akp = a(k, p), akq = a(k, q);
          a(k, p) = c * akp - s * akq;
          a(k, q) = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {  // rows p, q
          const double apk = a(p, k), aqk = a(q, k);
          a(p, k) = c * apk - s * aqk;
          a(q, k) = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double vkp = V[size_t(k) * n + p], vkq = V[size_t(k) * n + q];
          V[size_t(k) * n + p] = c * vkp - s * vkq;
          V[size_t(k) * n + q] = s * vkp + c * vkq;
        }
      }
  }
  std::vector<int> ord(n);
  for (int i = 0; i < n; ++i) ord[i] = i;
  std::sort(ord.begin(), ord.end(), [&](int x, int y) { return a(x, x) < a(y, y); });
  evals.resize(n);
  evecs.assign(size_t(n) * n, 0.0);
  for (int k = 0; k < n; ++k) {
    evals[k] = a(ord[k], ord[k]);
    for (int i = 0; i < n; ++i) evecs[size_t(i) * n + k] = V[size_t(i) * n + ord[k]];
  }
}

// Jacobi eigen-decomposition of a small Hermitian matrix H (row major);
// eigenvalues ascending, evecs[k*n + j] = component j of eigenvector k.
template <class Real>
void jacobi_hermitian(const std::vector<std::complex<Real>>& H, int n, std::vector<Real>& evals,
                      std::vector<std::complex<Real>>& evecs) {
  using C = std::complex<Real>;
  std::vector<C> A = H, V(size_t(n) * n, C(0));
  auto a = [&](int i, int j) -> C& { return A[size_t(i) * n + j]; };
  auto v = [&](int i, int j) -> C& { return V[size_t(i) * n + j]; };
  for (int i = 0; i < n; ++i) v(i, i) = Real(1);
  for (int iter = 0; iter < 1000; ++iter) {
    Real max_off = 0; int p = 0, q = 0;
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j)
        if (std::abs(a(i, j)) > max_off) { max_off = std::abs(a(i, j)); p = i; q = j; }
    if (max_off < Real(1e-15)) break;
    const C app = a(p, p), aqq = a(q, q), apq = a(p, q);
    const Real phi = Real(0.5) * std::atan2(Real(2) * std::abs(apq), std::real(app - aqq));
    const C c = std::cos(phi);
    const C s = std::sin(phi) * apq / std::abs(apq);
    for (int i = 0; i < n; ++i) {
      const C vip = v(i, p), viq = v(i, q);
      v(i, p) = c * vip + s * viq;
      v(i, q) = -std::conj(s) * vip + c * viq;
      if (i != p && i != q) {
        const C aip = a(i, p), aiq = a(i, q);
        a(i, p) = a(p, i) = c * aip + s * aiq;
        a(i, q) = a(q, i) = -std::conj(s) * aip + c * aiq;
      }
    }
    a(p, p) = c * c * app + s * std::conj(s) * aqq + Real(2) * std::real(c * s * std::conj(apq));
    a(q, q) = s * std::conj(s) * app + c * c * aqq - Real(2) * std::real(c * s * std::conj(apq));
    a(p, q) = a(q, p) = Real(0);
  }
  std::vector<int> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  std::sort(idx.begin(), idx.end(), [&](int i, int j) { return std::real(a(i, i)) < std::real(a(j, j)); });
  evals.clear();
  evecs.assign(size_t(n) * n, C(0));
  for (int k = 0; k < n; ++k) {
    evals.push_back(std::real(a(idx[k], idx[k])));
    for (int j = 0; j < n; ++j) evecs[size_t(k) * n + j] = v(j, idx[k]);
  }
}

}  // namespace qkb
