#include "solvers.hpp"
#include "npy.hpp"

#include <algorithm>
#include <cstring>
#include <chrono>
#include <cmath>
#include <numeric>
#include <random>

#include "dense.hpp"

namespace qkb {

namespace {

template <class Real> using C = std::complex<Real>;

// Device helpers on the operator's context stream.
struct Dev {
  const Operator& H;
  Context& c;
  qk_dtype t;
  uint64_t n;
  explicit Dev(const Operator& op, qk_dtype dt) : H(op), c(op.ctx()), t(dt), n(op.dim()) {}

  DevVec vec(bool zero = true) const { return DevVec(n, t, H.device(), zero); }
  template <class Real> void upload(const C<Real>* h, DevVec& v) const {
    cuda_check(cudaMemcpyAsync(v.data(), h, n * sizeof(C<Real>), cudaMemcpyHostToDevice, c.stream), "H2D");
  }
  template <class Real> void download(const DevVec& v, std::vector<C<Real>>& h) const {
    h.resize(n);
    cuda_check(cudaMemcpyAsync(h.data(), v.data(), n * sizeof(C<Real>), cudaMemcpyDeviceToHost, c.stream), "D2H");
    c.sync();
  }
  std::complex<double> dot(const void* x, const void* y) const {
    qkd_check(qkd_dot(c.ws, t, n, x, y, c.dres(0), c.stream), "dot");
    const double* r = c.fetch(c.dres(0), 2);
    return {r[0], r[1]};
  }
  void scal(double a, void* x) const { qkd_check(qkd_scal(t, n, a, 0.0, x, c.stream), "scal"); }
  void scale_into(double a, const void* x, void* y) const {
    qkd_check(qkd_axpby(t, n, a, 0.0, x, 0.0, 0.0, y, c.stream), "scale");
  }
  void axpy(std::complex<double> a, const void* x, void* y) const {
    qkd_check(qkd_axpy(t, n, a.real(), a.imag(), x, y, c.stream), "axpy");
  }
  // out[j] = <P_j, x> for j < k, after x -= sum a_m U_m (M <= 2); P chunked by 511.
  void update_mdot(int M, const void* const* U, const double* a, const PtrArray& P, int k, void* x,
                   double* out) const {
    constexpr int kChunk = 511;
    if (k == 0) {
      if (M > 0) qkd_check(qkd_update_mdot(c.ws, t, n, M, U, a, 0, nullptr, x, out, c.stream), "update");
      return;
    }
    for (int j0 = 0; j0 < k; j0 += kChunk) {
      const int kk = std::min(kChunk, k - j0);
      qkd_check(qkd_update_mdot(c.ws, t, n, j0 == 0 ? M : 0, U, a, kk, P.at(j0), x, out + 2 * j0, c.stream),
                "multi-dot");
    }
  }
  // x -= sum_j coef_j P_j (coef device, 2k doubles); nrm2 (device) if given.
  void mupdate(const PtrArray& P, int k, const double* coef, void* x, double* nrm2) const {
    constexpr int kChunk = 511;
    if (k == 0) {
      if (nrm2) qkd_check(qkd_mupdate(c.ws, t, n, 0, nullptr, nullptr, x, nrm2, c.stream), "norm");
      return;
    }
    for (int j0 = 0; j0 < k; j0 += kChunk) {
      const int kk = std::min(kChunk, k - j0);
      const bool last = (j0 + kk == k);
      qkd_check(qkd_mupdate(c.ws, t, n, kk, P.at(j0), coef + 2 * j0, x, last ? nrm2 : nullptr, c.stream),
                "block update");
    }
  }
};

template <class Real> void normalize(const Dev& d, void* x) {  // vector_ops.hpp:90-96
  const Real nr = Real(std::sqrt(Real(d.dot(x, x).real())));
  if (nr == Real(0)) return;
  d.scal(double(Real(1) / nr), x);
}

}  // namespace

template <class Real>
void reference_uniform_start(uint64_t dim, std::vector<std::complex<Real>>& v) {
  std::mt19937 rng(1234);
  std::uniform_real_distribution<Real> dist(-1.0, 1.0);
  v.resize(dim);
  for (uint64_t i = 0; i < dim; ++i) {
    const Real im = dist(rng);
    const Real re = dist(rng);
    v[i] = {re, im};
  }
}

template <class Real>
LanczosOut<Real> lanczos(const Operator& H, int maxiter, Real tol, const std::complex<Real>* start,
                         std::vector<std::complex<Real>>* ritz) {
  LanczosOut<Real> res;
  const uint64_t dim = H.dim();
  if (dim == 0) return res;
  const qk_dtype T = complex_dtype<Real>();
  Dev d(H, T);
  const int lim = int(std::min<uint64_t>(uint64_t(std::max(maxiter, 0)), dim));

  std::vector<DevVec> V;
  PtrArray P(size_t(lim) + 3, H.device());
  DevVec w = d.vec();
  DevVec coef(size_t(2) * (lim + 4), QK_F64, H.device());
  double* cd = static_cast<double*>(coef.data());

  {
    std::vector<C<Real>> hv;
    if (start) hv.assign(start, start + dim);
    else reference_uniform_start<Real>(dim, hv);
    V.push_back(d.vec(false));
    d.upload<Real>(hv.data(), V[0]);
  }
  normalize<Real>(d, V[0].data());
  P.set(0, V[0].data(), d.c.stream);

  std::vector<Real>& alphas = res.alphas;
  std::vector<Real>& betas = res.betas;
  bool converged = false;
  Real e_old = Real(1e100);
  int actual = 0;
  for (int iter = 0; iter < lim; ++iter) {
    actual = iter + 1;
    const int k = int(V.size()) - 1;  // current vector index (== iter)
    H.apply_dot(T, V[k].data(), w.data(), d.c.dres(0));
    const Real alpha = Real(d.c.fetch(d.c.dres(0), 1)[0]);
    alphas.push_back(alpha);

    // w -= alpha v_k + beta v_{k-1}, then c_j = <v_j, w> (j <= k) and <w, w>.
    const void* U[2] = {V[k].data(), k > 0 ? V[k - 1].data() : nullptr};
    const double a[4] = {double(alpha), 0.0, k > 0 ? double(betas.back()) : 0.0, 0.0};
    P.set(k + 1, w.data(), d.c.stream);
    d.update_mdot(k > 0 ? 2 : 1, U, a, P, k + 2, w.data(), cd);
    d.mupdate(P, k + 1, cd, w.data(), cd + 2 * (k + 2));
    const double* h = d.c.fetch(cd + 2 * (k + 1), 4);
    const double before = h[0];
    double after = h[2];
    if (after < 0.25 * before) {  // CGS lost accuracy: project once more
      ++res.reorth_second_rounds;
      d.update_mdot(0, nullptr, nullptr, P, k + 1, w.data(), cd);
      d.mupdate(P, k + 1, cd, w.data(), cd + 2 * (k + 2));
      after = d.c.fetch(cd + 2 * (k + 2), 1)[0];
    }
    const Real beta = Real(std::sqrt(Real(after)));
    if (beta < Real(1e-15)) { converged = true; break; }
    if (iter + 1 == lim) break;
    betas.push_back(beta);
    V.push_back(d.vec(false));
    d.scale_into(double(Real(1) / beta), w.data(), V.back().data());
    P.set(k + 1, V.back().data(), d.c.stream);
    if (iter > 0) {
      const Real e = tridiag_ground<Real>(alphas, betas, int(alphas.size()), nullptr);
      if (std::abs(e - e_old) < tol) { e_old = e; converged = true; break; }
      e_old = e;
    }
  }
  std::vector<Real> z;
  res.energy = tridiag_ground<Real>(alphas, betas, int(alphas.size()), &z);
  res.iterations = actual;
  res.converged = converged;
  if (ritz) {
    DevVec r = d.vec(true);
    const int m = int(alphas.size());
    std::vector<double> nz(2 * size_t(std::max(m, 1)), 0.0);
    for (int i = 0; i < m; ++i) nz[2 * i] = -double(z[i]);
    cuda_check(cudaMemcpyAsync(cd, nz.data(), sizeof(double) * 2 * m, cudaMemcpyHostToDevice, d.c.stream), "H2D");
    d.mupdate(P, m, cd, r.data(), nullptr);
    normalize<Real>(d, r.data());
    d.download<Real>(r, *ritz);
  }
  return res;
}


namespace {
double now_s() {
  using clk = std::chrono::steady_clock;
  return std::chrono::duration<double>(clk::now().time_since_epoch()).count();
}
}  // namespace

CoreOut lanczos_core(const Operator& H, qk_dtype T, const void* start, int maxiter, double tol_dE, double tol_res,
                     qk_dtype tout, void* ritz, double t0) {
  CoreOut res;
  const uint64_t dim = H.dim();
  if (dim == 0) return res;
  Dev d(H, T);
  const int lim = int(std::min<uint64_t>(uint64_t(std::max(maxiter, 0)), dim));
  std::vector<DevVec> V;
  PtrArray P(size_t(lim) + 3, H.device());
  DevVec w = d.vec();
  DevVec coef(size_t(2) * (lim + 4), QK_F64, H.device());
  double* cd = static_cast<double*>(coef.data());
  V.push_back(d.vec(false));
  qkd_check(qkd_copy(T, dim, start, V[0].data(), d.c.stream), "copy");
  {
    const double n0 = std::sqrt(d.dot(V[0].data(), V[0].data()).real());
    if (n0 == 0.0) throw std::invalid_argument("qkrylov_b200: zero start vector");
    d.scal(1.0 / n0, V[0].data());
  }
  P.set(0, V[0].data(), d.c.stream);
  std::vector<double>& a = res.alphas;
  std::vector<double>& b = res.betas;
  double e_old = 1e300;
  for (int iter = 0; iter < lim; ++iter) {
    res.iterations = iter + 1;
    const int k = int(V.size()) - 1;
    H.apply_dot(T, V[k].data(), w.data(), d.c.dres(0));
    const double alpha = d.c.fetch(d.c.dres(0), 1)[0];
    a.push_back(alpha);
    const void* U[2] = {V[k].data(), k > 0 ? V[k - 1].data() : nullptr};
    const double co[4] = {alpha, 0.0, k > 0 ? b.back() : 0.0, 0.0};
    P.set(k + 1, w.data(), d.c.stream);
    d.update_mdot(k > 0 ? 2 : 1, U, co, P, k + 2, w.data(), cd);
    d.mupdate(P, k + 1, cd, w.data(), cd + 2 * (k + 2));
    const double* hh = d.c.fetch(cd + 2 * (k + 1), 4);
    double after = hh[2];
    if (after < 0.25 * hh[0]) {
      d.update_mdot(0, nullptr, nullptr, P, k + 1, w.data(), cd);
      d.mupdate(P, k + 1, cd, w.data(), cd + 2 * (k + 2));
      after = d.c.fetch(cd + 2 * (k + 2), 1)[0];
    }
    const double beta = std::sqrt(after);
    std::vector<double> z;
    const double e = tridiag_ground<double>(a, b, int(a.size()), &z);
    const double rest = beta * std::abs(z.back());
    res.trace.push_back({iter + 1, e, now_s() - t0, rest});
    res.energy = e;
    res.resid_est = rest;
    if (beta < 1e-15 || rest <= tol_res * std::abs(e) || (iter > 0 && std::abs(e - e_old) < tol_dE * std::abs(e))) {
      res.converged = true;
      break;
    }
    e_old = e;
    if (iter + 1 == lim) break;
    b.push_back(beta);
    V.push_back(d.vec(false));
    d.scale_into(1.0 / beta, w.data(), V.back().data());
    P.set(k + 1, V.back().data(), d.c.stream);
  }
  if (ritz) {
    std::vector<double> z;
    const int m = int(a.size());
    tridiag_ground<double>(a, b, m, &z);
    std::vector<double> cz(2 * size_t(m), 0.0);
    for (int i = 0; i < m; ++i) cz[2 * i] = z[i];
    cuda_check(cudaMemcpyAsync(cd, cz.data(), sizeof(double) * 2 * m, cudaMemcpyHostToDevice, d.c.stream), "H2D");
    constexpr int kChunk = 511;
    // ritz = sum_i z_i V_i assembled in dtype tout (chunks accumulate through
    // a temporary when m exceeds one launch)
    if (m <= kChunk) {
      qkd_check(qkd_combine(T, dim, m, P.data(), cd, tout, ritz, d.c.stream), "combine");
    } else {
      throw std::invalid_argument("qkrylov_b200: Ritz assembly over more than 511 vectors is not supported");
    }
    Dev dout(H, tout);
    const double nr = std::sqrt(dout.dot(ritz, ritz).real());
    if (nr > 0) dout.scal(1.0 / nr, ritz);
  }
  return res;
}

namespace {
// One refinement pass: Lanczos in dtype ti on the Krylov space of r = H psi -
// E psi, kept orthogonal to psi, then psi <- the Ritz vector of
// span{psi, v_1..v_m}.  With v_1 = r / |r| the projection of H onto that
// span is the tridiagonal [E, |r|; |r|, a_1, b_1; ...], so the Rayleigh-Ritz
// step needs no further products.  The v_j can be FP32: they only carry the
// correction, whose size is that of the residual, so their rounding enters
// psi at (FP32 epsilon) x |r|.  Stops when the Ritz residual estimate
// b_m |z_m| / |theta| <= target, at breakdown or after maxiter steps.
// partial: partial reorthogonalisation (below); otherwise every step is
// orthogonalised against psi and all stored v_k.
int refine_pass(const Operator& H, qk_dtype ti, qk_dtype hi, DevVec& psi, const DevVec& r, double E, double nr,
                int maxiter, double target, std::vector<DevVec>& V, DevVec& psi_t, DevVec& wt, DevVec& tmp,
                PtrArray& P, DevVec& coef, std::vector<TraceEntry>& trace, int it0, double t0, bool partial) {
  Dev d(H, ti), dh(H, hi);
  const uint64_t dim = H.dim();
  double* cd = static_cast<double*>(coef.data());
  if (ti == hi) qkd_check(qkd_copy(hi, dim, psi.data(), psi_t.data(), d.c.stream), "copy");
  else qkd_check(qkd_convert(hi, psi.data(), ti, psi_t.data(), dim, d.c.stream), "convert");
  while (V.size() < 1) V.push_back(d.vec(false));
  qkd_check(qkd_convert(hi, r.data(), ti, V[0].data(), dim, d.c.stream), "convert");
  d.scal(1.0 / nr, V[0].data());
  P.set(0, psi_t.data(), d.c.stream);
  P.set(1, V[0].data(), d.c.stream);
  std::vector<double> a{E}, b{nr}, z;
  // Partial reorthogonalisation (H. D. Simon, "The Lanczos algorithm with
  // partial reorthogonalization", Math. Comp. 42 (1984) 115-142): a step
  // orthogonalises w against psi only, after the three-term recurrence; the
  // omega recurrence estimates <v_{j+1}, v_k> for the stored v_k, and when
  // the largest estimate passes sqrt(u) (u the unit roundoff of the pass's
  // vectors) w is orthogonalised against all of them, at that step and the
  // next, and the estimates restart at u.  The Krylov basis stays
  // semi-orthogonal, which keeps the tridiagonal's Ritz values those of the
  // projection to working accuracy.
  const double u = (ti == QK_F32 || ti == QK_C64) ? 0x1p-24 : 0x1p-53, wmax = std::sqrt(u);
  PtrArray L(2, H.device());
  L.set(0, psi_t.data(), d.c.stream);
  L.set(1, wt.data(), d.c.stream);
  std::vector<double> wprev, wcur{1.0}, wnew;  // omega_{j-1,k}, omega_{j,k}, omega_{j+1,k} over the stored v_k
  double anorm = std::abs(E) + nr;
  bool full = !partial;
  int m = 0;
  for (int j = 0; j < maxiter; ++j) {
    m = j + 1;
    H.apply_dot(ti, V[j].data(), wt.data(), d.c.dres(0));
    const double alpha = d.c.fetch(d.c.dres(0), 1)[0];
    a.push_back(alpha);
    const void* U[2] = {V[j].data(), j > 0 ? V[j - 1].data() : nullptr};
    const double co[4] = {alpha, 0.0, j > 0 ? b.back() : 0.0, 0.0};
    const int np = j + 2;  // psi_t, v_1..v_{j+1}
    auto orth_all = [&]() {  // w -= sum <P_i, w> P_i over psi_t and every stored v; returns |w|^2
      d.update_mdot(0, nullptr, nullptr, P, np, wt.data(), cd);
      d.mupdate(P, np, cd, wt.data(), cd + 2 * (np + 1));
      return d.c.fetch(cd + 2 * (np + 1), 1)[0];
    };
    double before, after;
    if (full) {
      P.set(np, wt.data(), d.c.stream);
      d.update_mdot(j > 0 ? 2 : 1, U, co, P, np + 1, wt.data(), cd);
      d.mupdate(P, np, cd, wt.data(), cd + 2 * (np + 1));
      const double* hh = d.c.fetch(cd + 2 * np, 4);
      before = hh[0];
      after = hh[2];
      if (after < 0.25 * before) after = orth_all();
    } else {
      d.update_mdot(j > 0 ? 2 : 1, U, co, L, 2, wt.data(), cd);
      d.mupdate(L, 1, cd, wt.data(), cd + 4);
      const double* hh = d.c.fetch(cd + 2, 4);
      before = hh[0];
      after = hh[2];
    }
    double beta = std::sqrt(after);
    anorm = std::max(anorm, std::abs(alpha) + b[j] + beta);
    wnew.assign(size_t(j) + 2, 0.0);
    double worst = 0.0;
    if (!full && beta > 0.0) {
      for (int k = 0; k < j; ++k) {
        double v = b[k + 1] * wcur[k + 1] + (a[k + 1] - alpha) * wcur[k] - b[j] * wprev[k];
        if (k > 0) v += b[k] * wcur[k - 1];
        v += std::copysign(2.0 * u * anorm, v);  // rounding of this step
        wnew[k] = v / beta;
        worst = std::max(worst, std::abs(wnew[k]));
      }
    }
    const bool now = !full && (worst > wmax || after < 0.25 * before);
    if (now) {
      after = orth_all();
      beta = std::sqrt(after);
    }
    if (full || now) std::fill(wnew.begin(), wnew.begin() + j, u);
    wnew[j] = beta > 0.0 ? std::max(u, u * anorm / beta) : u;
    wnew[j + 1] = 1.0;
    full = now || !partial;  // a step that orthogonalised against all is followed by one more
    const double theta = tridiag_ground<double>(a, b, int(a.size()), &z);
    const double est = beta * std::abs(z.back()) / std::abs(theta);
    trace.push_back({it0 + m, theta, now_s() - t0, est});
    if (est <= target || beta < 1e-15 || j + 1 == maxiter) break;
    b.push_back(beta);
    wprev.swap(wcur);
    wcur.swap(wnew);
    if (int(V.size()) < j + 2) V.push_back(d.vec(false));
    d.scale_into(1.0 / beta, wt.data(), V[j + 1].data());
    P.set(j + 2, V[j + 1].data(), d.c.stream);
  }
  // psi <- z_0 psi + sum_i z_i v_i, assembled in FP64, normalised
  std::vector<double> cz(2 * size_t(m), 0.0);
  for (int i = 0; i < m; ++i) cz[2 * i] = z[i + 1];
  cuda_check(cudaMemcpyAsync(cd, cz.data(), sizeof(double) * 2 * m, cudaMemcpyHostToDevice, d.c.stream), "H2D");
  qkd_check(qkd_combine(ti, dim, m, P.at(1), cd, hi, tmp.data(), d.c.stream), "combine");
  qkd_check(qkd_axpby(hi, dim, 1.0, 0.0, tmp.data(), z[0], 0.0, psi.data(), d.c.stream), "axpby");
  const double np2 = dh.dot(psi.data(), psi.data()).real();
  dh.scal(1.0 / std::sqrt(np2), psi.data());
  return m;
}
}  // namespace

MixedOut lanczos_mixed(const Operator& H, const void* start, uint64_t seed, int maxiter, double tol_res,
                       void* psi_out, bool low_phase, bool partial) {
  MixedOut out;
  const uint64_t dim = H.dim();
  if (dim == 0) return out;
  if (maxiter < 1 || maxiter > 511) throw std::invalid_argument("qkrylov_b200: maxiter must be in [1, 511]");
  const bool real = H.all_real();
  const qk_dtype lo = real ? QK_F32 : QK_C64, hi = real ? QK_F64 : QK_C128;
  const double t0 = now_s();
  Dev dh(H, hi);
  DevVec psi = dh.vec(false), w = dh.vec(false);
  PtrArray Pw(1, H.device());
  Pw.set(0, w.data(), dh.c.stream);
  // E = <psi, H psi> and w <- H psi - E psi, |w|^2 (one FP64 apply)
  auto residual = [&](double& E) {
    H.apply_dot(hi, psi.data(), w.data(), dh.c.dres(0));
    E = dh.c.fetch(dh.c.dres(0), 1)[0];
    const void* U[1] = {psi.data()};
    const double co[2] = {E, 0.0};
    dh.update_mdot(1, U, co, Pw, 1, w.data(), dh.c.dres(0));
    return std::sqrt(dh.c.fetch(dh.c.dres(0), 1)[0]);
  };
  if (!low_phase) {
    // plain FP64: Lanczos from the start, restarted from the Ritz vector
    // until the explicit residual meets tol_res
    if (start) qkd_check(qkd_copy(hi, dim, start, psi.data(), dh.c.stream), "copy");
    else qkd_check(qkd_random(hi, dim, seed, 0, psi.data(), dh.c.stream), "random");
    double e = 0.0;
    for (int rs = 0; rs < 8; ++rs) {
      auto p2 = lanczos_core(H, hi, psi.data(), maxiter, 0.0, 0.1 * tol_res, hi, psi.data(), t0);
      out.iters_high += p2.iterations;
      for (auto te : p2.trace) { te.iteration += out.iters_high - p2.iterations; out.trace.push_back(te); }
      const double nr = residual(e);
      out.residual = nr / std::abs(e);
      out.restarts = rs + 1;
      if (out.residual <= tol_res) { out.converged = true; break; }
    }
    out.energy = e;
    out.seconds_high = now_s() - t0;
    if (psi_out) qkd_check(qkd_copy(hi, dim, psi.data(), psi_out, dh.c.stream), "copy");
    dh.c.sync();
    return out;
  }
  // Mixed: FP64 iterate psi and FP64 residuals; the Krylov passes that
  // build each correction run on FP32 vectors (FP64 scalars).  A pass that
  // fails to halve the residual switches the passes to FP64.
  {
    Dev dl(H, lo);
    DevVec s0 = dl.vec(false);
    if (start) qkd_check(qkd_copy(lo, dim, start, s0.data(), dl.c.stream), "copy");
    else qkd_check(qkd_random(lo, dim, seed, 0, s0.data(), dl.c.stream), "random");
    qkd_check(qkd_convert(lo, s0.data(), hi, psi.data(), dim, dl.c.stream), "convert");
    const double n0 = std::sqrt(dh.dot(psi.data(), psi.data()).real());
    if (n0 == 0.0) throw std::invalid_argument("qkrylov_b200: zero start vector");
    dh.scal(1.0 / n0, psi.data());
  }
  std::vector<DevVec> V;
  qk_dtype ti = lo;
  DevVec psi_t(dim, ti, H.device(), false), wt(dim, ti, H.device(), false), tmp = dh.vec(false);
  PtrArray P(size_t(maxiter) + 3, H.device());
  DevVec coef(size_t(2) * (maxiter + 8), QK_F64, H.device());
  double e = 0.0, eps_prev = 1e300, t_fp64 = 0.0;
  int steps = 0;
  // passes of at most `pass` steps: the orthogonalisations a pass needs
  // grow with its length, a restart from the Ritz vector resets them.
  // Heisenberg N=28 to residual 1e-10 (partial reorthogonalisation): 0.126 s
  // with passes of 32 (118 FP32 steps), 0.130 s with 48 (110), 0.135 s with
  // 64 (112); Hubbard 4x4 1.62 s / 1.22 s / 1.26 s (239 / 177 / 179 steps).
  // With full reorthogonalisation of every step, 32 was also the best of 24,
  // 32 and 64 on Heisenberg, and 16 made Hubbard's FP32 passes stall and fall
  // back to FP64.  A pass that cuts the residual less than twentyfold (a
  // small relative gap, where restarting from the Ritz vector alone
  // converges slowly) doubles the length of the next one: Hubbard 4x4 1.62 s
  // (239 steps) with a tenfold rule, 1.09 s (159) with twentyfold, the same
  // with 33- and 100-fold; J1-J2 N=24 over 224 couplings 6.2 s with ten- and
  // twentyfold, 6.6 s with 33-fold.
  constexpr int kPass = 32;
  int pass = std::min(maxiter, kPass);
  for (int outer = 0; outer < 40; ++outer) {
    const double tr0 = now_s();
    const double nr = residual(e);
    t_fp64 += now_s() - tr0;
    const double eps = nr / std::abs(e);
    out.iters_high += 1;
    out.trace.push_back({steps + out.iters_high, e, now_s() - t0, eps});
    out.residual = eps;
    out.restarts = outer;
    if (eps <= tol_res || nr == 0.0) { out.converged = true; break; }
    if (ti == lo && outer > 0 && eps > 0.5 * eps_prev) {
      ti = hi;  // FP32 passes stopped helping: finish in FP64
      V.clear();
      psi_t = DevVec(dim, ti, H.device(), false);
      wt = DevVec(dim, ti, H.device(), false);
    }
    if (outer > 0 && eps > 0.05 * eps_prev) {
      // a longer pass stores more vectors: at most half of the device's free memory more
      size_t free_b = 0, total_b = 0;
      cuda_check(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
      const size_t room = V.size() + free_b / 2 / (dim * qk_dtype_size(ti));
      pass = int(std::min<size_t>({size_t(maxiter), size_t(2) * pass, std::max(room, size_t(pass))}));
    }
    eps_prev = eps;
    const double target = std::max(0.3 * tol_res, 1e-6 * eps);
    const double tp0 = now_s();
    const int m = refine_pass(H, ti, hi, psi, w, e, nr, pass, target, V, psi_t, wt, tmp, P,
                              coef, out.trace, steps + out.iters_high, t0, partial);
    steps += m;
    if (ti == lo) out.iters_low += m;
    else { out.iters_high += m; t_fp64 += now_s() - tp0; }
  }
  out.energy = e;
  out.seconds_high = t_fp64;
  out.seconds_low = now_s() - t0 - t_fp64;
  if (psi_out) qkd_check(qkd_copy(hi, dim, psi.data(), psi_out, dh.c.stream), "copy");
  dh.c.sync();
  return out;
}

// Block Davidson for real operators on real vectors (float32 / float64).
// Only the basis V is stored: H V_j is formed once, when v_j enters, for
// the new column of the projection T = V^T H V, and the residuals of the
// lowest `block` Ritz pairs are recomputed as H u - theta u from the Ritz
// vectors u = V y.  Corrections t = r / (diag - theta) (the reference's
// clamped preconditioner) are orthogonalised against V twice (classical
// Gram-Schmidt) and appended; when V would exceed max_subspace it restarts
// from the lowest 2*block Ritz vectors (T becomes diagonal) plus the block's
// Ritz vectors of the previous iteration (GD+k, Stathopoulos & Saad 1998,
// "Restarting techniques for the (Jacobi-)Davidson symmetric eigenvalue
// methods"): the pair (current, previous) Ritz vector spans the direction of
// the recurrence a plain thick restart discards, which keeps the upper pairs
// converging at the rate they had before the restart.
DavidsonBlockOut davidson_block(const Operator& H, qk_dtype t, int n_eig, int block, int max_subspace, double tol,
                                uint64_t seed, int maxiter, double* evecs_out) {
  if (t != QK_F32 && t != QK_F64) throw std::invalid_argument("qkrylov_b200: block Davidson needs real vectors");
  if (!H.all_real()) throw std::invalid_argument("qkrylov_b200: block Davidson needs a real operator");
  const uint64_t dim = H.dim();
  if (n_eig < 1 || block < n_eig || max_subspace < 2 * block + block || uint64_t(max_subspace) > dim || maxiter < 1 ||
      max_subspace > 510)
    throw std::invalid_argument("qkrylov_b200: block Davidson sizes (n_eig <= block, 3 block <= max_subspace <= dim)");
  DavidsonBlockOut out;
  const double t0 = now_s();
  Dev d(H, t);
  const int dev = H.device();
  DevVec diag = d.vec(false);
  H.diagonal(t, diag.data());
  std::vector<DevVec> V;
  V.reserve(max_subspace);
  std::vector<DevVec> U(2 * block), R(block), Uprev(block);
  DevVec w = d.vec(false);
  PtrArray P(size_t(max_subspace) + 4, dev);
  DevVec coef(size_t(2) * (max_subspace + 8), QK_F64, dev);
  double* cd = static_cast<double*>(coef.data());
  // many-against-many passes: up to kX vectors X_a against the basis in one
  // pass over it (projections <V_i, X_a>, combinations sum_i c_ia V_i)
  constexpr int kX = 8;
  PtrArray PX(kX, dev), PN(size_t(block), dev);
  const int mrows = (max_subspace + 7) / 8 * 8;
  DevVec cm(size_t(max_subspace) * kX, QK_F64, dev), dm(size_t(16) * mrows, QK_F64, dev);
  std::vector<double> dmh(size_t(16) * mrows);
  // D[i*nx + a] = <V_i, X_a> for i < mm
  auto multi_dot = [&](int mm, const std::vector<void*>& xs) {
    const int nx = int(xs.size());
    for (int a = 0; a < nx; ++a) PX.set(a, xs[a], d.c.stream);
    qkd_check(qkd_multi_dot(d.c.ws, t, dim, mm, P.at(0), nx, PX.data(), static_cast<double*>(dm.data()), d.c.stream),
              "multi-dot");
    const size_t rows = size_t(mm + 7) / 8 * 8;
    cuda_check(cudaMemcpyAsync(dmh.data(), dm.data(), sizeof(double) * 16 * rows, cudaMemcpyDeviceToHost, d.c.stream),
               "D2H");
    d.c.sync();
    std::vector<double> D(size_t(mm) * nx);
    for (int i = 0; i < mm; ++i)
      for (int a = 0; a < nx; ++a) D[size_t(i) * nx + a] = dmh[2 * (size_t(i) * kX + a)];
    return D;
  };
  // X_a = sum_i c[i*nx + a] V_i (acc false) or X_a -= ... (acc true), i < mm
  auto multi_update = [&](int mm, const std::vector<double>& c, const std::vector<void*>& xs, bool acc) {
    const int nx = int(xs.size());
    for (int a = 0; a < nx; ++a) PX.set(a, xs[a], d.c.stream);
    cuda_check(cudaMemcpyAsync(cm.data(), c.data(), sizeof(double) * size_t(mm) * nx, cudaMemcpyHostToDevice,
                               d.c.stream), "H2D");
    qkd_check(qkd_multi_update(t, dim, mm, P.at(0), static_cast<const double*>(cm.data()), nx,
                               const_cast<void* const*>(reinterpret_cast<const void* const*>(PX.data())), acc ? 1 : 0,
                               d.c.stream), "multi-update");
    d.c.sync();  // c is host memory reused by the caller
  };
  std::vector<double> T;  // m x m, row major
  int m = 0, m_proj = 0;  // basis size; columns of T filled
  // Orthonormalise x against V[0..m) (two passes) and append it; false if
  // it vanished (linearly dependent).  `before`: |x|^2 before any
  // orthogonalisation (< 0: take it now).
  auto append = [&](DevVec&& x, double before = -1.0) -> bool {
    if (before < 0.0) before = d.dot(x.data(), x.data()).real();
    for (int pass = 0; pass < 2 && m > 0; ++pass) {
      d.update_mdot(0, nullptr, nullptr, P, m, x.data(), cd);
      d.mupdate(P, m, cd, x.data(), cd + 2 * (m + 1));
    }
    const double nn = d.dot(x.data(), x.data()).real();
    if (!(nn > 1e-20 * std::max(before, 1e-300)) || nn == 0.0) return false;
    d.scal(1.0 / std::sqrt(nn), x.data());
    P.set(m, x.data(), d.c.stream);
    V.push_back(std::move(x));
    ++m;
    return true;
  };
  for (int a = 0; a < block; ++a) {
    DevVec x = d.vec(false);
    qkd_check(qkd_random(t, dim, seed * 7919ull + uint64_t(a) + 1, 0, x.data(), d.c.stream), "random");
    append(std::move(x));
  }
  for (auto& r : R) r = d.vec(false);
  std::vector<double> theta, Y;
  for (int it = 0; it < maxiter; ++it) {
    out.iterations = it + 1;
    // new columns of T: T[i][j] = <v_i, H v_j> for the vectors added since,
    // H v_j formed into the residual buffers (free at this point) and
    // projected onto the basis up to kX columns per pass
    for (int j0 = m_proj; j0 < m;) {
      const int cnt = std::min({kX, block, m - j0});
      std::vector<void*> xs;
      for (int b = 0; b < cnt; ++b) {
        H.apply(t, V[j0 + b].data(), R[b].data());
        ++out.applies;
        xs.push_back(R[b].data());
      }
      const std::vector<double> D = multi_dot(j0 + cnt, xs);
      const int mn = j0 + cnt;
      std::vector<double> Tn(size_t(mn) * mn, 0.0);
      for (int r = 0; r < j0; ++r)
        for (int c = 0; c < j0; ++c) Tn[size_t(r) * mn + c] = T[size_t(r) * j0 + c];
      for (int b = 0; b < cnt; ++b) {
        const int j = j0 + b;
        for (int i = 0; i <= j; ++i) {
          Tn[size_t(i) * mn + j] = D[size_t(i) * cnt + b];
          Tn[size_t(j) * mn + i] = D[size_t(i) * cnt + b];
        }
      }
      T.swap(Tn);
      j0 += cnt;
    }
    m_proj = m;
    jacobi_symmetric(T, m, theta, Y);
    // Ritz vectors of the lowest nb pairs in one pass over the basis (kX at
    // a time), then their residuals; the previous iteration's Ritz vectors
    // move to Uprev (kept for the restart)
    const int nb = std::min(block, m);
    double worst = 0.0;
    out.residuals.assign(nb, 0.0);
    for (int a = 0; a < nb; ++a) std::swap(U[a], Uprev[a]);
    auto ritz = [&](int a0, int a1) {  // U[a] = V y_a for a in [a0, a1)
      for (int c0 = a0; c0 < a1; c0 += kX) {
        const int cnt = std::min(kX, a1 - c0);
        std::vector<double> c(size_t(m) * cnt);
        std::vector<void*> xs;
        for (int b = 0; b < cnt; ++b) {
          if (!U[c0 + b].data()) U[c0 + b] = d.vec(false);
          xs.push_back(U[c0 + b].data());
          for (int i = 0; i < m; ++i) c[size_t(i) * cnt + b] = Y[size_t(i) * m + c0 + b];
        }
        multi_update(m, c, xs, false);
      }
    };
    ritz(0, nb);
    for (int a = 0; a < nb; ++a) {
      H.apply(t, U[a].data(), R[a].data());
      ++out.applies;
      d.axpy({-theta[a], 0.0}, U[a].data(), R[a].data());
      out.residuals[a] = std::sqrt(d.dot(R[a].data(), R[a].data()).real());
      if (a < n_eig) worst = std::max(worst, out.residuals[a]);
    }
    out.trace.push_back({it + 1, theta[0], now_s() - t0, worst});
    out.eigenvalues.assign(theta.begin(), theta.begin() + n_eig);
    if (worst < tol) { out.converged = true; break; }
    if (it + 1 == maxiter) break;
    // corrections of the unconverged pairs among the lowest nb
    std::vector<DevVec> C;
    for (int a = 0; a < nb; ++a) {
      if (out.residuals[a] < tol) continue;
      DevVec c = d.vec(false);
      qkd_check(qkd_dav_precond(t, dim, diag.data(), theta[a], R[a].data(), c.data(), d.c.stream), "precond");
      C.push_back(std::move(c));
    }
    if (m + int(C.size()) > max_subspace) {  // restart from the lowest 2*block Ritz vectors
      const int keep = std::min(2 * block, m);
      ritz(nb, keep);
      std::vector<DevVec> NV;
      for (int a = 0; a < keep; ++a) { NV.push_back(std::move(U[a])); U[a] = DevVec(); }
      for (int a = 0; a < keep; ++a) { U[a] = std::move(V[a]); }  // recycle storage
      V.clear();
      for (int a = 0; a < keep; ++a) {
        V.push_back(std::move(NV[a]));
        P.set(a, V[a].data(), d.c.stream);
      }
      for (int a = keep; a < int(U.size()); ++a) U[a] = DevVec();
      m = keep;
      m_proj = keep;
      T.assign(size_t(keep) * keep, 0.0);
      for (int a = 0; a < keep; ++a) T[size_t(a) * keep + a] = theta[a];
      ++out.restarts;
      // GD+k: the previous iteration's Ritz vectors of the block, made
      // orthogonal to the kept ones (dropped where they add no direction);
      // their columns of T are formed at the top of the next iteration
      for (int a = 0; a < nb && it > 0 && m + int(C.size()) < max_subspace; ++a) {
        if (!Uprev[a].data()) break;
        DevVec pv = d.vec(false);
        qkd_check(qkd_copy(t, dim, Uprev[a].data(), pv.data(), d.c.stream), "copy");
        append(std::move(pv));
      }
    }
    // the corrections against the basis as one block (classical Gram-Schmidt:
    // a projection pass and an update pass over the basis per kX
    // corrections), then one by one against the corrections already taken.
    // Each is repeated only when the first round removed more than half of a
    // vector's squared norm ("twice is enough": Daniel, Gragg, Kaufman and
    // Stewart, Math. Comp. 30 (1976) 772-795); the norm after the block round
    // is |x|^2 - sum_i <v_i, x>^2, known from the projections.
    int added = 0;
    const int m_old = m;
    for (size_t c0 = 0; c0 < C.size(); c0 += kX) {
      const int cnt = int(std::min<size_t>(kX, C.size() - c0));
      std::vector<void*> xs;
      std::vector<double> before(cnt);
      for (int b = 0; b < cnt; ++b) {
        xs.push_back(C[c0 + b].data());
        before[b] = d.dot(C[c0 + b].data(), C[c0 + b].data()).real();
      }
      for (int pass = 0; pass < 2; ++pass) {
        const std::vector<double> D = multi_dot(m_old, xs);
        multi_update(m_old, D, xs, true);
        bool again = false;
        for (int b = 0; b < cnt; ++b) {
          double s2 = 0.0;
          for (int i = 0; i < m_old; ++i) s2 += D[size_t(i) * cnt + b] * D[size_t(i) * cnt + b];
          again = again || before[b] - s2 < 0.5 * before[b];
        }
        if (!again) break;
      }
      for (int b = 0; b < cnt; ++b) {
        if (m >= max_subspace) break;
        DevVec x = std::move(C[c0 + b]);
        double nn = d.dot(x.data(), x.data()).real();
        for (int pass = 0; pass < 2 && added > 0; ++pass) {  // against the corrections taken so far
          d.update_mdot(0, nullptr, nullptr, PN, added, x.data(), cd);
          d.mupdate(PN, added, cd, x.data(), cd + 2 * (added + 1));
          const double now = d.c.fetch(cd + 2 * (added + 1), 1)[0];
          const bool enough = now >= 0.5 * nn;
          nn = now;
          if (enough) break;
        }
        if (!(nn > 1e-20 * std::max(before[b], 1e-300)) || nn == 0.0) continue;
        d.scal(1.0 / std::sqrt(nn), x.data());
        P.set(m, x.data(), d.c.stream);
        PN.set(added, x.data(), d.c.stream);
        V.push_back(std::move(x));
        ++m;
        ++added;
      }
    }
    if (added == 0) break;  // no new direction: stagnated
  }
  if (evecs_out) {
    const size_t es = qk_dtype_size(t);
    std::vector<char> buf(dim * es);
    for (int a = 0; a < n_eig && a < int(U.size()); ++a) {
      if (!U[a].data()) break;
      cuda_check(cudaMemcpyAsync(buf.data(), U[a].data(), dim * es, cudaMemcpyDeviceToHost, d.c.stream), "D2H");
      d.c.sync();
      for (uint64_t i = 0; i < dim; ++i)
        evecs_out[a * dim + i] = t == QK_F64 ? reinterpret_cast<const double*>(buf.data())[i]
                                             : double(reinterpret_cast<const float*>(buf.data())[i]);
    }
  }
  d.c.sync();
  out.seconds = now_s() - t0;
  return out;
}

namespace {
// The three-term recurrence of continued_fraction_coeffs
// (src/solvers/dynamics.cpp:12-59) from step res.alphas.size() up to step
// n_iter: v is the current normalised Lanczos vector, vp the previous one
// (zero before the first step).  Returns true when it stopped on
// beta < 1e-15 (breakdown).  A run split into several calls performs the
// same device operations in the same order as one call.
template <class Real>
bool cf_steps(const Operator& H, Dev& d, DevVec& v, DevVec& vp, DevVec& w, CFOut<Real>& res, int n_iter) {
  const qk_dtype T = d.t;
  PtrArray P(1, H.device());
  P.set(0, w.data(), d.c.stream);
  double* r = d.c.dres(0);
  for (int iter = int(res.alphas.size()); iter < n_iter; ++iter) {
    H.apply_dot(T, v.data(), w.data(), r);
    const Real alpha = Real(d.c.fetch(r, 1)[0]);
    res.alphas.push_back(alpha);
    const void* U[2] = {v.data(), vp.data()};
    const double a[4] = {double(alpha), 0.0, iter > 0 ? double(res.betas.back()) : 0.0, 0.0};
    d.update_mdot(iter > 0 ? 2 : 1, U, a, P, 1, w.data(), r);
    const Real beta = Real(std::sqrt(Real(d.c.fetch(r, 1)[0])));
    if (beta < Real(1e-15)) return true;
    res.betas.push_back(beta);
    d.scale_into(double(Real(1) / beta), w.data(), vp.data());
    std::swap(v, vp);  // v <- w / beta, v_prev <- old v
  }
  return false;
}
}  // namespace

template <class Real>
CFOut<Real> continued_fraction(const Operator& H, const std::complex<Real>* phi0, int n_iter) {
  CFOut<Real> res;
  const uint64_t dim = H.dim();
  if (dim == 0) return res;
  const qk_dtype T = complex_dtype<Real>();
  Dev d(H, T);
  DevVec v = d.vec(false), vp = d.vec(true), w = d.vec(false);
  d.upload<Real>(phi0, v);
  const Real nphi = Real(std::sqrt(Real(d.dot(v.data(), v.data()).real())));
  if (nphi < Real(1e-15)) return res;
  d.scal(double(Real(1) / nphi), v.data());
  res.norm_phi0 = nphi;
  cf_steps<Real>(H, d, v, vp, w, res, n_iter);
  return res;
}

// The continued fraction with a checkpoint of its state (the coefficients
// so far, the norm of phi0, the current and previous Lanczos vectors) read
// from resume_dir and/or written to save_dir as .npy files: alphas.npy,
// betas.npy, norm_phi0.npy, state.npy ([steps, stopped]), v.npy, v_prev.npy
// (complex128).  Resuming and running to n_iter steps gives the same
// coefficients, bit for bit, as one uninterrupted run.
CFOut<double> continued_fraction_checkpointed(const Operator& H, const std::complex<double>* phi0,
                                              const std::string& resume_dir, int n_iter,
                                              const std::string& save_dir) {
  CFOut<double> res;
  const uint64_t dim = H.dim();
  if (dim == 0) return res;
  const qk_dtype T = QK_C128;
  Dev d(H, T);
  DevVec v = d.vec(false), vp = d.vec(true), w = d.vec(false);
  bool stopped = false;
  std::vector<std::complex<double>> hv;
  auto load_vec = [&](const std::string& name, DevVec& dst) {
    std::string descr;
    std::vector<uint64_t> shape;
    std::vector<char> raw = npy_read(resume_dir + "/" + name, descr, shape);
    if (descr != "<c16" || shape.size() != 1 || shape[0] != dim)
      throw std::invalid_argument("qkrylov_b200: checkpoint " + name + " does not match this operator");
    d.upload<double>(reinterpret_cast<const std::complex<double>*>(raw.data()), dst);
  };
  auto load_f8 = [&](const std::string& name) {
    std::string descr;
    std::vector<uint64_t> shape;
    std::vector<char> raw = npy_read(resume_dir + "/" + name, descr, shape);
    if (descr != "<f8") throw std::invalid_argument("qkrylov_b200: checkpoint " + name + " is not float64");
    std::vector<double> out(raw.size() / 8);
    std::memcpy(out.data(), raw.data(), raw.size());
    return out;
  };
  if (!resume_dir.empty()) {
    res.alphas = load_f8("alphas.npy");
    res.betas = load_f8("betas.npy");
    const std::vector<double> nrm = load_f8("norm_phi0.npy"), st = load_f8("state.npy");
    if (nrm.size() != 1 || st.size() != 2 || st[0] != double(res.alphas.size()) ||
        res.betas.size() + (st[1] != 0.0 ? 1 : 0) != res.alphas.size())
      throw std::invalid_argument("qkrylov_b200: inconsistent continued-fraction checkpoint in " + resume_dir);
    res.norm_phi0 = nrm[0];
    stopped = st[1] != 0.0;
    if (res.norm_phi0 < 1e-15) return res;
    load_vec("v.npy", v);
    load_vec("v_prev.npy", vp);
  } else {
    if (!phi0) throw std::invalid_argument("qkrylov_b200: continued fraction needs phi0 or a checkpoint");
    d.upload<double>(phi0, v);
    const double nphi = std::sqrt(d.dot(v.data(), v.data()).real());
    res.norm_phi0 = nphi;
    if (nphi >= 1e-15) d.scal(1.0 / nphi, v.data());
    else stopped = true;
  }
  if (!stopped) stopped = cf_steps<double>(H, d, v, vp, w, res, n_iter);
  if (!save_dir.empty()) {
    npy_write(save_dir + "/alphas.npy", res.alphas.data(), "<f8", {res.alphas.size()});
    npy_write(save_dir + "/betas.npy", res.betas.data(), "<f8", {res.betas.size()});
    npy_write(save_dir + "/norm_phi0.npy", &res.norm_phi0, "<f8", {});
    const double st[2] = {double(res.alphas.size()), stopped ? 1.0 : 0.0};
    npy_write(save_dir + "/state.npy", st, "<f8", {2});
    hv.resize(dim);
    for (const auto& pr : {std::make_pair(&v, "v.npy"), std::make_pair(&vp, "v_prev.npy")}) {
      cuda_check(cudaMemcpyAsync(hv.data(), pr.first->data(), dim * 16, cudaMemcpyDeviceToHost, d.c.stream), "D2H");
      d.c.sync();
      npy_write(save_dir + "/" + pr.second, hv.data(), "<c16", {dim});
    }
  }
  return res;
}

namespace {
// src/solvers/ftlm.cpp:24-53 on a device start vector (not modified).
template <class Real>
void ftlm_tridiag(const Dev& d, const DevVec& start, int n_steps, std::vector<Real>& a,
                  std::vector<Real>& b, DevVec& v, DevVec& vp, DevVec& w, PtrArray& P) {
  const qk_dtype T = d.t;
  qkd_check(qkd_copy(T, d.n, start.data(), v.data(), d.c.stream), "copy");
  normalize<Real>(d, v.data());
  qkd_check(qkd_fill(T, d.n, vp.data(), 0.0, 0.0, d.c.stream), "fill");
  a.clear(); b.clear();
  double* r = d.c.dres(0);
  P.set(0, w.data(), d.c.stream);
  for (int i = 0; i < n_steps; ++i) {
    d.H.apply_dot(T, v.data(), w.data(), r);
    const Real alpha = Real(d.c.fetch(r, 1)[0]);
    a.push_back(alpha);
    const void* U[2] = {v.data(), vp.data()};
    const double co[4] = {double(alpha), 0.0, i > 0 ? double(b.back()) : 0.0, 0.0};
    d.update_mdot(i > 0 ? 2 : 1, U, co, P, 1, w.data(), r);
    const Real beta = Real(std::sqrt(Real(d.c.fetch(r, 1)[0])));
    if (beta < Real(1e-15)) break;
    b.push_back(beta);
    d.scale_into(double(Real(1) / beta), w.data(), vp.data());
    std::swap(v, vp);
  }
}
}  // namespace

template <class Real>
std::vector<FTLMOut<Real>> ftlm(const Operator& H, const std::vector<Real>& betas, int n_random,
                                int n_steps) {
  std::vector<FTLMOut<Real>> out(betas.size());
  for (size_t q = 0; q < betas.size(); ++q) out[q].beta = betas[q];
  const uint64_t dim = H.dim();
  if (dim == 0) return out;
  const qk_dtype T = complex_dtype<Real>();
  Dev d(H, T);
  std::mt19937 rng(42);
  std::normal_distribution<Real> dist(0.0, 1.0);
  std::vector<Real> Z(betas.size(), 0), E(betas.size(), 0), E2(betas.size(), 0);
  DevVec rv = d.vec(false), v = d.vec(false), vp = d.vec(false), w = d.vec(false);
  PtrArray P(1, H.device());
  std::vector<C<Real>> hv(dim);
  std::vector<Real> a, b, ev, fc;
  for (int r = 0; r < n_random; ++r) {
    for (uint64_t i = 0; i < dim; ++i) {
      const Real im = dist(rng);
      const Real re = dist(rng);
      hv[i] = {re, im};
    }
    d.upload<Real>(hv.data(), rv);
    const Real nrm = Real(std::sqrt(Real(d.dot(rv.data(), rv.data()).real())));
    ftlm_tridiag<Real>(d, rv, n_steps, a, b, v, vp, w, P);
    tridiag_first<Real>(a, b, ev, fc);
    for (size_t q = 0; q < betas.size(); ++q) {
      for (size_t i = 0; i < ev.size(); ++i) {
        const Real wgt = nrm * nrm * fc[i] * fc[i] * std::exp(-betas[q] * ev[i]);
        Z[q] += wgt;
        E[q] += ev[i] * wgt;
        E2[q] += ev[i] * ev[i] * wgt;
      }
    }
  }
  for (size_t q = 0; q < betas.size(); ++q) {
    const Real z = Z[q] / Real(n_random), e = E[q] / Real(n_random), e2 = E2[q] / Real(n_random);
    out[q].Z = z;
    out[q].U = e / z;
    out[q].Cv = (betas[q] * betas[q]) * (e2 / z - (e / z) * (e / z));
  }
  return out;
}

template <class Real>
DavidsonOut<Real> davidson(const Operator& H, int n_eig, int max_subspace, Real tol) {
  DavidsonOut<Real> res;
  const uint64_t dim = H.dim();
  if (dim == 0) return res;
  const qk_dtype T = complex_dtype<Real>();
  Dev d(H, T);
  n_eig = int(std::min<uint64_t>(uint64_t(std::max(n_eig, 0)), dim));
  max_subspace = std::max(max_subspace, 2 * n_eig);
  const int dev = H.device();

  DevVec diag = d.vec(false);
  H.diagonal(T, diag.data());
  std::vector<C<Real>> dh;
  d.download<Real>(diag, dh);

  std::mt19937 rng(1234);
  std::uniform_real_distribution<Real> dist(-1.0, 1.0);
  std::vector<uint64_t> idx(dim);
  std::iota(idx.begin(), idx.end(), uint64_t(0));
  // Same comparator and std::sort as the reference, so ties among equal
  // diagonal entries resolve the same way.
  std::sort(idx.begin(), idx.end(), [&](uint64_t i, uint64_t j) { return dh[i].real() < dh[j].real(); });

  const int cap = max_subspace + 2 * n_eig + 2;
  std::vector<DevVec> V, HV;
  PtrArray PV(size_t(cap) * 2, dev);   // [V..., HV...] for residuals
  DevVec coef(size_t(4) * cap + 8, QK_F64, dev);
  double* cd = static_cast<double*>(coef.data());
  auto set_ptrs = [&]() {
    for (size_t i = 0; i < V.size(); ++i) PV.set(i, V[i].data(), d.c.stream);
  };
  // t <- t - sum_v <v, t> v over the current V, twice (classical GS with
  // reorthogonalisation; the reference runs one modified GS sweep).
  auto orthogonalize = [&](DevVec& t) {
    set_ptrs();
    const int m = int(V.size());
    for (int round = 0; round < 2 && m > 0; ++round) {
      d.update_mdot(0, nullptr, nullptr, PV, m, t.data(), cd);
      d.mupdate(PV, m, cd, t.data(), nullptr);
    }
  };
  for (int i = 0; i < n_eig; ++i) {
    DevVec v = d.vec(true);
    const C<Real> one(1, 0);
    cuda_check(cudaMemcpyAsync(static_cast<char*>(v.data()) + idx[i] * sizeof(C<Real>), &one, sizeof(one),
                               cudaMemcpyHostToDevice, d.c.stream), "H2D");
    orthogonalize(v);
    Real nrm = Real(std::sqrt(Real(d.dot(v.data(), v.data()).real())));
    if (nrm < Real(1e-10)) {
      std::vector<C<Real>> hv(dim);
      for (uint64_t j = 0; j < dim; ++j) { const Real im = dist(rng); const Real re = dist(rng); hv[j] = {re, im}; }
      d.upload<Real>(hv.data(), v);
      orthogonalize(v);
      nrm = Real(std::sqrt(Real(d.dot(v.data(), v.data()).real())));
    }
    d.scal(double(Real(1) / nrm), v.data());
    DevVec hv = d.vec(false);
    H.apply(T, v.data(), hv.data());
    V.push_back(std::move(v));
    HV.push_back(std::move(hv));
  }

  std::vector<std::vector<C<Real>>> Hs;  // cached <V_i, HV_j>, i >= j
  for (int iter = 0; iter < 100; ++iter) {
    const int m = int(V.size());
    set_ptrs();
    // Entries involving new vectors; unchanged vectors give the same values.
    if (int(Hs.size()) != m) {
      Hs.assign(m, std::vector<C<Real>>(m));
      for (int j = 0; j < m; ++j) {
        d.update_mdot(0, nullptr, nullptr, PV, m, HV[j].data(), cd);
        const double* h = d.c.fetch(cd, 2 * m);
        for (int i = j; i < m; ++i) {
          Hs[i][j] = C<Real>(Real(h[2 * i]), Real(h[2 * i + 1]));
          if (i != j) Hs[j][i] = std::conj(Hs[i][j]);
        }
      }
    }
    std::vector<C<Real>> Hflat(size_t(m) * m);
    for (int i = 0; i < m; ++i) for (int j = 0; j < m; ++j) Hflat[size_t(i) * m + j] = Hs[i][j];
    std::vector<Real> ev;
    std::vector<C<Real>> es;
    jacobi_hermitian<Real>(Hflat, m, ev, es);

    bool all = true;
    std::vector<DevVec> corr;
    for (int k = 0; k < n_eig; ++k) {
      const Real lam = ev[k];
      // r = sum_i s_i HV_i - lambda s_i V_i
      for (int i = 0; i < m; ++i) PV.set(m + i, HV[i].data(), d.c.stream);
      std::vector<double> nc(4 * size_t(m));
      for (int i = 0; i < m; ++i) {
        const C<Real> s = es[size_t(k) * m + i];
        nc[2 * i] = double(lam * s.real());  nc[2 * i + 1] = double(lam * s.imag());      // -(-lambda s)
        nc[2 * (m + i)] = -double(s.real()); nc[2 * (m + i) + 1] = -double(s.imag());     // -(s)
      }
      cuda_check(cudaMemcpyAsync(cd, nc.data(), sizeof(double) * 4 * m, cudaMemcpyHostToDevice, d.c.stream), "H2D");
      DevVec r = d.vec(true);
      d.mupdate(PV, 2 * m, cd, r.data(), cd + 4 * m);
      const Real rn = Real(std::sqrt(Real(d.c.fetch(cd + 4 * m, 1)[0])));
      if (rn > tol) {
        all = false;
        DevVec t = d.vec(false);
        qkd_check(qkd_dav_precond(T, dim, diag.data(), double(lam), r.data(), t.data(), d.c.stream), "precond");
        corr.push_back(std::move(t));
      }
    }
    if (all || iter == 99) {
      res.iterations = iter + 1;
      res.converged = all;
      for (int k = 0; k < n_eig; ++k) {
        res.eigenvalues.push_back(ev[k]);
        std::vector<double> nc(2 * size_t(m));
        for (int i = 0; i < m; ++i) { nc[2 * i] = -double(es[size_t(k) * m + i].real()); nc[2 * i + 1] = -double(es[size_t(k) * m + i].imag()); }
        cuda_check(cudaMemcpyAsync(cd, nc.data(), sizeof(double) * 2 * m, cudaMemcpyHostToDevice, d.c.stream), "H2D");
        DevVec e = d.vec(true);
        d.mupdate(PV, m, cd, e.data(), nullptr);
        std::vector<C<Real>> he;
        d.download<Real>(e, he);
        res.eigenvectors.push_back(std::move(he));
      }
      return res;
    }
    if (V.size() + corr.size() > size_t(max_subspace)) {
      std::vector<DevVec> nV, nHV;
      for (int i = 0; i < m; ++i) PV.set(m + i, HV[i].data(), d.c.stream);
      for (int k = 0; k < n_eig; ++k) {
        std::vector<double> nc(2 * size_t(m));
        for (int i = 0; i < m; ++i) { nc[2 * i] = -double(es[size_t(k) * m + i].real()); nc[2 * i + 1] = -double(es[size_t(k) * m + i].imag()); }
        cuda_check(cudaMemcpyAsync(cd, nc.data(), sizeof(double) * 2 * m, cudaMemcpyHostToDevice, d.c.stream), "H2D");
        DevVec rv = d.vec(true), rhv = d.vec(true);
        d.mupdate(PV, m, cd, rv.data(), nullptr);
        PtrArray PH(size_t(m), dev);
        for (int i = 0; i < m; ++i) PH.set(i, HV[i].data(), d.c.stream);
        d.mupdate(PH, m, cd, rhv.data(), nullptr);
        d.c.sync();
        nV.push_back(std::move(rv));
        nHV.push_back(std::move(rhv));
      }
      V = std::move(nV);
      HV = std::move(nHV);
      Hs.clear();
    }
    for (auto& t : corr) {
      orthogonalize(t);
      const Real nrm = Real(std::sqrt(Real(d.dot(t.data(), t.data()).real())));
      if (nrm > Real(1e-10)) {
        d.scal(double(Real(1) / nrm), t.data());
        DevVec ht = d.vec(false);
        H.apply(T, t.data(), ht.data());
        V.push_back(std::move(t));
        HV.push_back(std::move(ht));
      }
    }
    if (int(Hs.size()) == m && int(V.size()) != m) {
      // grow the cached projection by the new rows/columns
      const int m2 = int(V.size());
      set_ptrs();
      std::vector<std::vector<C<Real>>> H2(m2, std::vector<C<Real>>(m2));
      for (int i = 0; i < m; ++i) for (int j = 0; j < m; ++j) H2[i][j] = Hs[i][j];
      for (int j = 0; j < m2; ++j) {
        d.update_mdot(0, nullptr, nullptr, PV, m2, HV[j].data(), cd);
        const double* h = d.c.fetch(cd, 2 * m2);
        for (int i = std::max(j, m); i < m2; ++i) {
          H2[i][j] = C<Real>(Real(h[2 * i]), Real(h[2 * i + 1]));
          if (i != j) H2[j][i] = std::conj(H2[i][j]);
        }
      }
      Hs = std::move(H2);
    }
  }
  return res;
}

template <class Real>
Real spectral_function(const Real* alphas, const Real* betas, size_t n, Real norm_phi0, Real omega,
                       Real E0, Real eta) {
  if (n == 0) return Real(0);
  const std::complex<Real> z(omega + E0, eta);
  std::complex<Real> f = Real(0);
  for (int i = int(n) - 1; i >= 0; --i) {
    if (i == int(n) - 1) f = Real(1.0) / (z - alphas[i]);
    else f = Real(1.0) / (z - alphas[i] - betas[i] * betas[i] * f);
  }
  return Real(-1.0 / M_PI * std::imag(norm_phi0 * norm_phi0 * f));
}

#define QKB_INST(R)                                                                                 \
  template void reference_uniform_start<R>(uint64_t, std::vector<std::complex<R>>&);               \
  template LanczosOut<R> lanczos<R>(const Operator&, int, R, const std::complex<R>*,                \
                                    std::vector<std::complex<R>>*);                                 \
  template CFOut<R> continued_fraction<R>(const Operator&, const std::complex<R>*, int);            \
  template std::vector<FTLMOut<R>> ftlm<R>(const Operator&, const std::vector<R>&, int, int);       \
  template DavidsonOut<R> davidson<R>(const Operator&, int, int, R);                                \
  template R spectral_function<R>(const R*, const R*, size_t, R, R, R, R);
QKB_INST(double)
QKB_INST(float)
#undef QKB_INST

}  // namespace qkb
