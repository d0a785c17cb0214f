// Batched coupling sweep: ground states of H(g) = H0 + g H1 for up to 128
// couplings g at once, each column of a row-interleaved block (element
// (i, c) at i*R + c) running its own FP64 Lanczos recurrence, restarted
// from its Ritz vector until the explicit residual |H psi - E psi| / |E| <=
// tol for every column.
//
// One Lanczos step of all columns is two block applies (H0 X and H1 X, the
// row's tables read once for all R columns), one column axpy that forms
// H(g) X = H0 X + diag(g) H1 X with the column dots alpha, and the
// three-term update with fused column norms.  Orthogonality is kept by
// partial reorthogonalisation (H. D. Simon, Math. Comp. 42 (1984) 115-142):
// the host advances Simon's recurrence for the estimates w_{j+1,k} of
// <v_{j+1}, v_k> per column, and when any column's estimate exceeds
// sqrt(eps) every column of the new block (and of the next one) is
// orthogonalised against all stored blocks by classical Gram-Schmidt
// (column-wise multi-dots and multi-updates, a second pass when a column
// loses more than 3/4 of its norm).  This keeps the basis semi-orthogonal,
// which leaves the Ritz values accurate to working precision, at a
// fraction of the traffic of reorthogonalising every step.  The R
// tridiagonals are solved on the host, every few steps.  Columns are
// independent and stop growing (their later vectors are zero) once their
// Ritz residual estimate meets the pass target or their Krylov space is
// exhausted (beta < 1e-15); a column whose explicit residual has met tol is
// locked for the rest of the run, so a converged coupling is never
// disturbed by the steps the others still need.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <stdexcept>

#include "dense.hpp"
#include "solvers.hpp"
#include "warmstart.hpp"

namespace qkb {

namespace {
constexpr double kEps = 2.220446049250313e-16;
constexpr double kOrthoLimit = 1.4901161193847656e-08;  // sqrt(kEps): semi-orthogonality
constexpr int kCheckEvery = 4;  // Lanczos steps between convergence checks
double wall_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
}  // namespace

SweepOut lanczos_sweep(const Operator& H0, const Operator& H1, const std::vector<double>& couplings, int pass_len,
                       int max_passes, double tol, uint64_t seed, WarmStartNet* net) {
  const int nc = int(couplings.size());
  if (nc < 1 || nc > 128) throw std::invalid_argument("qkrylov_b200: 1 to 128 couplings");
  if (pass_len < 2 || pass_len > 128) throw std::invalid_argument("qkrylov_b200: pass_len must be in [2, 128]");
  if (max_passes < 1 || max_passes > 64) throw std::invalid_argument("qkrylov_b200: max_passes must be in [1, 64]");
  if (!(tol > 0)) throw std::invalid_argument("qkrylov_b200: tol must be positive");
  if (H0.dim() != H1.dim() || H0.device() != H1.device())
    throw std::invalid_argument("qkrylov_b200: H0 and H1 must share the basis and the device");
  if (!H0.all_real() || !H1.all_real()) throw std::invalid_argument("qkrylov_b200: the sweep needs real operators");
  if (net && (net->dim() != H0.dim() || net->device() != H0.device()))
    throw std::invalid_argument("qkrylov_b200: the network's basis does not match the operators");
  const double t0 = wall_s();
  const int R = nc <= 32 ? 32 : nc <= 64 ? 64 : 128;
  const qk_dtype t = QK_F64;
  const uint64_t n = H0.dim();
  const int dev = H0.device();
  Context& c = H0.ctx();
  c.activate();
  SweepOut out;
  out.R = R;
  out.energies.assign(nc, 0.0);
  out.residuals.assign(nc, 0.0);
  out.converged.assign(nc, 0);
  if (n == 0) return out;
  const int m = pass_len;
  std::vector<double> g(R, couplings.back());
  std::copy(couplings.begin(), couplings.end(), g.begin());
  DevVec gdev(size_t(R), QK_F64, dev, false);
  cuda_check(cudaMemcpyAsync(gdev.data(), g.data(), sizeof(double) * R, cudaMemcpyHostToDevice, c.stream), "H2D");
  DevVec d0(n, t, dev, false), d1(n, t, dev, false);
  H0.diagonal(t, d0.data());
  H1.diagonal(t, d1.data());
  DevVec psi(n * R, t, dev, false), W(n * R, t, dev, false), Y1;  // Y1: H1 X when it cannot be accumulated
  std::vector<DevVec> V;
  V.reserve(size_t(m) + 1);
  PtrArray P(size_t(m) + 2, dev);
  const size_t G = size_t(qkd_block_partials_grid(n, R));
  const size_t pcap = (size_t(m) + 2) * R * G;
  DevVec part(pcap, QK_F64, dev, false), res(size_t(2) * (m + 2) * R, QK_F64, dev, false),
      res2(size_t(2) * (m + 2) * R, QK_F64, dev, false), nrm(size_t(2) * R, QK_F64, dev, false),
      beta(size_t(R), QK_F64, dev, false), coef(size_t(2) * (m + 1) * R, QK_F64, dev, false);
  DevVec lenv(size_t(R), QK_F32, dev, false);  // R ints for qkd_block_scale
  double* pd = static_cast<double*>(part.data());
  double* rd = static_cast<double*>(res.data());
  double* rd2 = static_cast<double*>(res2.data());
  double* nd = static_cast<double*>(nrm.data());
  double* bd = static_cast<double*>(beta.data());
  double* cd = static_cast<double*>(coef.data());
  int* ld = static_cast<int*>(lenv.data());
  auto fetch = [&](const double* src, size_t count) {
    std::vector<double> h(count);
    cuda_check(cudaMemcpyAsync(h.data(), src, sizeof(double) * count, cudaMemcpyDeviceToHost, c.stream), "D2H");
    c.sync();
    return h;
  };
  // columns of psi normalised; len[] unused here (no column is zero)
  auto normalise = [&](void* X) {
    std::vector<int> big(R, 1 << 30);
    cuda_check(cudaMemcpyAsync(ld, big.data(), sizeof(int) * R, cudaMemcpyHostToDevice, c.stream), "H2D");
    qkd_check(qkd_block_update(c.ws, t, n, R, nullptr, nullptr, nullptr, nullptr, X, nd, c.stream), "norms");
    qkd_check(qkd_block_scale(t, n, R, nd, X, bd, ld, 0, c.stream), "scale");
  };
  qkd_check(qkd_random(t, n * R, seed, 0, psi.data(), c.stream), "random");
  if (net) {
    // learned start vectors: the network's prediction at each coupling
    // (inference included in the run time); padding columns keep random starts
    const double ti = wall_s();
    DevVec phi(n, QK_F32, dev, false);
    for (int col = 0; col < nc; ++col) {
      net->start_vector(couplings[col], static_cast<float*>(phi.data()));
      qkd_check(qkd_block_put_column(QK_F32, phi.data(), n, R, col, t, psi.data(), c.stream), "start column");
    }
    c.sync();
    out.seconds_inference = wall_s() - ti;
  }
  normalise(psi.data());
  qk_plan* p0 = const_cast<qk_plan*>(H0.plan());
  qk_plan* p1 = const_cast<qk_plan*>(H1.plan());
  int lanes = 0;
  if (!qkd_rows_shape(p0, t, R))
    qkd_check(qkd_tune_rows(p0, c.ws, t, R, psi.data(), W.data(), d0.data(), c.stream, &lanes), "tune");
  if (!qkd_rows_shape(p1, t, R)) {  // H1 runs in the accumulating form where its plan has row tables
    const int rc = qkd_tune_rows_acc(p1, c.ws, t, R, psi.data(), W.data(), static_cast<const double*>(gdev.data()),
                                     c.stream, &lanes);
    if (rc != QKD_OK) qkd_check(qkd_tune_rows(p1, c.ws, t, R, psi.data(), W.data(), d1.data(), c.stream, &lanes), "tune");
  }
  out.lanes_per_row = qkd_rows_shape(p0, t, R);
  // Y = H(g) X, dots[2 c] = <X_c, Y_c>: H1 X accumulated into H0 X by the
  // block kernel's epilogue where the plan has row tables, else applied
  // into Y1 and added by a column axpy
  bool fused = true;
  auto apply = [&](const void* X, void* Y, double* dots) {
    qkd_check(qkd_apply_rows(p0, c.ws, t, R, 0, X, Y, d0.data(), nullptr, c.stream), "block apply");
    out.applies += 2;
    if (fused) {
      const int rc = qkd_apply_rows_acc(p1, c.ws, t, R, 0, X, Y, static_cast<const double*>(gdev.data()), dots,
                                        c.stream);
      if (rc == QKD_OK) return;
      if (rc != QKD_EINVAL) qkd_check(rc, "block apply");
      fused = false;
    }
    if (!Y1.data()) Y1 = DevVec(n * R, t, dev, false);
    qkd_check(qkd_apply_rows(p1, c.ws, t, R, 0, X, Y1.data(), d1.data(), nullptr, c.stream), "block apply");
    qkd_check(qkd_block_axpy_cols(t, n, R, static_cast<const double*>(gdev.data()), Y1.data(), Y, X, pd, pcap, dots,
                                  c.stream), "column axpy");
  };
  // a column whose explicit residual has met tol keeps its iterate: it is
  // locked for the rest of the run (padding columns are locked from the start)
  std::vector<int> locked(R, 0);
  for (int col = nc; col < R; ++col) locked[col] = 1;
  for (int pass = 0; pass < max_passes; ++pass) {
    // explicit residuals of the current iterates
    apply(psi.data(), W.data(), rd);
    const std::vector<double> E = fetch(rd, size_t(2) * R);
    P.set(0, psi.data(), c.stream);
    qkd_check(qkd_block_mcomb(t, n, R, 1, P.data(), rd, 1, W.data(), pd, pcap, nd, c.stream), "residual");
    const std::vector<double> r2 = fetch(nd, size_t(2) * R);
    bool all = true;
    for (int col = 0; col < nc; ++col) {
      if (locked[col]) continue;
      out.energies[col] = E[2 * col];
      out.residuals[col] = std::sqrt(r2[2 * col]) / std::abs(E[2 * col]);
      out.converged[col] = out.residuals[col] <= tol;
      locked[col] = out.converged[col];
      all = all && out.converged[col];
    }
    out.passes = pass + 1;
    if (all || pass + 1 == max_passes) break;
    // Lanczos pass of at most m steps from psi
    if (V.empty()) V.emplace_back(n * R, t, dev, false);
    std::swap(V[0], psi);
    P.set(0, V[0].data(), c.stream);
    std::vector<std::vector<double>> a(R), b(R), z(R), om(R), omp(R);
    std::vector<int> len(R, 0);  // steps in each column's tridiagonal
    // stopped: the column's tridiagonal is final (locked, converged in this
    // pass, or Krylov space exhausted); its later vectors are zero
    std::vector<int> stopped(locked);
    for (int col = 0; col < R; ++col)
      if (locked[col]) { a[col] = {0.0}; len[col] = 1; z[col] = {1.0}; }
    std::vector<double> anorm(R, 0.0);
    // rounding level of the orthogonality estimates for vectors of n
    // elements (the sqrt(n) eps / 2 of Larsen's PROPACK)
    const double eps1 = std::sqrt(double(n)) * kEps / 2;
    for (int col = 0; col < R; ++col) om[col] = {1.0};
    {
      std::vector<int> big(R, 1 << 30);
      cuda_check(cudaMemcpyAsync(ld, big.data(), sizeof(int) * R, cudaMemcpyHostToDevice, c.stream), "H2D");
    }
    int steps = 0;
    bool force = false;  // a reorthogonalised step is followed by another one
    for (int j = 0; j < m; ++j) {
      if (int(V.size()) < j + 2) V.emplace_back(n * R, t, dev, false);
      void* Wj = V[j + 1].data();
      P.set(j + 1, Wj, c.stream);
      apply(V[j].data(), Wj, rd2);
      const std::vector<double> al = fetch(rd2, size_t(2) * R);
      // three-term recurrence W -= alpha_j v_j + beta_j v_{j-1}
      std::vector<double> co(size_t(3) * R, 0.0);
      for (int col = 0; col < R; ++col) {
        co[2 * col] = stopped[col] ? 0.0 : al[2 * col];
        co[2 * R + col] = (j > 0 && !stopped[col]) ? b[col][j - 1] : 0.0;
      }
      cuda_check(cudaMemcpyAsync(cd, co.data(), sizeof(double) * co.size(), cudaMemcpyHostToDevice, c.stream), "H2D");
      qkd_check(qkd_block_update(c.ws, t, n, R, V[j].data(), cd, j > 0 ? V[j - 1].data() : nullptr,
                                 j > 0 ? cd + 2 * R : nullptr, Wj, nd, c.stream), "three-term update");
      std::vector<double> after = fetch(nd, size_t(2) * R);
      // orthogonality estimates w_{j+1,k} ~ <v_{j+1}, v_k> (Simon's recurrence)
      std::vector<std::vector<double>> omn(R);
      bool need = force;
      for (int col = 0; col < R; ++col) {
        if (stopped[col]) continue;
        a[col].push_back(al[2 * col]);
        len[col] = j + 1;
        const double bt = std::sqrt(after[2 * col]);
        anorm[col] = std::max(anorm[col], std::abs(al[2 * col]) + bt + (j > 0 ? b[col][j - 1] : 0.0));
        if (bt < 1e-15) continue;
        const std::vector<double>& w = om[col];   // length j + 1
        const std::vector<double>& wp = omp[col]; // length j
        std::vector<double>& wn = omn[col];
        wn.assign(size_t(j) + 2, 0.0);
        const double noise = eps1 * anorm[col];
        for (int k = 0; k < j; ++k) {
          double T = b[col][k] * w[k + 1] + (a[col][k] - a[col][j]) * w[k];
          if (k > 0) T += b[col][k - 1] * w[k - 1];
          if (j > 0) T -= b[col][j - 1] * wp[k];
          T += std::copysign(noise, T);
          wn[k] = T / bt;
          if (std::abs(wn[k]) > kOrthoLimit && col < nc) need = true;
        }
        wn[j] = noise / bt;
        wn[j + 1] = 1.0;
      }
      if (need) {
        // classical Gram-Schmidt of every column against its v_0 .. v_j
        // (a second pass when a column loses more than 3/4 of its norm)
        for (int rep = 0; rep < 2; ++rep) {
          qkd_check(qkd_block_mdot(t, n, R, j + 1, P.data(), Wj, pd, pcap, rd, c.stream), "mdot");
          qkd_check(qkd_block_mcomb(t, n, R, j + 1, P.data(), rd, 1, Wj, pd, pcap, nd, c.stream), "mcomb");
          const std::vector<double> nn = fetch(nd, size_t(2) * R);
          bool again = false;
          for (int col = 0; col < R; ++col)
            if (!stopped[col] && nn[2 * col] < 0.25 * after[2 * col]) again = true;
          after = nn;
          if (!again) break;
        }
        for (int col = 0; col < R; ++col)
          if (!omn[col].empty()) {
            for (int k = 0; k <= j; ++k) omn[col][k] = eps1;
            omn[col][j + 1] = 1.0;
          }
        ++out.reorths;
      }
      force = need && !force;
      ++steps;
      // convergence (lowest Ritz pair of each tridiagonal) every few steps,
      // at the pass limit and when a column's Krylov space is exhausted
      bool check = (j + 1) % kCheckEvery == 0 || j + 1 == m;
      for (int col = 0; col < R; ++col)
        if (!stopped[col] && after[2 * col] < 1e-30) check = true;
      bool done = check;
      for (int col = 0; col < R; ++col) {
        if (stopped[col]) { after[2 * col] = 0.0; continue; }
        const double bt = std::sqrt(after[2 * col]);
        if (check) {
          const double th = tridiag_ground<double>(a[col], b[col], len[col], &z[col]);
          const double est = bt * std::abs(z[col].back()) / std::abs(th);
          if (bt >= 1e-15 && est > 0.1 * tol) done = false;
          else stopped[col] = 1;  // converged within the pass: its Ritz pair is final
        }
        if (bt < 1e-15) stopped[col] = 1;
        if (stopped[col]) { after[2 * col] = 0.0; continue; }
        b[col].push_back(bt);
        omp[col] = std::move(om[col]);
        om[col] = std::move(omn[col]);
      }
      if (done || j + 1 == m) break;
      // V_{j+1} = W / beta; the columns that stopped become zero
      cuda_check(cudaMemcpyAsync(nd, after.data(), sizeof(double) * 2 * R, cudaMemcpyHostToDevice, c.stream), "H2D");
      qkd_check(qkd_block_scale(t, n, R, nd, Wj, bd, ld, j, c.stream), "scale");
    }
    out.steps += steps;
    // psi_c = sum_i z_c[i] V_i[:, c] for i < len_c, then normalised
    int nvec = 0;
    for (int col = 0; col < R; ++col) nvec = std::max(nvec, len[col]);
    std::vector<double> cz(size_t(2) * nvec * R, 0.0);
    for (int col = 0; col < R; ++col)
      for (int i = 0; i < len[col]; ++i) cz[2 * (size_t(i) * R + col)] = -z[col][i];
    cuda_check(cudaMemcpyAsync(cd, cz.data(), sizeof(double) * cz.size(), cudaMemcpyHostToDevice, c.stream), "H2D");
    qkd_check(qkd_block_mcomb(t, n, R, nvec, P.data(), cd, 0, psi.data(), pd, pcap, nullptr, c.stream), "combine");
    normalise(psi.data());
  }
  c.sync();
  out.seconds = wall_s() - t0;
  return out;
}

}  // namespace qkb
