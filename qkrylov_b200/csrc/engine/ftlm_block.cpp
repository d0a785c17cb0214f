// Batched finite-temperature Lanczos: R random vectors advanced together as
// one row-interleaved block (element (i, r) at i*R + r).  The vectors are
// kept unnormalised (v_k = s_k U_k), so every step is two kernels: one
// block H.X (the row's term walk and target ranks shared by all R vectors,
// the diagonal read from a precomputed vector) with fused column dots, and
// one column recurrence with fused FP64 column norms that also produces
// alpha, beta and the next scales.  Nothing returns to the host between
// steps, so the M steps are captured once as a CUDA graph and replayed.  The R tridiagonals then give Z, U and Cv at every
// temperature on the host.  ftlm_loop runs the same random vectors one at
// a time through the single-vector kernels (the baseline).
//
// Thermodynamics (ftlm.cpp:122-170 of qkrylov, with an energy shift): for
// column r with |r|^2 = n_r and tridiagonal eigenpairs (e_i, z_0i),
// w_i = n_r z_0i^2 exp(-beta (e_i - E_min)); Z = exp(-beta E_min) sum w / R,
// U = sum e w / sum w, Cv = beta^2 (sum e^2 w / sum w - U^2).  The shift by
// the lowest Ritz value E_min keeps every exponent <= 0; log Z is reported.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <stdexcept>
#include <thread>

#include "dense.hpp"
#include "solvers.hpp"

namespace qkb {

namespace {
double wall() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Runs f(i) for i in [0, n) on up to the host's hardware threads, each
// thread a contiguous range (every f(i) is independent and computed exactly
// as in a serial loop, so the results do not depend on the thread count).
template <class F>
void parallel_range(int n, F f) {
  const int nth = std::max(1, std::min<int>(n, int(std::thread::hardware_concurrency())));
  if (nth <= 1) { for (int i = 0; i < n; ++i) f(i); return; }
  std::vector<std::thread> th;
  for (int k = 0; k < nth; ++k)
    th.emplace_back([&, k] { for (int i = n * k / nth; i < n * (k + 1) / nth; ++i) f(i); });
  for (auto& t : th) t.join();
}

void thermo(FtlmBlockOut& out, const std::vector<double>& temps) {
  const int R = out.R;
  std::vector<std::vector<double>> ev(R), fc(R);
  // the R tridiagonals' Ritz values and first components (one QL solve
  // each), then every temperature's sums over all Ritz pairs: both on the
  // host's cores (64 solves of 100 steps and 200 x 6,400 weights would
  // otherwise be ~45 ms of host time beside ~0.7 s on the GPU)
  parallel_range(R, [&](int r) {
    const int m = out.len[r];
    std::vector<double> a(out.alphas.begin() + size_t(r) * out.M, out.alphas.begin() + size_t(r) * out.M + m);
    std::vector<double> b(out.betas.begin() + size_t(r) * out.M, out.betas.begin() + size_t(r) * out.M + std::max(m - 1, 0));
    tridiag_first<double>(a, b, ev[r], fc[r]);
  });
  double emin = 1e300;
  for (int r = 0; r < R; ++r)
    for (double e : ev[r]) emin = std::min(emin, e);
  out.e_min = emin;
  const size_t nt = temps.size();
  out.logZ.assign(nt, 0.0); out.U.assign(nt, 0.0); out.Cv.assign(nt, 0.0);
  parallel_range(int(nt), [&](int q) {
    const double beta = 1.0 / temps[q];
    double z = 0.0, e1 = 0.0, e2 = 0.0;
    for (int r = 0; r < R; ++r)
      for (size_t i = 0; i < ev[r].size(); ++i) {
        const double w = out.norm2[r] * fc[r][i] * fc[r][i] * std::exp(-beta * (ev[r][i] - emin));
        z += w; e1 += ev[r][i] * w; e2 += ev[r][i] * ev[r][i] * w;
      }
    const double u = e1 / z;
    out.logZ[q] = std::log(z / R) - beta * emin;
    out.U[q] = u;
    out.Cv[q] = beta * beta * (e2 / z - u * u);
  });
}
}  // namespace

// R three-term Lanczos recurrences (no reorthogonalisation) from the
// columns of B0 (row-interleaved, dtype t, unnormalised; overwritten): M
// steps of block H.X with fused column dots and one column recurrence,
// captured once as a CUDA graph when use_graph.  Fills out.R, M, alphas,
// betas, len, norm2 (|column|^2 of B0), lanes_per_row, graph and
// seconds_device.
static void block_recurrence(const Operator& H, qk_dtype t, int R, int M, DevVec& B0, bool use_graph,
                             FtlmBlockOut& out) {
  out.R = R; out.M = M;
  const uint64_t n = H.dim();
  Context& c = H.ctx();
  const int dev = H.device();
  DevVec B1(n * R, t, dev, false), B2(n * R, t, dev, false);
  DevVec* B[3] = {&B0, &B1, &B2};
  DevVec dots(size_t(M) * 2 * R, QK_F64, dev), alpha(size_t(M) * R, QK_F64, dev), beta(size_t(M) * R, QK_F64, dev),
      scale(size_t(M + 1) * R, QK_F64, dev), nrm(2 * size_t(R), QK_F64, dev), diag(n, t, dev, false);
  DevVec len(size_t(R), QK_F32, dev, false);  // R ints
  std::vector<int> hl(R, M);
  cuda_check(cudaMemcpyAsync(len.data(), hl.data(), sizeof(int) * R, cudaMemcpyHostToDevice, c.stream), "H2D");
  double* dd = static_cast<double*>(dots.data());
  double* al = static_cast<double*>(alpha.data());
  double* bd = static_cast<double*>(beta.data());
  double* sd = static_cast<double*>(scale.data());
  double* nd = static_cast<double*>(nrm.data());
  int* ld = static_cast<int*>(len.data());
  // H's diagonal once (the block apply reads it instead of walking the
  // diagonal terms); column norms of the start block.  The vectors stay
  // unnormalised: v_k = s_k U_k.
  H.diagonal(t, diag.data());
  qkd_check(qkd_block_update(c.ws, t, n, R, nullptr, nullptr, nullptr, nullptr, B0.data(), nd, c.stream), "norms");
  const double* n2 = c.fetch(nd, 2 * R);
  out.norm2.resize(R);
  std::vector<double> s0(R);
  for (int r = 0; r < R; ++r) {
    out.norm2[r] = n2[2 * r];
    s0[r] = n2[2 * r] > 0 ? 1.0 / std::sqrt(n2[2 * r]) : 0.0;
  }
  cuda_check(cudaMemcpyAsync(sd, s0.data(), sizeof(double) * R, cudaMemcpyHostToDevice, c.stream), "H2D");
  qk_plan* plan = const_cast<qk_plan*>(H.plan());
  out.lanes_per_row = qkd_rows_shape(plan, t, R);  // tuned once per operator, dtype and block size
  if (!out.lanes_per_row)
    qkd_check(qkd_tune_rows(plan, c.ws, t, R, B0.data(), B1.data(), diag.data(), c.stream, &out.lanes_per_row),
              "tune");
  auto step = [&](int k) {
    void* U = B[k % 3]->data();
    void* Y = B[(k + 1) % 3]->data();
    void* Up = B[(k + 2) % 3]->data();
    qkd_check(qkd_apply_rows(plan, c.ws, t, R, 0, U, Y, diag.data(), dd + size_t(2) * R * k, c.stream),
              "block apply");
    qkd_check(qkd_block_lanczos(c.ws, t, n, R, U, k > 0 ? Up : nullptr, dd + size_t(2) * R * k,
                                k > 0 ? bd + size_t(R) * (k - 1) : nullptr, k > 0 ? sd + size_t(R) * (k - 1) : nullptr,
                                sd + size_t(R) * k, sd + size_t(R) * (k + 1), Y, al + size_t(R) * k,
                                bd + size_t(R) * k, ld, k, c.stream), "block step");
  };
  cudaEvent_t e0, e1;
  cuda_check(cudaEventCreate(&e0), "event");
  cuda_check(cudaEventCreate(&e1), "event");
  cudaGraphExec_t exec = nullptr;
  if (use_graph) {
    cudaGraph_t g = nullptr;
    cuda_check(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    try {
      for (int k = 0; k < M; ++k) step(k);
    } catch (...) {
      cudaStreamEndCapture(c.stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    cuda_check(cudaStreamEndCapture(c.stream, &g), "end capture");
    const cudaError_t ie = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    cuda_check(ie, "graph instantiate");
    out.graph = true;
  }
  cuda_check(cudaEventRecord(e0, c.stream), "event");
  if (exec) cuda_check(cudaGraphLaunch(exec, c.stream), "graph launch");
  else for (int k = 0; k < M; ++k) step(k);
  cuda_check(cudaEventRecord(e1, c.stream), "event");
  c.sync();
  float ms = 0.f;
  cuda_check(cudaEventElapsedTime(&ms, e0, e1), "event time");
  out.seconds_device = ms * 1e-3;
  if (exec) cudaGraphExecDestroy(exec);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  std::vector<double> ha(size_t(M) * R), hb(size_t(M) * R);
  cuda_check(cudaMemcpy(ha.data(), al, ha.size() * 8, cudaMemcpyDeviceToHost), "D2H");
  cuda_check(cudaMemcpy(hb.data(), bd, hb.size() * 8, cudaMemcpyDeviceToHost), "D2H");
  cuda_check(cudaMemcpy(hl.data(), ld, sizeof(int) * R, cudaMemcpyDeviceToHost), "D2H");
  out.len = hl;
  out.alphas.assign(size_t(R) * M, 0.0);
  out.betas.assign(size_t(R) * M, 0.0);
  for (int r = 0; r < R; ++r)
    for (int k = 0; k < M; ++k) {
      out.alphas[size_t(r) * M + k] = ha[size_t(k) * R + r];
      out.betas[size_t(r) * M + k] = hb[size_t(k) * R + r];
    }
}

FtlmBlockOut ftlm_block(const Operator& H, qk_dtype t, int R, int M, uint64_t seed, const std::vector<double>& temps,
                        bool use_graph) {
  if (R != 32 && R != 64 && R != 128) throw std::invalid_argument("qkrylov_b200: block size must be 32, 64 or 128");
  if (M < 1 || M > 1000) throw std::invalid_argument("qkrylov_b200: n_steps must be in [1, 1000]");
  if (!qk_dtype_complex(t) && !H.all_real()) throw std::invalid_argument("qkrylov_b200: complex operator needs complex vectors");
  for (double T : temps) if (!(T > 0)) throw std::invalid_argument("qkrylov_b200: temperatures must be positive");
  const double t0 = wall();
  FtlmBlockOut out;
  Context& c = H.ctx();
  c.activate();
  DevVec B0(H.dim() * R, t, H.device(), false);
  qkd_check(qkd_random(t, H.dim() * R, seed, 1, B0.data(), c.stream), "random");  // Rademacher start block
  block_recurrence(H, t, R, M, B0, use_graph, out);
  thermo(out, temps);
  out.seconds = wall() - t0;
  return out;
}

FtlmBlockOut cf_block(const Operator& H, qk_dtype t, int R, int M, const void* start, bool use_graph) {
  if (R != 32 && R != 64 && R != 128) throw std::invalid_argument("qkrylov_b200: block size must be 32, 64 or 128");
  if (M < 1 || M > 1000) throw std::invalid_argument("qkrylov_b200: n_steps must be in [1, 1000]");
  if (!start) throw std::invalid_argument("qkrylov_b200: no start block");
  if (!qk_dtype_complex(t) && !H.all_real()) throw std::invalid_argument("qkrylov_b200: complex operator needs complex vectors");
  const double t0 = wall();
  FtlmBlockOut out;
  Context& c = H.ctx();
  c.activate();
  DevVec B0(H.dim() * R, t, H.device(), false);
  qkd_check(qkd_copy(t, H.dim() * R, start, B0.data(), c.stream), "copy");
  block_recurrence(H, t, R, M, B0, use_graph, out);
  out.seconds = wall() - t0;
  return out;
}

FtlmBlockOut ftlm_loop(const Operator& H, qk_dtype t, int R, int M, uint64_t seed, const std::vector<double>& temps,
                       int nvec) {
  if (R < 1 || R > 512 || nvec < 1 || nvec > R || M < 1) throw std::invalid_argument("qkrylov_b200: bad FTLM sizes");
  if (!qk_dtype_complex(t) && !H.all_real()) throw std::invalid_argument("qkrylov_b200: complex operator needs complex vectors");
  for (double T : temps) if (!(T > 0)) throw std::invalid_argument("qkrylov_b200: temperatures must be positive");
  FtlmBlockOut out;
  out.R = nvec; out.M = M;
  const uint64_t n = H.dim();
  Context& c = H.ctx();
  c.activate();
  const int dev = H.device();
  DevVec blk(n * R, t, dev, false);
  qkd_check(qkd_random(t, n * R, seed, 1, blk.data(), c.stream), "random");
  DevVec v(n, t, dev, false), vp(n, t, dev), w(n, t, dev, false);
  PtrArray P(1, dev);
  P.set(0, w.data(), c.stream);
  double* r0 = c.dres(0);
  out.alphas.assign(size_t(nvec) * M, 0.0);
  out.betas.assign(size_t(nvec) * M, 0.0);
  out.len.assign(nvec, M);
  out.norm2.assign(nvec, 0.0);
  c.sync();
  const double t0 = wall();
  for (int r = 0; r < nvec; ++r) {
    qkd_check(qkd_block_column(t, n, R, blk.data(), r, v.data(), c.stream), "column");
    qkd_check(qkd_dot(c.ws, t, n, v.data(), v.data(), r0, c.stream), "dot");
    const double nn = c.fetch(r0, 1)[0];
    out.norm2[r] = nn;
    qkd_check(qkd_scal(t, n, 1.0 / std::sqrt(nn), 0.0, v.data(), c.stream), "scal");
    qkd_check(qkd_fill(t, n, vp.data(), 0.0, 0.0, c.stream), "fill");
    for (int k = 0; k < M; ++k) {
      H.apply_dot(t, v.data(), w.data(), r0);
      const double alpha = c.fetch(r0, 1)[0];
      out.alphas[size_t(r) * M + k] = alpha;
      const void* U[2] = {v.data(), vp.data()};
      const double co[4] = {alpha, 0.0, k > 0 ? out.betas[size_t(r) * M + k - 1] : 0.0, 0.0};
      qkd_check(qkd_update_mdot(c.ws, t, n, k > 0 ? 2 : 1, U, co, 1, P.data(), w.data(), r0, c.stream), "update");
      const double beta = std::sqrt(c.fetch(r0, 1)[0]);
      if (beta < 1e-15) { out.len[r] = k + 1; break; }
      out.betas[size_t(r) * M + k] = beta;
      qkd_check(qkd_axpby(t, n, 1.0 / beta, 0.0, w.data(), 0.0, 0.0, vp.data(), c.stream), "scale");
      std::swap(v, vp);  // v <- w / beta, v_prev <- old v
    }
  }
  c.sync();
  out.seconds_device = wall() - t0;
  thermo(out, temps);
  out.seconds = wall() - t0;
  return out;
}

}  // namespace qkb
