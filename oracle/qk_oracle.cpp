// CPU restatement of qkrylov's matrix-free H.x path and solvers.
// TEST INFRASTRUCTURE ONLY: the parity checker and the timed CPU baseline
// ("port").  Nothing in qkrylov_b200/ links or calls this file.
//
// Each function restates the reference algorithm it cites (paths relative to
// the qkrylov project).  The arithmetic follows the reference's order: the
// pull-mode row sum runs over terms in OpSum order (what the reference's CSR
// row holds), complex products are (ac - bd, ad + bc), dots are
// sum conj(x_i) y_i.  Dot/norm reductions are sequential here, so results
// agree with the reference to rounding, not bit for bit.
#include "qk_oracle.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>
#include <omp.h>

namespace {

using cd = std::complex<double>;
thread_local std::string g_err;

enum Kind { SPIN = 0, FERMION = 1, HUBBARD = 2, TJ = 3 };
enum Op {
  OP_UNKNOWN = -1, SZ, SP, SM, SX, SY,          // spin-1/2
  F_N, F_ID, F_C, F_CDAG,                       // spinless fermion
  H_NUP, H_NDN, H_NUPDN, H_CUP, H_CDAGUP, H_CDN, H_CDAGDN  // Hubbard / t-J
};

Op parse_op(int kind, const std::string& s) {
  switch (kind) {
    case SPIN:
      if (s == "Sz") return SZ; if (s == "Sp") return SP; if (s == "Sm") return SM;
      if (s == "Sx") return SX; if (s == "Sy") return SY; break;
    case FERMION:
      if (s == "N") return F_N; if (s == "Id") return F_ID; if (s == "C") return F_C;
      if (s == "Cdag") return F_CDAG; break;
    case HUBBARD:
    case TJ:
      if (s == "Nup") return H_NUP; if (s == "Ndn") return H_NDN;
      if (kind == HUBBARD && s == "Nupdn") return H_NUPDN;
      if (s == "CUp") return H_CUP; if (s == "CdagUp") return H_CDAGUP;
      if (s == "CDn") return H_CDN; if (s == "CdagDn") return H_CDAGDN; break;
  }
  return OP_UNKNOWN;
}

[[noreturn]] void throw_unknown(int kind, const std::string& s) {
  static const char* names[] = {"spin", "fermion", "Hubbard", "TJ"};
  throw std::runtime_error(std::string("Unknown ") + names[kind] + " operator: " + s);
}

struct Action { bool valid = false; uint64_t st = 0; cd me = 0.0; };

inline int popc(uint64_t x) { return __builtin_popcountll(x); }
// Jordan-Wigner sign from all occupied bits below `bit`
// (fermion_site.cpp:46-57, hubbard_site.cpp:32-46, tj_site.cpp:26-40).
inline double jw(uint64_t st, int bit) {
  const uint64_t m = (1ULL << bit) - 1;
  return (popc(st & m) % 2 == 0) ? 1.0 : -1.0;
}

// One factor acting on the intermediate state.
Action site_apply(int kind, Op op, const std::string& name, int i, uint64_t st) {
  Action a;
  switch (kind) {
    case SPIN: {  // spinhalf_site.cpp:18-121
      const bool up = (st >> i) & 1ULL;
      switch (op) {
        case SZ: a.valid = true; a.st = st; a.me = up ? 0.5 : -0.5; return a;
        case SP: if (up) return a; a.valid = true; a.st = st | (1ULL << i); a.me = 1.0; return a;
        case SM: if (!up) return a; a.valid = true; a.st = st & ~(1ULL << i); a.me = 1.0; return a;
        case SX: a.valid = true; a.st = st ^ (1ULL << i); a.me = 0.5; return a;
        case SY: a.valid = true; a.st = st ^ (1ULL << i);
                 a.me = up ? cd(0.0, -0.5) : cd(0.0, 0.5); return a;
        default: throw_unknown(kind, name);
      }
    }
    case FERMION: {  // fermion_site.cpp:59-111
      const bool occ = (st >> i) & 1ULL;
      switch (op) {
        case F_N: a.valid = true; a.st = st; a.me = occ ? 1.0 : 0.0; return a;
        case F_ID: a.valid = true; a.st = st; a.me = 1.0; return a;
        case F_C: if (!occ) return a; a.valid = true; a.st = st & ~(1ULL << i); a.me = jw(st, i); return a;
        case F_CDAG: if (occ) return a; a.valid = true; a.st = st | (1ULL << i); a.me = jw(st, i); return a;
        default: throw_unknown(kind, name);
      }
    }
    case HUBBARD:
    case TJ: {  // hubbard_site.cpp:48-125, tj_site.cpp:47-113
      const int bu = 2 * i, bd = 2 * i + 1;
      const bool up = (st >> bu) & 1ULL, dn = (st >> bd) & 1ULL;
      const bool tj = (kind == TJ);
      switch (op) {
        case H_NUP: a.valid = true; a.st = st; a.me = up ? 1.0 : 0.0; return a;
        case H_NDN: a.valid = true; a.st = st; a.me = dn ? 1.0 : 0.0; return a;
        case H_NUPDN: a.valid = true; a.st = st; a.me = (up && dn) ? 1.0 : 0.0; return a;
        case H_CUP: if (!up) return a; a.valid = true; a.st = st & ~(1ULL << bu); a.me = jw(st, bu); return a;
        case H_CDAGUP: if (up || (tj && dn)) return a; a.valid = true; a.st = st | (1ULL << bu); a.me = jw(st, bu); return a;
        case H_CDN: if (!dn) return a; a.valid = true; a.st = st & ~(1ULL << bd); a.me = jw(st, bd); return a;
        case H_CDAGDN: if (dn || (tj && up)) return a; a.valid = true; a.st = st | (1ULL << bd); a.me = jw(st, bd); return a;
        default: throw_unknown(kind, name);
      }
    }
  }
  throw std::runtime_error("bad site kind");
}

// ------------------------------------------------------------------ bases
struct Sec { bool use_sz; int sz2; bool use_nup; int nup; bool use_ndn; int ndn; bool use_n; int n; };
Sec read_sec(const int* s) {
  Sec r{};
  if (s) { r.use_sz = s[0]; r.sz2 = s[1]; r.use_nup = s[2]; r.nup = s[3]; r.use_ndn = s[4];
           r.ndn = s[5]; r.use_n = s[6]; r.n = s[7]; }
  return r;
}

// Sector membership as the reference's builders test it
// (spinhalf_basis.cpp:74-104, fermion_basis.cpp:59-89,
//  hubbard_basis.cpp:60-100, tj_basis.cpp:44-96).
struct Member {
  int kind, N; Sec sec; uint64_t upm = 0, dnm = 0;
  Member(int k, int n, Sec s) : kind(k), N(n), sec(s) {
    for (int i = 0; i < N && (kind == HUBBARD || kind == TJ); ++i) {
      upm |= 1ULL << (2 * i); dnm |= 1ULL << (2 * i + 1);
    }
  }
  bool operator()(uint64_t s) const {
    switch (kind) {
      case SPIN: if (!sec.use_sz) return true; { const int nu = popc(s); return nu - (N - nu) == sec.sz2; }
      case FERMION: return !sec.use_n || popc(s) == sec.n;
      case TJ: if ((s & upm) & ((s & dnm) >> 1)) return false; [[fallthrough]];
      case HUBBARD:
        if (kind == HUBBARD && !sec.use_nup && !sec.use_ndn) return true;
        return (!sec.use_nup || popc(s & upm) == sec.nup) && (!sec.use_ndn || popc(s & dnm) == sec.ndn);
    }
    return false;
  }
};

void check_n(int kind, int N) {
  if ((kind == SPIN || kind == FERMION) && (N <= 0 || N > 63))
    throw std::runtime_error(kind == SPIN ? "SpinHalfBasis: N must satisfy 1 <= N <= 63"
                                          : "FermionBasis: N must satisfy 1 <= N <= 63");
  if ((kind == HUBBARD || kind == TJ) && (N <= 0 || N > 31))
    throw std::runtime_error(kind == HUBBARD ? "HubbardBasis: N must satisfy 1 <= N <= 31"
                                             : "TJBasis: N must satisfy 1 <= N <= 31");
}

// Ascending enumeration.  Up to 2^26 candidates the reference's own loop over
// every integer is used; beyond that a depth-first walk from the top bit that
// skips subtrees with no member (same set, same order) keeps t-J N=20 feasible.
void enumerate(int kind, int N, Sec sec, std::vector<uint64_t>& out) {
  check_n(kind, N);
  const int nbits = (kind == HUBBARD || kind == TJ) ? 2 * N : N;
  Member mem(kind, N, sec);
  out.clear();
  if (nbits <= 26) {
    const uint64_t lim = 1ULL << nbits;
    for (uint64_t s = 0; s < lim; ++s) if (mem(s)) out.push_back(s);
    return;
  }
  const bool pair = (kind == HUBBARD || kind == TJ);
  int need_up = -1, need_dn = -1;  // -1: unconstrained
  if (kind == SPIN && sec.use_sz) { if ((sec.sz2 + N) % 2) return; need_up = (sec.sz2 + N) / 2; }
  if (kind == FERMION && sec.use_n) need_up = sec.n;
  if (pair) { if (sec.use_nup) need_up = sec.nup; if (sec.use_ndn) need_dn = sec.ndn; }
  // Recursive walk over sites from the top, values in ascending order.
  struct W {
    int N; bool pair, tj; std::vector<uint64_t>* out;
    void go(int site, uint64_t pre, int ru, int rd) {
      if (site < 0) { if (ru <= 0 && rd <= 0) out->push_back(pre); return; }
      const int rem = site + 1;  // sites left including this one
      if (ru > rem || rd > rem) return;
      if (tj && ru > 0 && rd > 0 && ru + rd > rem) return;
      if (!pair) {
        go(site - 1, pre, ru, rd);
        if (ru != 0) go(site - 1, pre | (1ULL << site), ru > 0 ? ru - 1 : ru, rd);
        return;
      }
      for (int v = 0; v < 4; ++v) {
        const int u = v & 1, d = v >> 1;
        if (tj && u && d) continue;
        if ((u && ru == 0) || (d && rd == 0)) continue;
        go(site - 1, pre | (uint64_t(u) << (2 * site)) | (uint64_t(d) << (2 * site + 1)),
           ru > 0 ? ru - u : ru, rd > 0 ? rd - d : rd);
      }
    }
  } w{N, pair, kind == TJ, &out};
  // encode "unconstrained" as a large negative budget that never reaches 0
  w.go(N - 1, 0, need_up, need_dn);
  if (!pair || true) {
    // the walk treats ru/rd < 0 as unconstrained; filter once more for safety
    std::vector<uint64_t> keep; keep.reserve(out.size());
    for (auto s : out) if (mem(s)) keep.push_back(s);
    out.swap(keep);
  }
}

// ------------------------------------------------------------ Hamiltonian
struct Factor { Op op; std::string name; int site; };
struct Term { cd coeff; std::vector<Factor> f; };
struct Ham {
  int kind, N;
  std::vector<uint64_t> states;
  std::vector<Term> terms;
  int64_t find(uint64_t s) const {  // Basis::contains + Basis::index
    auto it = std::lower_bound(states.begin(), states.end(), s);
    if (it == states.end() || *it != s) return -1;
    return it - states.begin();
  }
  // One term on one ket (matrix_free_hamiltonian.cpp:50-71).  Returns the
  // column (or -1) and conj(amp).
  int64_t entry(uint64_t s0, const Term& t, cd& val) const {
    uint64_t st = s0; cd amp = t.coeff;
    for (const auto& f : t.f) {
      Action a = site_apply(kind, f.op, f.name, f.site, st);
      if (!a.valid) return -1;
      st = a.st; amp *= a.me;
    }
    const int64_t b = find(st);
    if (b < 0) return -1;
    val = cd(amp.real(), -amp.imag());
    return b;
  }
};

inline cd cmul(cd a, cd b) {  // (ac - bd, ad + bc), as Kokkos::complex
  return cd(a.real() * b.real() - a.imag() * b.imag(), a.real() * b.imag() + a.imag() * b.real());
}

void ham_apply(const Ham& H, const cd* x, cd* y) {  // :140-168 without the CSR
  const int64_t dim = H.states.size();
  std::string err; bool bad = false;
  #pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t a = 0; a < dim; ++a) {
    if (bad) continue;
    try {
      cd sum(0.0, 0.0);
      for (const auto& t : H.terms) {
        cd v; const int64_t b = H.entry(H.states[a], t, v);
        if (b >= 0) sum += cmul(v, x[b]);
      }
      y[a] = sum;
    } catch (const std::exception& e) {
      #pragma omp critical
      { bad = true; err = e.what(); }
    }
  }
  if (bad) throw std::runtime_error(err);
}

// ----------------------------------------------------------- vector ops
// include/qkrylov/linalg/vector_ops.hpp:14-137
using Vec = std::vector<cd>;
cd dot(const Vec& x, const Vec& y) {
  double re = 0, im = 0;
  for (size_t i = 0; i < x.size(); ++i) {
    const cd p = cmul(std::conj(x[i]), y[i]);
    re += p.real(); im += p.imag();
  }
  return cd(re, im);
}
double norm(const Vec& x) { return std::sqrt(dot(x, x).real()); }
void scal(cd a, Vec& x) { for (auto& v : x) v = cmul(v, a); }
void axpy(cd a, const Vec& x, Vec& y) { for (size_t i = 0; i < x.size(); ++i) y[i] += cmul(a, x[i]); }
void normalize(Vec& x) { const double n = norm(x); if (n == 0.0) return; scal(cd(1.0 / n, 0.0), x); }
Vec happly(const Ham& H, const Vec& x) { Vec y(x.size()); ham_apply(H, x.data(), y.data()); return y; }

// ----------------------------------------------- small dense eigensolvers
// Implicit-shift QL sweeps of lanczos.cpp:25-98 (identical in ftlm.cpp:61-119).
void tridiag_ql(const std::vector<double>& alpha, const std::vector<double>& beta, int n,
                std::vector<double>& d, std::vector<std::vector<double>>* zout) {
  d = std::vector<double>(alpha.begin(), alpha.begin() + n);
  std::vector<double> e(beta);
  if ((int)e.size() < n) e.resize(n, 0.0);
  std::vector<std::vector<double>> z;
  if (zout) { z.assign(n, std::vector<double>(n, 0.0)); for (int i = 0; i < n; ++i) z[i][i] = 1.0; }
  for (int iter = 0; iter < 1000; ++iter) {
    for (int i = 0; i < n - 1; ++i)
      if (std::abs(e[i]) < 1e-14 * (std::abs(d[i]) + std::abs(d[i + 1]))) e[i] = 0.0;
    int m = n - 1;
    while (m > 0 && e[m - 1] == 0.0) m--;
    if (m == 0) break;
    int l = m - 1;
    while (l > 0 && e[l - 1] != 0.0) l--;
    const double b = (d[m - 1] - d[m]) / 2.0;
    const double c = e[m - 1] * e[m - 1];
    const double s = std::sqrt(b * b + c);
    const double shift = (b > 0) ? d[m] - c / (b + s) : d[m] - c / (b - s);
    double p = d[l] - shift, g = e[l];
    for (int i = l; i < m; ++i) {
      const double r = std::hypot(p, g);
      const double ct = p / r, st = g / r;
      if (i > l) e[i - 1] = r;
      const double f = ct * d[i] + st * e[i];
      const double gn = ct * e[i] + st * d[i + 1];
      const double h = st * d[i] - ct * e[i];
      const double k = st * e[i] - ct * d[i + 1];
      d[i] = ct * f + st * gn;
      e[i] = ct * h + st * k;
      d[i + 1] = st * h - ct * k;
      if (zout)
        for (int j = 0; j < n; ++j) {
          const double z1 = z[j][i], z2 = z[j][i + 1];
          z[j][i] = ct * z1 + st * z2;
          z[j][i + 1] = st * z1 - ct * z2;
        }
      if (i < m - 1) { p = e[i]; g = st * e[i + 1]; e[i + 1] = -ct * e[i + 1]; }
    }
  }
  if (zout) *zout = std::move(z);
}

struct Ground { double energy; std::vector<double> vec; };
Ground tridiag_ground(const std::vector<double>& a, const std::vector<double>& b, int n) {
  if (n == 0) return {0.0, {}};
  if (n == 1) return {a[0], {1.0}};
  std::vector<double> d; std::vector<std::vector<double>> z;
  tridiag_ql(a, b, n, d, &z);
  int mi = 0;
  for (int i = 1; i < n; ++i) if (d[i] < d[mi]) mi = i;
  std::vector<double> v(n);
  for (int i = 0; i < n; ++i) v[i] = z[i][mi];
  return {d[mi], v};
}

// davidson.cpp:22-82
void jacobi(const std::vector<std::vector<cd>>& H, std::vector<double>& evals,
            std::vector<std::vector<cd>>& evecs) {
  const int n = H.size();
  auto A = H;
  std::vector<std::vector<cd>> V(n, std::vector<cd>(n, 0.0));
  for (int i = 0; i < n; ++i) V[i][i] = 1.0;
  for (int iter = 0; iter < 1000; ++iter) {
    double max_off = 0.0; int p = 0, q = 0;
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j)
        if (std::abs(A[i][j]) > max_off) { max_off = std::abs(A[i][j]); p = i; q = j; }
    if (max_off < 1e-15) break;
    const cd app = A[p][p], aqq = A[q][q], apq = A[p][q];
    const double phi = 0.5 * std::atan2(2.0 * std::abs(apq), std::real(app - aqq));
    const cd c = std::cos(phi);
    const cd s = std::sin(phi) * apq / std::abs(apq);
    for (int i = 0; i < n; ++i) {
      const cd vip = V[i][p], viq = V[i][q];
      V[i][p] = c * vip + s * viq;
      V[i][q] = -std::conj(s) * vip + c * viq;
      if (i != p && i != q) {
        const cd aip = A[i][p], aiq = A[i][q];
        A[i][p] = A[p][i] = c * aip + s * aiq;
        A[i][q] = A[q][i] = -std::conj(s) * aip + c * aiq;
      }
    }
    A[p][p] = c * c * app + s * std::conj(s) * aqq + 2.0 * std::real(c * s * std::conj(apq));
    A[q][q] = s * std::conj(s) * app + c * c * aqq - 2.0 * std::real(c * s * std::conj(apq));
    A[p][q] = A[q][p] = 0.0;
  }
  std::vector<int> idx(n);
  for (int i = 0; i < n; ++i) idx[i] = i;
  std::sort(idx.begin(), idx.end(), [&](int i, int j) { return std::real(A[i][i]) < std::real(A[j][j]); });
  evals.clear(); evecs.clear();
  for (int i : idx) {
    evals.push_back(std::real(A[i][i]));
    std::vector<cd> v(n);
    for (int j = 0; j < n; ++j) v[j] = V[j][i];
    evecs.push_back(v);
  }
}

// Kokkos::complex division scaled by the divisor's 1-norm (used by the
// Davidson preconditioner, davidson.cpp:171-175).
cd kdiv(cd x, cd y) {
  const double s = std::fabs(y.real()) + std::fabs(y.imag());
  const cd xs(x.real() / s, x.imag() / s), yc(y.real() / s, -y.imag() / s);
  const double den = yc.real() * yc.real() + yc.imag() * yc.imag();
  const cd r = cmul(xs, yc);
  return cd(r.real() / den, r.imag() / den);
}

template <class F> int guard(F&& f) {
  try { return f(); } catch (const std::exception& e) { g_err = e.what(); return -2; }
}

}  // namespace

extern "C" {

const char* qko_last_error(void) { return g_err.c_str(); }

int qko_site_apply(int kind, const char* op, int site, uint64_t state, int* valid,
                   uint64_t* new_state, double* me) {
  return guard([&] {
    const std::string name(op);
    Action a = site_apply(kind, parse_op(kind, name), name, site, state);
    *valid = a.valid; *new_state = a.st; me[0] = a.me.real(); me[1] = a.me.imag();
    return 0;
  });
}

int64_t qko_basis_count(int kind, int nsites, const int* sec) {
  std::vector<uint64_t> v;
  try { enumerate(kind, nsites, read_sec(sec), v); } catch (const std::exception& e) { g_err = e.what(); return -1; }
  return v.size();
}

int qko_basis_states(int kind, int nsites, const int* sec, uint64_t* out) {
  return guard([&] {
    std::vector<uint64_t> v; enumerate(kind, nsites, read_sec(sec), v);
    std::memcpy(out, v.data(), v.size() * 8); return 0;
  });
}

void* qko_ham_create(int kind, int nsites, const int* sec, int nterms, const double* coef,
                     const int* nfac, const char* const* ops, const int* sites) {
  try {
    auto H = new Ham;
    H->kind = kind; H->N = nsites;
    enumerate(kind, nsites, read_sec(sec), H->states);
    int f = 0;
    for (int t = 0; t < nterms; ++t) {
      Term term; term.coeff = cd(coef[2 * t], coef[2 * t + 1]);
      for (int k = 0; k < nfac[t]; ++k, ++f)
        term.f.push_back({parse_op(kind, ops[f]), ops[f], sites[f]});
      H->terms.push_back(term);
    }
    return H;
  } catch (const std::exception& e) { g_err = e.what(); return nullptr; }
}

void qko_ham_destroy(void* h) { delete static_cast<Ham*>(h); }
uint64_t qko_ham_dim(void* h) { return static_cast<Ham*>(h)->states.size(); }
int qko_ham_states(void* h, uint64_t* out) {
  auto& H = *static_cast<Ham*>(h);
  std::memcpy(out, H.states.data(), H.states.size() * 8);
  return 0;
}

int qko_ham_apply(void* h, const double* x, double* y) {
  return guard([&] {
    ham_apply(*static_cast<Ham*>(h), reinterpret_cast<const cd*>(x), reinterpret_cast<cd*>(y));
    return 0;
  });
}

int64_t qko_ham_coo_count(void* h) {
  auto& H = *static_cast<Ham*>(h);
  int64_t n = 0;
  try {
    for (auto s : H.states) for (const auto& t : H.terms) { cd v; if (H.entry(s, t, v) >= 0) ++n; }
  } catch (const std::exception& e) { g_err = e.what(); return -1; }
  return n;
}

int qko_ham_coo(void* h, int64_t* rows, int64_t* cols, double* vals) {  // :45-91
  return guard([&] {
    auto& H = *static_cast<Ham*>(h);
    int64_t n = 0;
    for (int64_t a = 0; a < (int64_t)H.states.size(); ++a)
      for (const auto& t : H.terms) {
        cd v; const int64_t b = H.entry(H.states[a], t, v);
        if (b < 0) continue;
        rows[n] = a; cols[n] = b; vals[2 * n] = v.real(); vals[2 * n + 1] = v.imag(); ++n;
      }
    return 0;
  });
}

int qko_ham_diagonal(void* h, double* d) {  // :86-89
  return guard([&] {
    auto& H = *static_cast<Ham*>(h);
    for (int64_t a = 0; a < (int64_t)H.states.size(); ++a) {
      cd acc(0.0, 0.0);
      for (const auto& t : H.terms) { cd v; if (H.entry(H.states[a], t, v) == a) acc += v; }
      d[2 * a] = acc.real(); d[2 * a + 1] = acc.imag();
    }
    return 0;
  });
}

int qko_lanczos_start(uint64_t dim, double* v) {
  std::mt19937 rng(1234);
  std::uniform_real_distribution<double> dist(-1.0, 1.0);
  for (uint64_t i = 0; i < dim; ++i) { const double im = dist(rng); const double re = dist(rng); v[2 * i] = re; v[2 * i + 1] = im; }
  return 0;
}

int qko_ftlm_vectors(uint64_t dim, int n_random, double* v) {
  std::mt19937 rng(42);
  std::normal_distribution<double> dist(0.0, 1.0);
  for (int r = 0; r < n_random; ++r)
    for (uint64_t i = 0; i < dim; ++i) {
      const double im = dist(rng); const double re = dist(rng);
      v[2 * (r * dim + i)] = re; v[2 * (r * dim + i) + 1] = im;
    }
  return 0;
}

int qko_lanczos(void* h, int maxiter, double tol, double* energy, int* iters, int* conv,
                double* evec, double* alphas_out, double* betas_out, int* n_alpha, int* n_beta) {
  return guard([&] {
    auto& H = *static_cast<Ham*>(h);
    const int64_t dim = H.states.size();
    *energy = 0; *iters = 0; *conv = 0;
    if (n_alpha) *n_alpha = 0;
    if (n_beta) *n_beta = 0;
    if (dim == 0) return 0;
    Vec v_prev(dim), v_curr(dim), w;
    qko_lanczos_start(dim, reinterpret_cast<double*>(v_curr.data()));
    normalize(v_curr);
    std::vector<Vec> basis{v_curr};
    std::vector<double> alphas, betas;
    bool converged = false; double e_old = 1e100; int actual = 0;
    const int lim = (int)std::min<int64_t>(maxiter, dim);
    for (int iter = 0; iter < lim; ++iter) {
      actual = iter + 1;
      w = happly(H, v_curr);
      const double alpha = dot(v_curr, w).real();
      alphas.push_back(alpha);
      axpy(cd(-alpha, 0.0), v_curr, w);
      if (iter > 0) axpy(cd(-betas.back(), 0.0), v_prev, w);
      for (const auto& bv : basis) axpy(-dot(bv, w), bv, w);
      const double beta = norm(w);
      if (beta < 1e-15) { converged = true; break; }
      if (iter + 1 == lim) break;
      betas.push_back(beta);
      v_prev = v_curr; v_curr = w; scal(cd(1.0 / beta, 0.0), v_curr);
      basis.push_back(v_curr);
      if (iter > 0) {
        const auto tr = tridiag_ground(alphas, betas, alphas.size());
        if (std::abs(tr.energy - e_old) < tol) { e_old = tr.energy; converged = true; break; }
        e_old = tr.energy;
      }
    }
    const auto fin = tridiag_ground(alphas, betas, alphas.size());
    *energy = fin.energy; *iters = actual; *conv = converged;
    if (evec) {
      Vec ritz(dim);
      for (size_t i = 0; i < alphas.size(); ++i) axpy(cd(fin.vec[i], 0.0), basis[i], ritz);
      normalize(ritz);
      std::memcpy(evec, ritz.data(), dim * sizeof(cd));
    }
    if (alphas_out) std::copy(alphas.begin(), alphas.end(), alphas_out);
    if (betas_out) std::copy(betas.begin(), betas.end(), betas_out);
    if (n_alpha) *n_alpha = alphas.size();
    if (n_beta) *n_beta = betas.size();
    return 0;
  });
}

int qko_cf(void* h, const double* phi0, int n_iter, double* alphas, double* betas,
           double* norm_phi0, int* n_alpha, int* n_beta) {
  return guard([&] {
    auto& H = *static_cast<Ham*>(h);
    const int64_t dim = H.states.size();
    *norm_phi0 = 0; *n_alpha = 0; *n_beta = 0;
    if (dim == 0) return 0;
    Vec p(reinterpret_cast<const cd*>(phi0), reinterpret_cast<const cd*>(phi0) + dim);
    const double nphi = norm(p);
    if (nphi < 1e-15) return 0;
    Vec v_curr = p, v_prev(dim), w;
    scal(cd(1.0 / nphi, 0.0), v_curr);
    *norm_phi0 = nphi;
    std::vector<double> a, b;
    for (int iter = 0; iter < n_iter; ++iter) {
      w = happly(H, v_curr);
      const double alpha = dot(v_curr, w).real();
      a.push_back(alpha);
      axpy(cd(-alpha, 0.0), v_curr, w);
      if (iter > 0) axpy(cd(-b.back(), 0.0), v_prev, w);
      const double beta = norm(w);
      if (beta < 1e-15) break;
      b.push_back(beta);
      v_prev = v_curr; v_curr = w; scal(cd(1.0 / beta, 0.0), v_curr);
    }
    std::copy(a.begin(), a.end(), alphas); std::copy(b.begin(), b.end(), betas);
    *n_alpha = a.size(); *n_beta = b.size();
    return 0;
  });
}

double qko_spectral(const double* alphas, const double* betas, size_t n, double norm_phi0,
                    double omega, double E0, double eta) {
  if (n == 0) return 0.0;
  const cd z(omega + E0, eta);
  cd f = 0.0;
  for (int i = (int)n - 1; i >= 0; --i) {
    if (i == (int)n - 1) f = 1.0 / (z - alphas[i]);
    else f = 1.0 / (z - alphas[i] - betas[i] * betas[i] * f);
  }
  return -1.0 / M_PI * std::imag(norm_phi0 * norm_phi0 * f);
}

namespace {
// ftlm.cpp:24-53
void ftlm_tridiag(const Ham& H, const Vec& start, int n_steps, std::vector<double>& a,
                  std::vector<double>& b) {
  const int64_t dim = H.states.size();
  Vec v_curr = start, v_prev(dim), w;
  normalize(v_curr);
  a.clear(); b.clear();
  for (int i = 0; i < n_steps; ++i) {
    w = happly(H, v_curr);
    const double alpha = dot(v_curr, w).real();
    a.push_back(alpha);
    axpy(cd(-alpha, 0.0), v_curr, w);
    if (i > 0) axpy(cd(-b.back(), 0.0), v_prev, w);
    const double beta = norm(w);
    if (beta < 1e-15) break;
    b.push_back(beta);
    v_prev = v_curr; v_curr = w; scal(cd(1.0 / beta, 0.0), v_curr);
  }
}
}  // namespace

int qko_ftlm_tridiag(void* h, const double* v_start, int n_steps, double* alphas, double* betas,
                     int* n_alpha, int* n_beta) {
  return guard([&] {
    auto& H = *static_cast<Ham*>(h);
    const int64_t dim = H.states.size();
    Vec s(reinterpret_cast<const cd*>(v_start), reinterpret_cast<const cd*>(v_start) + dim);
    std::vector<double> a, b;
    ftlm_tridiag(H, s, n_steps, a, b);
    std::copy(a.begin(), a.end(), alphas); std::copy(b.begin(), b.end(), betas);
    *n_alpha = a.size(); *n_beta = b.size();
    return 0;
  });
}

int qko_tridiag_eig(const double* alphas, const double* betas, int n, double* evals,
                    double* first_comp) {
  return guard([&] {
    if (n == 0) return 0;
    if (n == 1) { evals[0] = alphas[0]; if (first_comp) first_comp[0] = 1.0; return 0; }
    std::vector<double> a(alphas, alphas + n), b(betas, betas + n - 1), d;
    std::vector<std::vector<double>> z;
    tridiag_ql(a, b, n, d, &z);
    for (int i = 0; i < n; ++i) { evals[i] = d[i]; if (first_comp) first_comp[i] = z[0][i]; }
    return 0;
  });
}

int qko_jacobi_eig(const double* Hm, int n, double* evals, double* evecs) {
  return guard([&] {
    std::vector<std::vector<cd>> A(n, std::vector<cd>(n));
    for (int i = 0; i < n; ++i) for (int j = 0; j < n; ++j) A[i][j] = cd(Hm[2 * (i * n + j)], Hm[2 * (i * n + j) + 1]);
    std::vector<double> ev; std::vector<std::vector<cd>> V;
    jacobi(A, ev, V);
    for (int k = 0; k < n; ++k) {
      evals[k] = ev[k];
      for (int j = 0; j < n; ++j) { evecs[2 * (k * n + j)] = V[k][j].real(); evecs[2 * (k * n + j) + 1] = V[k][j].imag(); }
    }
    return 0;
  });
}

int qko_ftlm(void* h, double beta, int n_random, int n_steps, double* Zo, double* Uo, double* Cvo) {
  return guard([&] {
    auto& H = *static_cast<Ham*>(h);
    const int64_t dim = H.states.size();
    *Zo = 0; *Uo = 0; *Cvo = 0;
    if (dim == 0) return 0;
    std::mt19937 rng(42);
    std::normal_distribution<double> dist(0.0, 1.0);
    double Z = 0, E = 0, E2 = 0;
    for (int r = 0; r < n_random; ++r) {
      Vec rv(dim);
      for (int64_t i = 0; i < dim; ++i) { const double im = dist(rng); const double re = dist(rng); rv[i] = cd(re, im); }
      const double nrm = norm(rv);
      std::vector<double> a, b;
      ftlm_tridiag(H, rv, n_steps, a, b);
      // diagonalize_tridiag_components (ftlm.cpp:61-119)
      const int n = a.size();
      std::vector<double> ev, fc;
      if (n == 1) { ev = {a[0]}; fc = {1.0}; }
      else if (n > 1) {
        std::vector<double> d; std::vector<std::vector<double>> z;
        tridiag_ql(a, b, n, d, &z);
        for (int i = 0; i < n; ++i) { ev.push_back(d[i]); fc.push_back(z[0][i]); }
      }
      for (size_t i = 0; i < ev.size(); ++i) {
        const double w = nrm * nrm * fc[i] * fc[i] * std::exp(-beta * ev[i]);
        Z += w; E += ev[i] * w; E2 += ev[i] * ev[i] * w;
      }
    }
    Z /= n_random; E /= n_random; E2 /= n_random;
    *Zo = Z; *Uo = E / Z; *Cvo = (beta * beta) * (E2 / Z - (E / Z) * (E / Z));
    return 0;
  });
}

int qko_davidson(void* h, int n_eig, int max_subspace, double tol, double* evals, double* evecs,
                 int* n_out, int* iters, int* conv) {
  return guard([&] {
    auto& H = *static_cast<Ham*>(h);
    const int64_t dim = H.states.size();
    *n_out = 0; *iters = 0; *conv = 0;
    if (dim == 0) return 0;
    n_eig = (int)std::min<int64_t>(n_eig, dim);
    max_subspace = std::max(max_subspace, 2 * n_eig);
    std::vector<double> dg(2 * dim);
    qko_ham_diagonal(h, dg.data());
    std::vector<Vec> V, HV;
    std::mt19937 rng(1234);
    std::uniform_real_distribution<double> dist(-1.0, 1.0);
    std::vector<int64_t> idx(dim);
    for (int64_t i = 0; i < dim; ++i) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](int64_t i, int64_t j) { return dg[2 * i] < dg[2 * j]; });
    for (int i = 0; i < n_eig; ++i) {
      Vec v(dim); v[idx[i]] = 1.0;
      for (const auto& vp : V) axpy(-dot(vp, v), vp, v);
      double nrm = norm(v);
      if (nrm < 1e-10) {
        for (int64_t j = 0; j < dim; ++j) { const double im = dist(rng); const double re = dist(rng); v[j] = cd(re, im); }
        for (const auto& vp : V) axpy(-dot(vp, v), vp, v);
        nrm = norm(v);
      }
      scal(cd(1.0 / nrm, 0.0), v);
      V.push_back(v); HV.push_back(happly(H, v));
    }
    for (int iter = 0; iter < 100; ++iter) {
      const int m = V.size();
      std::vector<std::vector<cd>> Hs(m, std::vector<cd>(m));
      for (int i = 0; i < m; ++i)
        for (int j = 0; j <= i; ++j) { Hs[i][j] = dot(V[i], HV[j]); if (i != j) Hs[j][i] = std::conj(Hs[i][j]); }
      std::vector<double> ev; std::vector<std::vector<cd>> es;
      jacobi(Hs, ev, es);
      bool all = true; std::vector<Vec> corr;
      for (int k = 0; k < n_eig; ++k) {
        const double lam = ev[k]; const auto& s = es[k];
        Vec r(dim);
        for (int i = 0; i < m; ++i) {
          axpy(s[i], HV[i], r);
          axpy(cd(-lam * s[i].real(), -lam * s[i].imag()), V[i], r);
        }
        const double rn = norm(r);
        if (rn > tol) {
          all = false;
          Vec t(dim);
          for (int64_t i = 0; i < dim; ++i) {
            cd diff(dg[2 * i] - lam, dg[2 * i + 1]);
            if (std::hypot(diff.real(), diff.imag()) < 1e-10) diff = (diff.real() >= 0) ? 1e-10 : -1e-10;
            t[i] = kdiv(r[i], diff);
          }
          corr.push_back(t);
        }
      }
      if (all || iter == 99) {
        *iters = iter + 1; *conv = all; *n_out = n_eig;
        for (int k = 0; k < n_eig; ++k) {
          evals[k] = ev[k];
          if (evecs) {
            Vec e(dim);
            for (int i = 0; i < m; ++i) axpy(es[k][i], V[i], e);
            std::memcpy(evecs + 2 * k * dim, e.data(), dim * sizeof(cd));
          }
        }
        return 0;
      }
      if (V.size() + corr.size() > (size_t)max_subspace) {
        std::vector<Vec> nV, nHV;
        for (int k = 0; k < n_eig; ++k) {
          Vec rv(dim), rhv(dim);
          for (int i = 0; i < m; ++i) { axpy(es[k][i], V[i], rv); axpy(es[k][i], HV[i], rhv); }
          nV.push_back(rv); nHV.push_back(rhv);
        }
        V = nV; HV = nHV;
      }
      for (auto& t : corr) {
        for (const auto& v : V) axpy(-dot(v, t), v, t);
        const double nrm = norm(t);
        if (nrm > 1e-10) { scal(cd(1.0 / nrm, 0.0), t); V.push_back(t); HV.push_back(happly(H, t)); }
      }
    }
    return 0;
  });
}

}  // extern "C"
