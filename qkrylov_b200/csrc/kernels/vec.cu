// Krylov vector kernels: fills, copies, scalings, axpy, and the FP64
// reductions (dot, multi-vector dot, block update with norm) under the
// solvers.  All are bandwidth-bound streams; element loads are 8/16-byte
// vector loads, grid sizes are fixed multiples of the SM count, and the
// reductions are deterministic (reduce.cuh).
#include <algorithm>
#include <atomic>

#include "reduce.cuh"

namespace qkd {

static std::atomic<uint64_t> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

int sm_count(int device) {
  static int cache[64] = {0};
  if (device < 0 || device >= 64) return 148;
  if (!cache[device]) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || v <= 0) v = 148;
    cache[device] = v;
  }
  return cache[device];
}

namespace {

constexpr int kThreads = 256;

inline int current_device() { int d = 0; cudaGetDevice(&d); return d; }

inline unsigned stream_grid(size_t n, int per_thread = 4) {
  const size_t need = (n + size_t(kThreads) * per_thread - 1) / (size_t(kThreads) * per_thread);
  const size_t cap = size_t(sm_count(current_device())) * 8;
  return unsigned(std::max<size_t>(1, std::min(need, cap)));
}

inline unsigned reduce_grid(size_t n) {
  const size_t need = (n + 2047) / 2048;
  const size_t cap = std::min<size_t>(size_t(sm_count(current_device())) * 4, kMaxG);
  return unsigned(std::max<size_t>(1, std::min(need, cap)));
}

template <int DT>
__global__ void k_fill(size_t n, void* x, double re, double im) {
  using T = VT<DT>;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    T::st(x, i, typename T::R(re), typename T::R(im));
}

template <int DI, int DO>
__global__ void k_convert(size_t n, const void* x, void* y) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
    typename VT<DI>::R re, im;
    VT<DI>::ld(x, i, re, im);
    VT<DO>::st(y, i, typename VT<DO>::R(re), typename VT<DO>::R(im));
  }
}

// y = a x + b y (complex a, b; b = 0 skips reading y)
template <int DT>
__global__ void k_axpby(size_t n, double are, double aim, const void* x, double bre, double bim,
                        void* y, int read_y) {
  using T = VT<DT>;
  using R = typename T::R;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
    R xr, xi, yr = 0, yi = 0;
    T::ld(x, i, xr, xi);
    if (read_y) T::ld_plain(y, i, yr, yi);
    R r = R(are) * xr - R(aim) * xi;
    R m = R(are) * xi + R(aim) * xr;
    if (read_y) { r += R(bre) * yr - R(bim) * yi; m += R(bre) * yi + R(bim) * yr; }
    T::st(y, i, r, m);
  }
}

// x *= a, in place
template <int DT>
__global__ void k_scal(size_t n, double are, double aim, void* x) {
  using T = VT<DT>;
  using R = typename T::R;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
    R xr, xi;
    T::ld_plain(x, i, xr, xi);
    T::st(x, i, R(are) * xr - R(aim) * xi, R(are) * xi + R(aim) * xr);
  }
}

template <int DT>
__global__ void k_normalize_into(size_t n, const double* nrm2, const void* x, void* y) {
  using T = VT<DT>;
  using R = typename T::R;
  const double sc = 1.0 / sqrt(nrm2[0]);
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
    R xr, xi;
    T::ld(x, i, xr, xi);
    T::st(y, i, R(double(xr) * sc), R(double(xi) * sc));
  }
}

struct UPack { const void* u[4]; double ar[4], ai[4]; };

// 16-byte packs: W consecutive elements per lane and load (one complex128,
// two complex64 or float64, four float32).
template <int DT> struct Pk;
template <> struct Pk<QK_C128> {
  using V = double2; static constexpr int W = 1;
  __device__ static void un(const V& v, double* re, double* im) { re[0] = v.x; im[0] = v.y; }
  __device__ static V pk(const double* re, const double* im) { return make_double2(re[0], im[0]); }
};
template <> struct Pk<QK_C64> {
  using V = float4; static constexpr int W = 2;
  __device__ static void un(const V& v, double* re, double* im) { re[0] = v.x; im[0] = v.y; re[1] = v.z; im[1] = v.w; }
  __device__ static V pk(const double* re, const double* im) {
    return make_float4(float(re[0]), float(im[0]), float(re[1]), float(im[1]));
  }
};
template <> struct Pk<QK_F64> {
  using V = double2; static constexpr int W = 2;
  __device__ static void un(const V& v, double* re, double* im) { re[0] = v.x; re[1] = v.y; im[0] = 0.0; im[1] = 0.0; }
  __device__ static V pk(const double* re, const double*) { return make_double2(re[0], re[1]); }
};
template <> struct Pk<QK_F32> {
  using V = float4; static constexpr int W = 4;
  __device__ static void un(const V& v, double* re, double* im) {
    re[0] = v.x; re[1] = v.y; re[2] = v.z; re[3] = v.w; im[0] = im[1] = im[2] = im[3] = 0.0;
  }
  __device__ static V pk(const double* re, const double*) {
    return make_float4(float(re[0]), float(re[1]), float(re[2]), float(re[3]));
  }
};

__device__ __forceinline__ bool al16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// Multi-dot with optional update, out_j = <V_j, x> after x -= sum_m a_m U_m.
// Each warp owns tiles of 32*E packs of 16 bytes: the x tile stays in
// registers (after the update) while the warp streams the matching tiles
// of J vectors V_j at a time, all their loads in flight together, and adds
// the warp-reduced partials to its own slots in shared memory.  The inner
// loop is branch-free: a missing vector (j >= k) reads V_{k-1} with weight
// 0 and a partial tile clamps its pack index with weight 0.  Elements past
// the last whole pack are done by one warp with scalar loads.  If any
// pointer is not 16-byte aligned the same scheme runs on single elements.
template <int DT> struct MdotShape { static constexpr int E = 4, J = 4; };
// 4-byte elements: four per 16-byte pack, so two packs per lane keep the
// 64 loaded values of four vectors within the registers of three CTAs per SM
template <> struct MdotShape<QK_F32> { static constexpr int E = 2, J = 4; };
template <> struct MdotShape<QK_C64> { static constexpr int E = 2, J = 4; };

template <int DT, int W, class LD, class ST>
__device__ __forceinline__ void mdot_tiles(size_t nq, int M, const UPack& U, int k, const void* const* sV,
                                          void* x, double* wacc, LD ld, ST st) {
  constexpr int E = MdotShape<DT>::E, J = MdotShape<DT>::J;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t tile = size_t(32) * E;
  const size_t nwarps = size_t(gridDim.x) * (kThreads / 32);
  for (size_t qb = (size_t(blockIdx.x) * (kThreads / 32) + warp) * tile; qb < nq; qb += nwarps * tile) {
    const bool full = qb + tile <= nq;
    size_t iq[E];
    bool in[E];
    #pragma unroll
    for (int e = 0; e < E; ++e) {
      const size_t q = qb + size_t(e) * 32 + lane;
      in[e] = full || q < nq;
      iq[e] = in[e] ? q : nq - 1;
    }
    double xr[E][W], xi[E][W];
    #pragma unroll
    for (int e = 0; e < E; ++e) ld(x, iq[e], xr[e], xi[e], false);
    if (M > 0) {
      #pragma unroll
      for (int m = 0; m < 4; ++m) {
        if (m >= M) break;
        const double ar = U.ar[m], ai = U.ai[m];
        #pragma unroll
        for (int e = 0; e < E; ++e) {
          double ur[W], ui[W];
          ld(U.u[m], iq[e], ur, ui, true);
          #pragma unroll
          for (int w = 0; w < W; ++w) {
            xr[e][w] -= ar * ur[w] - ai * ui[w];
            xi[e][w] -= ar * ui[w] + ai * ur[w];
          }
        }
      }
      #pragma unroll
      for (int e = 0; e < E; ++e)
        if (in[e]) st(x, iq[e], xr[e], xi[e]);  // rounds xr, xi to the stored values
    }
    #pragma unroll
    for (int e = 0; e < E; ++e)
      if (!in[e]) {
        #pragma unroll
        for (int w = 0; w < W; ++w) { xr[e][w] = 0.0; xi[e][w] = 0.0; }
      }
    for (int j0 = 0; j0 < k; j0 += J) {
      double pr[J], pi[J];
      #pragma unroll
      for (int jj = 0; jj < J; ++jj) {
        const void* vj = sV[j0 + jj < k ? j0 + jj : k - 1];
        pr[jj] = 0.0; pi[jj] = 0.0;
        #pragma unroll
        for (int e = 0; e < E; ++e) {
          double vr[W], vi[W];
          ld(vj, iq[e], vr, vi, true);
          #pragma unroll
          for (int w = 0; w < W; ++w) {
            pr[jj] += vr[w] * xr[e][w] + vi[w] * xi[e][w];
            if (VT<DT>::cplx) pi[jj] += vr[w] * xi[e][w] - vi[w] * xr[e][w];
          }
        }
      }
      #pragma unroll
      for (int jj = 0; jj < J; ++jj) {
        pr[jj] = warp_sum(pr[jj]);
        if (VT<DT>::cplx) pi[jj] = warp_sum(pi[jj]);
      }
      if (lane == 0) {
        #pragma unroll
        for (int jj = 0; jj < J; ++jj)
          if (j0 + jj < k) { wacc[2 * (j0 + jj)] += pr[jj]; wacc[2 * (j0 + jj) + 1] += pi[jj]; }
      }
    }
  }
}

// Three CTAs per SM (at most 85 registers): 24 warps keep the streams of
// vector loads in flight (two CTAs, 102 registers: 4.6 TB/s at 32 float64
// vectors of 16 M elements, long-scoreboard bound).
template <int DT>
__global__ void __launch_bounds__(kThreads, 3)
k_update_mdot(size_t n, int M, UPack U, int k,
              const void* const* __restrict__ V, void* x, double* partials, unsigned* ticket,
              double* out) {
  using T = VT<DT>;
  using R = typename T::R;
  using P = Pk<DT>;
  constexpr int W = P::W;
  extern __shared__ double sacc[];  // [8 warps][k][2], then k pointers
  const void** sV = reinterpret_cast<const void**>(sacc + size_t(kThreads / 32) * k * 2);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* wacc = sacc + size_t(warp) * k * 2;
  for (int j = lane; j < k; j += 32) { wacc[2 * j] = 0.0; wacc[2 * j + 1] = 0.0; }
  bool ok = al16(x);
  for (int m = 0; m < M; ++m) ok = ok && al16(U.u[m]);
  for (int j = threadIdx.x; j < k; j += kThreads) {
    sV[j] = V[j];
    ok = ok && al16(sV[j]);
  }
  ok = __syncthreads_and(ok) != 0;
  if (ok && W > 1) {
    auto ld = [](const void* p, size_t q, double* re, double* im, bool ro) {
      const typename P::V* v = reinterpret_cast<const typename P::V*>(p) + q;
      P::un(ro ? __ldg(v) : *v, re, im);
    };
    auto st = [](void* p, size_t q, double* re, double* im) {
      const typename P::V v = P::pk(re, im);
      reinterpret_cast<typename P::V*>(p)[q] = v;
      P::un(v, re, im);
    };
    const size_t nq = n / W;
    mdot_tiles<DT, W>(nq, M, U, k, sV, x, wacc, ld, st);
    // elements past the last whole pack: one warp, scalar
    if (blockIdx.x == 0 && warp == 0 && nq * W < n) {
      const size_t i = nq * W + lane;
      const bool in = i < n;
      double xr = 0.0, xi = 0.0;
      if (in) {
        R r, m; T::ld_plain(x, in ? i : 0, r, m); xr = r; xi = m;
        for (int mm = 0; mm < M; ++mm) {
          R ur, ui; T::ld(U.u[mm], i, ur, ui);
          xr -= U.ar[mm] * double(ur) - U.ai[mm] * double(ui);
          xi -= U.ar[mm] * double(ui) + U.ai[mm] * double(ur);
        }
        if (M > 0) { T::st(x, i, R(xr), R(xi)); xr = double(R(xr)); xi = double(R(xi)); }
      }
      for (int j = 0; j < k; ++j) {
        double pr = 0.0, pi = 0.0;
        if (in) {
          R vr, vi; T::ld(sV[j], i, vr, vi);
          pr = double(vr) * xr + double(vi) * xi;
          pi = double(vr) * xi - double(vi) * xr;
        }
        pr = warp_sum(pr);
        pi = warp_sum(pi);
        if (lane == 0) { wacc[2 * j] += pr; wacc[2 * j + 1] += pi; }
      }
    }
  } else {
    auto ld = [](const void* p, size_t i, double* re, double* im, bool ro) {
      R r, m;
      if (ro) T::ld(p, i, r, m); else T::ld_plain(p, i, r, m);
      re[0] = r; im[0] = m;
    };
    auto st = [](void* p, size_t i, double* re, double* im) {
      T::st(p, i, R(re[0]), R(im[0]));
      re[0] = double(R(re[0])); im[0] = double(R(im[0]));
    };
    mdot_tiles<DT, 1>(n, M, U, k, sV, x, wacc, ld, st);
  }
  __syncthreads();
  const int G = gridDim.x;
  for (int j = threadIdx.x; j < k; j += kThreads) {
    double re = 0.0, im = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) { re += sacc[(size_t(w) * k + j) * 2]; im += sacc[(size_t(w) * k + j) * 2 + 1]; }
    partials[(size_t(j) * G + blockIdx.x) * 2] = re;
    partials[(size_t(j) * G + blockIdx.x) * 2 + 1] = im;
  }
  grid_finish(partials, ticket, k, out);
}

// x <- x - sum_j c_j V_j, optional ||x||^2.  Coefficients and V_j pointers
// are staged in shared memory; with 16-byte aligned pointers each thread
// handles 16-byte packs, and the j loop is unrolled so several vectors'
// loads are in flight at once.
template <int DT, bool NRM>
__global__ void __launch_bounds__(kThreads)
k_mupdate(size_t n, int k, const void* const* __restrict__ V, const double* __restrict__ c, void* x,
          double* partials, unsigned* ticket, double* nrm2) {
  using T = VT<DT>;
  using R = typename T::R;
  using P = Pk<DT>;
  constexpr int W = P::W;
  extern __shared__ double sc[];  // 2k coefficients, 2*8 reduction scratch, then k pointers
  const void** sV = reinterpret_cast<const void**>(sc + 2 * k + 16);
  bool ok = al16(x);
  for (int j = threadIdx.x; j < 2 * k; j += kThreads) sc[j] = c[j];
  for (int j = threadIdx.x; j < k; j += kThreads) {
    sV[j] = V[j];
    ok = ok && al16(sV[j]);
  }
  ok = __syncthreads_and(ok) != 0;
  double acc = 0.0;
  size_t done = 0;  // elements handled by the pack loop
  if (ok && W > 1) {
    const size_t nq = n / W;
    done = nq * W;
    using PV = typename P::V;
    for (size_t q = blockIdx.x * size_t(kThreads) + threadIdx.x; q < nq; q += size_t(gridDim.x) * kThreads) {
      double xr[W], xi[W];
      P::un(reinterpret_cast<const PV*>(x)[q], xr, xi);
      #pragma unroll 4
      for (int j = 0; j < k; ++j) {
        double vr[W], vi[W];
        P::un(__ldg(reinterpret_cast<const PV*>(sV[j]) + q), vr, vi);
        const double cr = sc[2 * j], ci = sc[2 * j + 1];
        #pragma unroll
        for (int w = 0; w < W; ++w) {
          xr[w] -= cr * vr[w] - ci * vi[w];
          if (T::cplx) xi[w] -= cr * vi[w] + ci * vr[w];
        }
      }
      const PV v = P::pk(xr, xi);
      reinterpret_cast<PV*>(x)[q] = v;
      if (NRM) {
        P::un(v, xr, xi);
        #pragma unroll
        for (int w = 0; w < W; ++w) acc += xr[w] * xr[w] + xi[w] * xi[w];
      }
    }
  }
  for (size_t i = done + blockIdx.x * size_t(kThreads) + threadIdx.x; i < n; i += size_t(gridDim.x) * kThreads) {
    R r0, i0; T::ld_plain(x, i, r0, i0);
    double xr = r0, xi = i0;
    #pragma unroll 8
    for (int j = 0; j < k; ++j) {
      R vr, vi; T::ld(sV[j], i, vr, vi);
      xr -= sc[2 * j] * double(vr) - sc[2 * j + 1] * double(vi);
      if (T::cplx) xi -= sc[2 * j] * double(vi) + sc[2 * j + 1] * double(vr);
    }
    const R sr = R(xr), si = R(xi);
    T::st(x, i, sr, si);
    if (NRM) acc += double(sr) * double(sr) + double(si) * double(si);
  }
  if (NRM) {
    double im = 0.0;
    block_sum2(acc, im, sc + 2 * k);
    if (threadIdx.x == 0) { partials[2 * blockIdx.x] = acc; partials[2 * blockIdx.x + 1] = 0.0; }
    grid_finish(partials, ticket, 1, nrm2);
  }
}

// Many-against-many forms for the block Davidson (real vectors): the
// projections of nx <= 8 vectors X_a onto a tile of up to 8 basis vectors
// V_i in one pass (64 FP64 accumulators per thread), and X_a = (or -=) the
// combinations sum_i c[i][a] V_i of m basis vectors in one pass.  Elements
// are read in pairs (8- or 16-byte loads); a pointer that is not aligned to
// a pair sends the launch through the single-element loop.
constexpr int kMX = 8;  // X vectors per launch
constexpr int kMV = 8;  // V vectors per multi-dot launch

template <int DT> struct Pair;
template <> struct Pair<QK_F64> {
  using V = double2;
  __device__ static void un(const V& v, double& a, double& b) { a = v.x; b = v.y; }
  __device__ static V pk(double a, double b) { return make_double2(a, b); }
};
template <> struct Pair<QK_F32> {
  using V = float2;
  __device__ static void un(const V& v, double& a, double& b) { a = v.x; b = v.y; }
  __device__ static V pk(double a, double b) { return make_float2(float(a), float(b)); }
};

template <int DT>
__global__ void __launch_bounds__(kThreads, 1)
k_multi_dot(size_t n, int mv, const void* const* __restrict__ V, int nx, const void* const* __restrict__ X,
            double* partials, unsigned* ticket, double* out) {
  using T = VT<DT>;
  using R = typename T::R;
  using P = Pair<DT>;
  __shared__ const void* sV[kMV];
  __shared__ const void* sX[kMX];
  __shared__ double red[kThreads / 32][kMV * kMX];
  // tiles shorter than kMV repeat their last vector, and fewer than kMX
  // X vectors repeat the last one: the extra outputs are computed and not used
  bool ok = true;
  if (threadIdx.x < kMV) {
    sV[threadIdx.x] = V[threadIdx.x < mv ? threadIdx.x : mv - 1];
    ok = (reinterpret_cast<uintptr_t>(sV[threadIdx.x]) % sizeof(typename P::V)) == 0;
  } else if (threadIdx.x >= 32 && threadIdx.x < 32 + kMX) {
    const int a = threadIdx.x - 32;
    sX[a] = X[a < nx ? a : nx - 1];
    ok = (reinterpret_cast<uintptr_t>(sX[a]) % sizeof(typename P::V)) == 0;
  }
  ok = __syncthreads_and(ok) != 0;
  double acc[kMV][kMX];
  #pragma unroll
  for (int i = 0; i < kMV; ++i)
    #pragma unroll
    for (int a = 0; a < kMX; ++a) acc[i][a] = 0.0;
  const size_t np = ok ? n / 2 : 0;  // whole pairs
  for (size_t q = blockIdx.x * size_t(kThreads) + threadIdx.x; q < np; q += size_t(gridDim.x) * kThreads) {
    double x0[kMX], x1[kMX];
    #pragma unroll
    for (int a = 0; a < kMX; ++a) P::un(__ldg(reinterpret_cast<const typename P::V*>(sX[a]) + q), x0[a], x1[a]);
    #pragma unroll
    for (int i = 0; i < kMV; ++i) {
      double v0, v1;
      P::un(__ldg(reinterpret_cast<const typename P::V*>(sV[i]) + q), v0, v1);
      #pragma unroll
      for (int a = 0; a < kMX; ++a) acc[i][a] += v0 * x0[a] + v1 * x1[a];
    }
  }
  for (size_t e = 2 * np + blockIdx.x * size_t(kThreads) + threadIdx.x; e < n; e += size_t(gridDim.x) * kThreads) {
    double xe[kMX];
    #pragma unroll
    for (int a = 0; a < kMX; ++a) { R r, m; T::ld(sX[a], e, r, m); xe[a] = double(r); }
    #pragma unroll
    for (int i = 0; i < kMV; ++i) {
      R r, m;
      T::ld(sV[i], e, r, m);
      #pragma unroll
      for (int a = 0; a < kMX; ++a) acc[i][a] += double(r) * xe[a];
    }
  }
  // block sums in a fixed order: warps, then warps' partials in warp order
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  #pragma unroll
  for (int i = 0; i < kMV; ++i)
    #pragma unroll
    for (int a = 0; a < kMX; ++a) {
      const double v = warp_sum(acc[i][a]);
      if (lane == 0) red[warp][i * kMX + a] = v;
    }
  __syncthreads();
  const int G = gridDim.x;
  for (int j = threadIdx.x; j < kMV * kMX; j += kThreads) {
    double sum = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) sum += red[w][j];
    partials[(size_t(j) * G + blockIdx.x) * 2] = sum;
    partials[(size_t(j) * G + blockIdx.x) * 2 + 1] = 0.0;
  }
  grid_finish(partials, ticket, kMV * kMX, out);
}

// X_a = sum_i c[i*nx + a] V_i (acc = 0) or X_a -= sum_i c[i*nx + a] V_i
// (acc = 1), a < nx, i < m; FP64 accumulation.
template <int DT>
__global__ void __launch_bounds__(kThreads)
k_multi_update(size_t n, int m, const void* const* __restrict__ V, const double* __restrict__ c, int nx,
               void* const* __restrict__ X, int acc) {
  using T = VT<DT>;
  using R = typename T::R;
  using P = Pair<DT>;
  extern __shared__ double sm[];  // m*nx coefficients, then m + nx pointers
  double* sc = sm;
  const void** sV = reinterpret_cast<const void**>(sc + size_t(m) * nx);
  void** sX = reinterpret_cast<void**>(sc + size_t(m) * nx + m);
  bool ok = true;
  for (int j = threadIdx.x; j < m * nx; j += kThreads) sc[j] = c[j];
  for (int j = threadIdx.x; j < m; j += kThreads) {
    sV[j] = V[j];
    ok = ok && (reinterpret_cast<uintptr_t>(sV[j]) % sizeof(typename P::V)) == 0;
  }
  for (int a = threadIdx.x; a < kMX; a += kThreads) {
    sX[a] = X[a < nx ? a : nx - 1];
    ok = ok && (reinterpret_cast<uintptr_t>(sX[a]) % sizeof(typename P::V)) == 0;
  }
  ok = __syncthreads_and(ok) != 0;
  const size_t np = ok ? n / 2 : 0;
  for (size_t q = blockIdx.x * size_t(kThreads) + threadIdx.x; q < np; q += size_t(gridDim.x) * kThreads) {
    double x0[kMX], x1[kMX];
    #pragma unroll
    for (int a = 0; a < kMX; ++a) {
      x0[a] = 0.0; x1[a] = 0.0;
      if (acc && a < nx) P::un(reinterpret_cast<const typename P::V*>(sX[a])[q], x0[a], x1[a]);
    }
    // eight basis loads in flight per thread (block Davidson on Hubbard 4x4:
    // 28.1 s with four, 27.1 s with eight, 28.6 s with sixteen)
    #pragma unroll 8
    for (int i = 0; i < m; ++i) {
      double v0, v1;
      P::un(__ldg(reinterpret_cast<const typename P::V*>(sV[i]) + q), v0, v1);
      const double* ci = sc + size_t(i) * nx;
      #pragma unroll
      for (int a = 0; a < kMX; ++a)
        if (a < nx) {
          const double w = acc ? -ci[a] : ci[a];
          x0[a] += w * v0;
          x1[a] += w * v1;
        }
    }
    #pragma unroll
    for (int a = 0; a < kMX; ++a)
      if (a < nx) reinterpret_cast<typename P::V*>(sX[a])[q] = P::pk(x0[a], x1[a]);
  }
  for (size_t e = 2 * np + blockIdx.x * size_t(kThreads) + threadIdx.x; e < n; e += size_t(gridDim.x) * kThreads) {
    double xe[kMX];
    #pragma unroll
    for (int a = 0; a < kMX; ++a) {
      xe[a] = 0.0;
      if (acc && a < nx) { R r, mm; T::ld_plain(sX[a], e, r, mm); xe[a] = double(r); }
    }
    for (int i = 0; i < m; ++i) {
      R r, mm;
      T::ld(sV[i], e, r, mm);
      const double* ci = sc + size_t(i) * nx;
      #pragma unroll
      for (int a = 0; a < kMX; ++a)
        if (a < nx) xe[a] += (acc ? -ci[a] : ci[a]) * double(r);
    }
    #pragma unroll
    for (int a = 0; a < kMX; ++a)
      if (a < nx) T::st(sX[a], e, R(xe[a]), R(0));
  }
}

}  // namespace
}  // namespace qkd

using namespace qkd;

extern "C" {

int qkd_multi_dot(qk_workspace* w, qk_dtype t, size_t n, int m, const void* const* V, int nx, const void* const* X,
                  double* out, cudaStream_t s) {
  if (!w || !V || !X || !out || m <= 0 || nx <= 0 || nx > kMX || (t != QK_F64 && t != QK_F32)) return QKD_EINVAL;
  const unsigned G = std::max(1u, std::min(unsigned(sm_count(current_device())) * 2, unsigned(kMaxG)));
  for (int i0 = 0; i0 < m; i0 += kMV) {
    const int mv = std::min(kMV, m - i0);
    double* o = out + size_t(2) * i0 * kMX;
    if (t == QK_F64) k_multi_dot<QK_F64><<<G, kThreads, 0, s>>>(n, mv, V + i0, nx, X, w->partials, w->ticket, o);
    else k_multi_dot<QK_F32><<<G, kThreads, 0, s>>>(n, mv, V + i0, nx, X, w->partials, w->ticket, o);
    QKD_LAUNCH_CHECK();
  }
  return QKD_OK;
}

int qkd_multi_update(qk_dtype t, size_t n, int m, const void* const* V, const double* c, int nx, void* const* X,
                     int accumulate, cudaStream_t s) {
  if (!V || !c || !X || m <= 0 || m > kMaxK || nx <= 0 || nx > kMX || (t != QK_F64 && t != QK_F32)) return QKD_EINVAL;
  const size_t smem = size_t(m) * nx * sizeof(double) + size_t(m + kMX) * sizeof(void*);
  if (smem > 48 * 1024) return QKD_EINVAL;
  const unsigned G = stream_grid(n, 2);
  if (t == QK_F64) k_multi_update<QK_F64><<<G, kThreads, smem, s>>>(n, m, V, c, nx, X, accumulate ? 1 : 0);
  else k_multi_update<QK_F32><<<G, kThreads, smem, s>>>(n, m, V, c, nx, X, accumulate ? 1 : 0);
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

uint64_t qkd_launch_count(void) { return g_launches.load(); }

int qkd_workspace_create(int device, qk_workspace** out) {
  if (!out) return QKD_EINVAL;
  auto* w = new qk_workspace{};
  w->device = device;
  w->nsm = sm_count(device);
  if (cudaMalloc(&w->partials, sizeof(double) * 2 * kMaxK * kMaxG) != cudaSuccess ||
      cudaMalloc(&w->ticket, sizeof(unsigned)) != cudaSuccess ||
      cudaMalloc(&w->result, sizeof(double) * (2 * kMaxK + 16)) != cudaSuccess) {
    (void)cudaGetLastError();
    cudaFree(w->partials); cudaFree(w->ticket); cudaFree(w->result);
    delete w;
    return QKD_ENOMEM;
  }
  cudaMemset(w->ticket, 0, sizeof(unsigned));
  cudaMemset(w->result, 0, sizeof(double) * (2 * kMaxK + 16));
  *out = w;
  return QKD_OK;
}

int qkd_workspace_destroy(qk_workspace* w) {
  if (!w) return QKD_OK;
  cudaFree(w->partials); cudaFree(w->ticket); cudaFree(w->result);
  delete w;
  return QKD_OK;
}

double* qkd_workspace_results(qk_workspace* w) { return w ? w->result : nullptr; }

int qkd_fill(qk_dtype t, size_t n, void* x, double re, double im, cudaStream_t s) {
  if (n == 0) return QKD_OK;
  if (!x) return QKD_EINVAL;
  QKD_DISPATCH(t, k_fill<DT><<<stream_grid(n), kThreads, 0, s>>>(n, x, re, im));
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

int qkd_copy(qk_dtype t, size_t n, const void* x, void* y, cudaStream_t s) {
  if (n == 0 || x == y) return QKD_OK;
  if (!x || !y) return QKD_EINVAL;
  if (cudaMemcpyAsync(y, x, n * qk_dtype_size(t), cudaMemcpyDeviceToDevice, s) != cudaSuccess) {
    (void)cudaGetLastError();
    return QKD_ECUDA;
  }
  return QKD_OK;
}

int qkd_convert(qk_dtype tin, const void* x, qk_dtype tout, void* y, size_t n, cudaStream_t s) {
  if (n == 0) return QKD_OK;
  if (!x || !y) return QKD_EINVAL;
  if (tin == tout) return qkd_copy(tin, n, x, y, s);
  const unsigned g = stream_grid(n);
#define QKD_CONV(A, B) \
  if (tin == A && tout == B) { k_convert<A, B><<<g, kThreads, 0, s>>>(n, x, y); QKD_LAUNCH_CHECK(); return QKD_OK; }
  QKD_CONV(QK_C128, QK_C64) QKD_CONV(QK_C64, QK_C128) QKD_CONV(QK_F64, QK_F32) QKD_CONV(QK_F32, QK_F64)
  QKD_CONV(QK_F64, QK_C128) QKD_CONV(QK_F32, QK_C64) QKD_CONV(QK_C128, QK_F64) QKD_CONV(QK_C64, QK_F32)
  QKD_CONV(QK_F32, QK_C128) QKD_CONV(QK_C128, QK_F32) QKD_CONV(QK_F64, QK_C64) QKD_CONV(QK_C64, QK_F64)
#undef QKD_CONV
  return QKD_EINVAL;
}

int qkd_scal(qk_dtype t, size_t n, double re, double im, void* x, cudaStream_t s) {
  if (n == 0) return QKD_OK;
  if (!x) return QKD_EINVAL;
  QKD_DISPATCH(t, k_scal<DT><<<stream_grid(n), kThreads, 0, s>>>(n, re, im, x));
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

int qkd_axpy(qk_dtype t, size_t n, double re, double im, const void* x, void* y, cudaStream_t s) {
  return qkd_axpby(t, n, re, im, x, 1.0, 0.0, y, s);
}

int qkd_axpby(qk_dtype t, size_t n, double are, double aim, const void* x, double bre, double bim,
              void* y, cudaStream_t s) {
  if (n == 0) return QKD_OK;
  if (!x || !y) return QKD_EINVAL;
  const int read_y = (bre != 0.0 || bim != 0.0);
  QKD_DISPATCH(t, k_axpby<DT><<<stream_grid(n), kThreads, 0, s>>>(n, are, aim, x, bre, bim, y, read_y));
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

int qkd_update_mdot(qk_workspace* w, qk_dtype t, size_t n, int M, const void* const* U,
                    const double* a, int k, const void* const* V, void* x, double* out,
                    cudaStream_t s) {
  if (!w || !x || !out || M < 0 || M > 4 || k < 0 || k > kMaxK || (M > 0 && (!U || !a)) ||
      (k > 0 && !V))
    return QKD_EINVAL;
  if (k == 0 && M == 0) return QKD_OK;
  UPack up{};
  for (int m = 0; m < M; ++m) { up.u[m] = U[m]; up.ar[m] = a[2 * m]; up.ai[m] = a[2 * m + 1]; }
  const size_t smem = size_t(kThreads / 32) * std::max(k, 1) * 2 * sizeof(double) + size_t(k) * sizeof(void*);
  if (smem > 48 * 1024) {
    QKD_DISPATCH(t, cudaFuncSetAttribute(k_update_mdot<DT>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  }
  // one wave: no more CTAs than are resident at once (a second partial
  // wave would leave most SMs idle at the end)
  QKD_DISPATCH(t, {
    const unsigned G = std::min<unsigned>(reduce_grid(n), resident_grid(k_update_mdot<DT>, kThreads, smem, kMaxG));
    k_update_mdot<DT><<<std::max(1u, G), kThreads, smem, s>>>(n, M, up, k, V, x, w->partials, w->ticket, out);
  });
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

int qkd_dot(qk_workspace* w, qk_dtype t, size_t n, const void* x, const void* y, double* out,
            cudaStream_t s) {
  // <x, y> = one multi-dot with V = {x}; the pointer array lives in the
  // workspace's result scratch tail.
  if (!w || !x || !y || !out) return QKD_EINVAL;
  const void* host_ptr = x;
  void** dev_ptrs = reinterpret_cast<void**>(w->result + 2 * kMaxK + 8);
  if (cudaMemcpyAsync(dev_ptrs, &host_ptr, sizeof(void*), cudaMemcpyHostToDevice, s) != cudaSuccess) {
    (void)cudaGetLastError();
    return QKD_ECUDA;
  }
  // y is only read: pass it as x with M = 0 (no store happens).
  return qkd_update_mdot(w, t, n, 0, nullptr, nullptr, 1, reinterpret_cast<const void* const*>(dev_ptrs),
                         const_cast<void*>(y), out, s);
}

int qkd_mupdate(qk_workspace* w, qk_dtype t, size_t n, int k, const void* const* V,
                const double* c, void* x, double* nrm2, cudaStream_t s) {
  if (!w || !x || k < 0 || k > kMaxK || (k > 0 && (!V || !c))) return QKD_EINVAL;
  const size_t smem = (2 * size_t(k) + 16) * sizeof(double) + size_t(k) * sizeof(void*);
  const unsigned G0 = std::min<unsigned>(reduce_grid(n), kMaxG);
  if (nrm2) {
    QKD_DISPATCH(t, {
      const unsigned G = std::max(1u, std::min(G0, resident_grid(k_mupdate<DT, true>, kThreads, smem, kMaxG)));
      k_mupdate<DT, true><<<G, kThreads, smem, s>>>(n, k, V, c, x, w->partials, w->ticket, nrm2);
    });
  } else {
    if (k == 0) return QKD_OK;
    QKD_DISPATCH(t, {
      const unsigned G = std::max(1u, std::min(G0, resident_grid(k_mupdate<DT, false>, kThreads, smem, kMaxG)));
      k_mupdate<DT, false><<<G, kThreads, smem, s>>>(n, k, V, c, x, w->partials, w->ticket, nrm2);
    });
  }
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

int qkd_normalize_into(qk_dtype t, size_t n, const double* nrm2, const void* x, void* y,
                       cudaStream_t s) {
  if (n == 0) return QKD_OK;
  if (!nrm2 || !x || !y) return QKD_EINVAL;
  QKD_DISPATCH(t, k_normalize_into<DT><<<stream_grid(n), kThreads, 0, s>>>(n, nrm2, x, y));
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- Davidson
// t_i = r_i / (d_i - lambda), the divisor replaced by +-1e-10 when its modulus
// is below 1e-10, and the complex division scaled by the divisor's 1-norm
// (src/solvers/davidson.cpp:171-175).
namespace qkd {
namespace {
template <int DT>
__global__ void k_dav_precond(size_t n, const void* diag, double lambda, const void* r, void* t) {
  using T = VT<DT>;
  using R = typename T::R;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
    R dr, di, rr, ri;
    T::ld(diag, i, dr, di);
    T::ld(r, i, rr, ri);
    R er = dr - R(lambda), ei = di;
    if (sqrt(er * er + ei * ei) < R(1e-10)) { er = (er >= R(0)) ? R(1e-10) : R(-1e-10); ei = R(0); }
    const R s = fabs(er) + fabs(ei);
    const R xr = rr / s, xi = ri / s, yr = er / s, yi = -ei / s;
    const R den = yr * yr + yi * yi;
    T::st(t, i, (xr * yr - xi * yi) / den, (xr * yi + xi * yr) / den);
  }
}
}  // namespace
}  // namespace qkd

extern "C" int qkd_dav_precond(qk_dtype t, size_t n, const void* diag, double lambda, const void* r,
                               void* out, cudaStream_t s) {
  if (n == 0) return QKD_OK;
  if (!diag || !r || !out) return QKD_EINVAL;
  QKD_DISPATCH(t, qkd::k_dav_precond<DT><<<qkd::stream_grid(n), qkd::kThreads, 0, s>>>(n, diag, lambda, r, out));
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

// ------------------------------------------------------ device random vectors
// Counter-based: element i of stream `seed` is a function of (seed, i) only
// (SplitMix64 finaliser, Steele-Lea-Flood 2014), so a vector is reproducible
// for any grid shape.
namespace qkd {
namespace {
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ double unit_sym(uint64_t r) {  // uniform in [-1, 1)
  return double(r >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}
template <int DT>
__global__ void k_random(size_t n, uint64_t seed, int kind, void* x) {
  using T = VT<DT>;
  using R = typename T::R;
  const uint64_t key = mix64(seed ^ 0xD1B54A32D192ED03ull);
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
    const uint64_t a = mix64(key + 2 * i), b = mix64(key + 2 * i + 1);
    if (kind == 0) {
      T::st(x, i, R(unit_sym(a)), R(T::cplx ? unit_sym(b) : 0.0));
    } else {  // Rademacher +-1 on the real part
      T::st(x, i, (a >> 63) ? R(-1) : R(1), R(0));
    }
  }
}

// x (DX) = sum_j c_j V_j (DV), FP64 accumulation, x overwritten.
template <int DV, int DX>
__global__ void k_combine(size_t n, int k, const void* const* __restrict__ V, const double* __restrict__ c, void* x) {
  extern __shared__ double sc[];
  for (int j = threadIdx.x; j < 2 * k; j += blockDim.x) sc[j] = c[j];
  __syncthreads();
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
    double xr = 0.0, xi = 0.0;
    for (int j = 0; j < k; ++j) {
      typename VT<DV>::R vr, vi;
      VT<DV>::ld(V[j], i, vr, vi);
      xr += sc[2 * j] * double(vr) - sc[2 * j + 1] * double(vi);
      xi += sc[2 * j] * double(vi) + sc[2 * j + 1] * double(vr);
    }
    VT<DX>::st(x, i, typename VT<DX>::R(xr), typename VT<DX>::R(xi));
  }
}
}  // namespace
}  // namespace qkd

extern "C" int qkd_random(qk_dtype t, size_t n, uint64_t seed, int kind, void* x, cudaStream_t s) {
  if (n == 0) return QKD_OK;
  if (!x || kind < 0 || kind > 1) return QKD_EINVAL;
  QKD_DISPATCH(t, qkd::k_random<DT><<<qkd::stream_grid(n), qkd::kThreads, 0, s>>>(n, seed, kind, x));
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

extern "C" int qkd_combine(qk_dtype tv, size_t n, int k, const void* const* V, const double* c, qk_dtype tx,
                           void* x, cudaStream_t s) {
  if (n == 0) return QKD_OK;
  if (!V || !c || !x || k <= 0 || k > qkd::kMaxK) return QKD_EINVAL;
  const size_t smem = 2 * size_t(k) * sizeof(double);
  const unsigned g = qkd::stream_grid(n, 1);
#define QKD_COMB(A, B)                                                                          \
  if (tv == A && tx == B) {                                                                     \
    qkd::k_combine<A, B><<<g, qkd::kThreads, smem, s>>>(n, k, V, c, x);                         \
    QKD_LAUNCH_CHECK();                                                                         \
    return QKD_OK;                                                                              \
  }
  QKD_COMB(QK_F32, QK_F64) QKD_COMB(QK_F64, QK_F64) QKD_COMB(QK_F32, QK_F32) QKD_COMB(QK_C64, QK_C128)
  QKD_COMB(QK_C128, QK_C128) QKD_COMB(QK_C64, QK_C64) QKD_COMB(QK_F64, QK_C128) QKD_COMB(QK_F32, QK_C128)
#undef QKD_COMB
  return QKD_EINVAL;
}
