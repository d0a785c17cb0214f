// Matrix-free H.x: pull mode, no atomics.
//
// Rows are processed in tiles of up to 256 consecutive states of one sector
// block (fixed high part h), one thread per row.  A thread rebuilds its state
// s = (h << L) | llist[...] from the sector tables, evaluates every compiled
// term group of the operator (terms and groups staged in shared memory), and
// for each group with a valid term gathers x at the target's rank
// A[t >> L] + B[t & lmask].  Consecutive rows of a tile have consecutive low
// parts, so for every term that only flips high bits the warp's gathers are
// consecutive addresses (coalesced); terms that flip low bits stay inside
// the block, which L1 holds.  Each thread writes only its own y[row].
#include <algorithm>
#include <vector>

#include "reduce.cuh"
#include "../engine/sector.hpp"

namespace qkd {
struct SpinHandle;
SpinHandle* spin_plan_create(const qk_plan_desc* d, size_t* dev_bytes);
SpinHandle* gen_plan_create(const qk_plan_desc* d, size_t* dev_bytes);
struct PairHandle;
PairHandle* pair_plan_create(const qk_plan_desc* d, const uint64_t* A_dev, const uint32_t* B_dev,
                             const double* diag_ref, size_t* dev_bytes);
void pair_plan_destroy(PairHandle* h);
int pair_apply(const PairHandle* h, qk_dtype t, const void* x, void* y, cudaStream_t s, qk_workspace* w,
               double* dot_out);
bool spin_plan_is_gen(const SpinHandle* h);
int spin_plan_set_diag(SpinHandle* h, const double* diag);
int spin_apply_block(const SpinHandle* h, qk_dtype t, int R, int lpr, const void* X, void* Y, double* dots,
                     cudaStream_t s, qk_workspace* w, const double* gacc = nullptr, int tilec = 0);
void spin_plan_destroy(SpinHandle* h);
void spin_set_die_queues(bool on);
int spin_apply_range(const SpinHandle* h, qk_dtype t, const void* x, void* y, cudaStream_t s, uint64_t row_lo,
                     uint64_t row_hi);
int spin_apply(const SpinHandle* h, qk_dtype t, const void* x, void* y, cudaStream_t s, qk_workspace* w,
               double* dot_out);
}  // namespace qkd

static int g_kernel_policy = 0;  // 0: specialised kernels where eligible, 1: generic only
static bool g_pair_path = true;  // the spin-product path of Hubbard-type operators

struct qk_plan {
  qkd::SpinHandle* spin = nullptr;
  qkd::PairHandle* pair = nullptr;  // spin-product path (Hubbard-type operators), or null
  int device;
  int nbits, L;
  uint64_t dim, lmask;
  uint64_t* A;
  uint32_t* B;
  uint32_t* llist;
  qk_term_t* terms;
  qk_group_t* groups;
  qk_tile_t* tiles;
  uint32_t nterms, ngroups, ntiles;
  int has_diag, all_real;
  size_t bytes, smem;
  int rows_lpr[4][3];   // autotuned lanes per row of the block apply, by dtype and R = 32, 64, 128
  int rows_tile[4][3];  // autotuned tile shape of the block apply (row kernels: 256 / 128 / 512 rows)
  float rows_ms[4][3][9];  // the tuner's fastest launch (ms) per lanes per row (32/16/8) x tile code; 0: untimed
  double* diag_re;     // real diagonal (generic-kernel operators with a real diagonal), else null
};

namespace qkd {
namespace {

constexpr int kTile = 256;

struct DevPlan {
  int L;
  uint64_t lmask;
  const double* __restrict__ diag_re;
  const uint64_t* __restrict__ A;
  const uint32_t* __restrict__ B;
  const uint32_t* __restrict__ llist;
  const qk_term_t* __restrict__ terms;
  const qk_group_t* __restrict__ groups;
  const qk_tile_t* __restrict__ tiles;
  uint32_t nterms, ngroups, ntiles;
  int has_diag;
  uint64_t row_lo, row_hi;  // rows computed by k_hx: [row_lo, row_hi) (tiles never straddle a block)
};

DevPlan dev(const qk_plan* p, uint64_t row_lo = 0, uint64_t row_hi = ~0ull) {
  return DevPlan{p->L, p->lmask, p->diag_re, p->A, p->B, p->llist, p->terms, p->groups, p->tiles,
                 p->nterms, p->ngroups, p->ntiles, p->has_diag, row_lo, row_hi};
}

// Sum of the valid terms of one group on state s: returns false when none is valid.
template <bool CC, class R>
__device__ __forceinline__ bool group_coef(const qk_term_t* t, uint32_t first, uint32_t count,
                                           uint64_t s, R& cr, R& ci) {
  bool any = false;
  cr = R(0); ci = R(0);
  for (uint32_t q = first; q < first + count; ++q) {
    const qk_term_t term = t[q];
    if ((s & term.cmask) != term.cval) continue;
    any = true;
    const bool neg = __popcll(s & term.smask) & 1;
    const R wr = R(term.wre);
    cr += neg ? -wr : wr;
    if (CC) { const R wi = R(term.wim); ci += neg ? -wi : wi; }
  }
  return any;
}

__device__ __forceinline__ void stage_plan(const DevPlan& p, qk_term_t*& st, qk_group_t*& sg) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  st = reinterpret_cast<qk_term_t*>(smem_raw);
  sg = reinterpret_cast<qk_group_t*>(smem_raw + size_t(p.nterms) * sizeof(qk_term_t));
  for (uint32_t i = threadIdx.x; i < p.nterms; i += blockDim.x) st[i] = p.terms[i];
  for (uint32_t i = threadIdx.x; i < p.ngroups; i += blockDim.x) sg[i] = p.groups[i];
  __syncthreads();
}

// y = H x for one row; returns (y_re, y_im) and the row's own x element.
// The diagonal comes from the plan's precomputed real diagonal when it has
// one, else from the diagonal term group.  Off-diagonal groups are taken
// kGB at a time: their coefficients and targets first, then all of their
// gathers together, so up to kGB loads of x are in flight per row.
constexpr int kGB = 8;
template <int DT, bool CC>
__device__ __forceinline__ void row_apply(const DevPlan& p, const qk_term_t* st, const qk_group_t* sg,
                                          uint64_t row, uint64_t s, const void* x,
                                          typename VT<DT>::R& yr, typename VT<DT>::R& yi,
                                          typename VT<DT>::R& xr0, typename VT<DT>::R& xi0) {
  using T = VT<DT>;
  using R = typename T::R;
  yr = R(0); yi = R(0);
  T::ld(x, row, xr0, xi0);
  uint32_t g0 = 0;
  if (p.has_diag) {
    R cr = R(0), ci = R(0);
    bool any = true;
    if (p.diag_re) cr = R(__ldg(p.diag_re + row));
    else any = group_coef<CC, R>(st, sg[0].first, sg[0].count, s, cr, ci);
    if (any) {
      yr += cr * xr0;
      if (T::cplx) {
        yi += cr * xi0;
        if (CC) { yr -= ci * xi0; yi += ci * xr0; }
      }
    }
    g0 = 1;
  }
  for (uint32_t gb = g0; gb < p.ngroups; gb += kGB) {
    uint64_t col[kGB];
    R cr[kGB], ci[kGB];
    bool ok[kGB];
    #pragma unroll
    for (int b = 0; b < kGB; ++b) {
      const uint32_t g = gb + b;
      ok[b] = false; col[b] = row; cr[b] = R(0); ci[b] = R(0);
      if (g < p.ngroups) {
        const qk_group_t grp = sg[g];
        if (group_coef<CC, R>(st, grp.first, grp.count, s, cr[b], ci[b])) {
          const uint64_t t = s ^ grp.flip;
          const uint64_t a = __ldg(p.A + (t >> p.L));
          const uint32_t bb = __ldg(p.B + (t & p.lmask));
          // Membership is re-checked for every group (one byte compare), so a
          // gather index is always a valid row even where the compiler proved
          // the target stays in the sector.
          if (uint32_t(a >> 56) == (bb >> 24)) {
            ok[b] = true;
            col[b] = (a & qkb::kOffsetMask) + (bb & qkb::kRankMask);
          }
        }
      }
    }
    #pragma unroll
    for (int b = 0; b < kGB; ++b) {
      if (!ok[b]) continue;
      R vr, vi;
      T::ld(x, col[b], vr, vi);
      yr += cr[b] * vr;
      if (T::cplx) {
        yi += cr[b] * vi;
        if (CC) { yr -= ci[b] * vi; yi += ci[b] * vr; }
      }
    }
  }
}

template <int DT, bool CC, bool DOT>
__global__ void __launch_bounds__(kTile)
k_hx(DevPlan p, const void* __restrict__ x, void* __restrict__ y, double* partials,
     unsigned* ticket, double* dot_out) {
  using T = VT<DT>;
  using R = typename T::R;
  qk_term_t* st;
  qk_group_t* sg;
  stage_plan(p, st, sg);
  double dr = 0.0, di = 0.0;
  for (uint32_t ti = blockIdx.x; ti < p.ntiles; ti += gridDim.x) {
    const qk_tile_t tile = p.tiles[ti];
    if (tile.row0 < p.row_lo || tile.row0 >= p.row_hi) continue;
    if (threadIdx.x < tile.count) {
      const uint64_t row = tile.row0 + threadIdx.x;
      const uint64_t s = (uint64_t(tile.h) << p.L) | __ldg(p.llist + tile.lstart + threadIdx.x);
      R yr, yi, xr, xi;
      row_apply<DT, CC>(p, st, sg, row, s, x, yr, yi, xr, xi);
      T::st(y, row, yr, yi);
      if (DOT) {  // <x, Hx> partial: conj(x) * y
        dr += double(xr) * double(yr) + double(xi) * double(yi);
        di += double(xr) * double(yi) - double(xi) * double(yr);
      }
    }
  }
  if (DOT) {
    __shared__ double sbuf[2 * (kTile / 32)];
    block_sum2(dr, di, sbuf);
    if (threadIdx.x == 0) { partials[2 * blockIdx.x] = dr; partials[2 * blockIdx.x + 1] = di; }
    grid_finish(partials, ticket, 1, dot_out);
  }
}

// Block H.X on R vectors stored row-interleaved: element (i, r) at i*R + r.
// LPR consecutive lanes share one row and each covers VPL = R / LPR
// consecutive vectors with one vector load per gather, so the state, the
// term table walk and the target ranking of a row are done once and reused
// for all R vectors.  With dots != nullptr the column dots <X_r, Y_r> are
// reduced deterministically (fixed thread order, then block order).
template <class E, int VPL>
struct alignas(sizeof(E) * VPL) RowPack { E v[VPL]; };

template <int DT> __device__ __forceinline__ void unpack1(const typename VT<DT>::E& e, typename VT<DT>::R& re,
                                                        typename VT<DT>::R& im);
template <> __device__ __forceinline__ void unpack1<QK_C128>(const double2& e, double& re, double& im) { re = e.x; im = e.y; }
template <> __device__ __forceinline__ void unpack1<QK_C64>(const float2& e, float& re, float& im) { re = e.x; im = e.y; }
template <> __device__ __forceinline__ void unpack1<QK_F64>(const double& e, double& re, double& im) { re = e; im = 0; }
template <> __device__ __forceinline__ void unpack1<QK_F32>(const float& e, float& re, float& im) { re = e; im = 0; }
__device__ __forceinline__ double2 pack1(double re, double im, double2*) { return make_double2(re, im); }
__device__ __forceinline__ float2 pack1(float re, float im, float2*) { return make_float2(re, im); }
__device__ __forceinline__ double pack1(double re, double, double*) { return re; }
__device__ __forceinline__ float pack1(float re, float, float*) { return re; }

template <int DT, bool CC, int LPR, int VPL>
__global__ void __launch_bounds__(kTile)
k_hx_block(DevPlan p, const void* __restrict__ X, void* __restrict__ Y, const void* __restrict__ diag,
           double* partials, unsigned* ticket, double* dots) {
  using T = VT<DT>;
  using R = typename T::R;
  using E = typename T::E;
  using Pack = RowPack<E, VPL>;
  constexpr int RV = LPR * VPL, RPW = 32 / LPR;
  qk_term_t* st;
  qk_group_t* sg;
  stage_plan(p, st, sg);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sub = lane / LPR, l = lane % LPR;
  const E* __restrict__ Xe = reinterpret_cast<const E*>(X);
  E* __restrict__ Ye = reinterpret_cast<E*>(Y);
  double dr[VPL], di[VPL];
  #pragma unroll
  for (int v = 0; v < VPL; ++v) { dr[v] = 0.0; di[v] = 0.0; }
  for (uint32_t ti = blockIdx.x; ti < p.ntiles; ti += gridDim.x) {
    const qk_tile_t tile = p.tiles[ti];
    for (uint32_t rr = warp * RPW + sub; rr < tile.count; rr += (kTile / 32) * RPW) {
      const uint64_t row = tile.row0 + rr;
      const uint64_t s = (uint64_t(tile.h) << p.L) | __ldg(p.llist + tile.lstart + rr);
      const Pack x0 = *reinterpret_cast<const Pack*>(Xe + row * RV + l * VPL);
      R x0r[VPL], x0i[VPL], ar[VPL], ai[VPL];
      #pragma unroll
      for (int v = 0; v < VPL; ++v) { unpack1<DT>(x0.v[v], x0r[v], x0i[v]); ar[v] = R(0); ai[v] = R(0); }
      uint32_t g0 = 0;
      if (p.has_diag) {
        // the diagonal from the precomputed vector when given, else from the
        // diagonal term group
        R cr, ci;
        bool any = true;
        if (diag) T::ld(diag, row, cr, ci);
        else any = group_coef<CC, R>(st, sg[0].first, sg[0].count, s, cr, ci);
        if (any) {
          #pragma unroll
          for (int v = 0; v < VPL; ++v) {
            ar[v] += cr * x0r[v];
            if (T::cplx) {
              ai[v] += cr * x0i[v];
              if (CC) { ar[v] -= ci * x0i[v]; ai[v] += ci * x0r[v]; }
            }
          }
        }
        g0 = 1;
      }
      for (uint32_t g = g0; g < p.ngroups; ++g) {
        const qk_group_t grp = sg[g];
        R cr, ci;
        if (!group_coef<CC, R>(st, grp.first, grp.count, s, cr, ci)) continue;
        const uint64_t t = s ^ grp.flip;
        const uint64_t a = __ldg(p.A + (t >> p.L));
        const uint32_t b = __ldg(p.B + (t & p.lmask));
        if (uint32_t(a >> 56) != (b >> 24)) continue;  // target outside the sector
        const uint64_t col = (a & qkb::kOffsetMask) + (b & qkb::kRankMask);
        const Pack xv = *reinterpret_cast<const Pack*>(Xe + col * RV + l * VPL);
        #pragma unroll
        for (int v = 0; v < VPL; ++v) {
          R xr, xi;
          unpack1<DT>(xv.v[v], xr, xi);
          ar[v] += cr * xr;
          if (T::cplx) {
            ai[v] += cr * xi;
            if (CC) { ar[v] -= ci * xi; ai[v] += ci * xr; }
          }
        }
      }
      Pack yv;
      #pragma unroll
      for (int v = 0; v < VPL; ++v) {
        yv.v[v] = pack1(ar[v], ai[v], static_cast<E*>(nullptr));
        dr[v] += double(x0r[v]) * double(ar[v]) + double(x0i[v]) * double(ai[v]);
        di[v] += double(x0r[v]) * double(ai[v]) - double(x0i[v]) * double(ar[v]);
      }
      *reinterpret_cast<Pack*>(Ye + row * RV + l * VPL) = yv;
    }
  }
  // column c = l * VPL + v: sum over the threads with the same l, fixed order
  __shared__ double red[kTile * 2];
  for (int v = 0; v < VPL; ++v) {
    __syncthreads();
    red[2 * threadIdx.x] = dr[v];
    red[2 * threadIdx.x + 1] = di[v];
    __syncthreads();
    if (threadIdx.x < LPR) {
      double sr = 0.0, si = 0.0;
      for (int t = threadIdx.x; t < kTile; t += LPR) { sr += red[2 * t]; si += red[2 * t + 1]; }
      const int c = threadIdx.x * VPL + v;
      partials[(size_t(c) * gridDim.x + blockIdx.x) * 2] = sr;
      partials[(size_t(c) * gridDim.x + blockIdx.x) * 2 + 1] = si;
    }
  }
  grid_finish(partials, ticket, RV, dots);
}

template <int DT, bool CC>
__global__ void __launch_bounds__(kTile) k_diag(DevPlan p, void* __restrict__ d) {
  using T = VT<DT>;
  using R = typename T::R;
  qk_term_t* st;
  qk_group_t* sg;
  stage_plan(p, st, sg);
  for (uint32_t ti = blockIdx.x; ti < p.ntiles; ti += gridDim.x) {
    const qk_tile_t tile = p.tiles[ti];
    if (threadIdx.x < tile.count) {
      const uint64_t row = tile.row0 + threadIdx.x;
      const uint64_t s = (uint64_t(tile.h) << p.L) | __ldg(p.llist + tile.lstart + threadIdx.x);
      R cr = R(0), ci = R(0);
      if (p.has_diag) group_coef<CC, R>(st, sg[0].first, sg[0].count, s, cr, ci);
      T::st(d, row, cr, ci);
    }
  }
}

template <class K>
int set_smem(K kernel, size_t smem) {
  if (smem > 48 * 1024) {
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess) {
      (void)cudaGetLastError();
      return QKD_EINVAL;
    }
  }
  return QKD_OK;
}

template <class K>
unsigned hx_grid(const qk_plan* p, K kernel) {
  return std::max(1u, resident_grid(kernel, kTile, p->smem, std::max(1u, p->ntiles)));
}

template <int DT, bool CC>
int launch_apply(const qk_plan* p, const void* x, void* y, cudaStream_t s, qk_workspace* w,
                 double* dot_out, uint64_t row_lo = 0, uint64_t row_hi = ~0ull) {
  const DevPlan d = dev(p, row_lo, row_hi);
  if (dot_out) {
    auto k = k_hx<DT, CC, true>;
    if (set_smem(k, p->smem)) return QKD_EINVAL;
    const unsigned g = std::min<unsigned>(hx_grid(p, k), kMaxG);
    k<<<g, kTile, p->smem, s>>>(d, x, y, w->partials, w->ticket, dot_out);
  } else {
    auto k = k_hx<DT, CC, false>;
    if (set_smem(k, p->smem)) return QKD_EINVAL;
    k<<<hx_grid(p, k), kTile, p->smem, s>>>(d, x, y, nullptr, nullptr, nullptr);
  }
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

template <int DT, bool CC, int LPR, int VPL>
int launch_block(const qk_plan* p, qk_workspace* w, const void* X, void* Y, const void* diag, double* dots,
                 cudaStream_t s) {
  auto k = k_hx_block<DT, CC, LPR, VPL>;
  if (set_smem(k, p->smem)) return QKD_EINVAL;
  const unsigned g = std::min<unsigned>(hx_grid(p, k), kMaxG);
  k<<<g, kTile, p->smem, s>>>(dev(p), X, Y, diag, w->partials, w->ticket, dots ? dots : w->result);
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

template <int DT, bool CC>
int launch_block_shape(const qk_plan* p, qk_workspace* w, int R, int lpr, const void* X, void* Y, const void* diag,
                       double* dots, cudaStream_t s) {
#define QKD_BLK(RR, L, V) if (R == RR && lpr == L) return launch_block<DT, CC, L, V>(p, w, X, Y, diag, dots, s);
  QKD_BLK(32, 32, 1) QKD_BLK(32, 16, 2) QKD_BLK(32, 8, 4)
  QKD_BLK(64, 32, 2) QKD_BLK(64, 16, 4) QKD_BLK(64, 8, 8)
  QKD_BLK(128, 32, 4) QKD_BLK(128, 16, 8)
#undef QKD_BLK
  return QKD_EINVAL;
}

int r_index(int R) { return R == 32 ? 0 : R == 64 ? 1 : R == 128 ? 2 : -1; }

}  // namespace
}  // namespace qkd

using namespace qkd;

extern "C" {

int qkd_plan_create(const qk_plan_desc* d, int device, qk_plan** out) {
  if (!d || !out || d->nbits <= 0 || d->nbits > 64 || d->L < 0 || d->L > d->nbits) return QKD_EINVAL;
  if (d->nterms > 0 && (!d->terms || !d->groups)) return QKD_EINVAL;
  // Tiles: runs of <= 256 rows inside each non-empty block.
  std::vector<qk_tile_t> tiles;
  for (uint64_t h = 0; h < d->nA; ++h) {
    const uint32_t need = uint32_t(d->A[h] >> 56);
    if (need == qkb::kEmptyBlockKey) continue;
    const uint32_t start = d->key_off[need], size = d->key_off[need + 1] - start;
    const uint64_t off = d->A[h] & qkb::kOffsetMask;
    for (uint32_t r = 0; r < size; r += kTile)
      tiles.push_back(qk_tile_t{off + r, uint32_t(h), start + r, std::min<uint32_t>(kTile, size - r), 0});
  }
  if (tiles.size() > 0xFFFFFFFFull) return QKD_EINVAL;
  auto* p = new qk_plan{};
  p->device = device;
  p->nbits = d->nbits; p->L = d->L; p->dim = d->dim;
  p->lmask = (d->L >= 64) ? ~0ULL : ((1ULL << d->L) - 1);
  p->nterms = d->nterms; p->ngroups = d->ngroups; p->ntiles = uint32_t(tiles.size());
  p->has_diag = d->has_diag; p->all_real = d->all_real;
  p->smem = size_t(d->nterms) * sizeof(qk_term_t) + size_t(d->ngroups) * sizeof(qk_group_t);
  if (p->smem > 200 * 1024) { delete p; return QKD_EINVAL; }
  auto up = [&](void** dst, const void* src, size_t bytes) -> bool {
    if (bytes == 0) { *dst = nullptr; return true; }
    if (cudaMalloc(dst, bytes) != cudaSuccess) return false;
    p->bytes += bytes;
    return cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice) == cudaSuccess;
  };
  bool ok = up((void**)&p->A, d->A, d->nA * 8) && up((void**)&p->B, d->B, d->nB * 4) &&
            up((void**)&p->llist, d->llist, d->nllist * 4) &&
            up((void**)&p->terms, d->terms, size_t(d->nterms) * sizeof(qk_term_t)) &&
            up((void**)&p->groups, d->groups, size_t(d->ngroups) * sizeof(qk_group_t)) &&
            up((void**)&p->tiles, tiles.data(), tiles.size() * sizeof(qk_tile_t));
  if (!ok) {
    (void)cudaGetLastError();
    qkd_plan_destroy(p);
    return QKD_ENOMEM;
  }
  p->spin = qkd::spin_plan_create(d, &p->bytes);
  if (!p->spin) p->spin = qkd::gen_plan_create(d, &p->bytes);
  // Operators on the generic kernel with a real diagonal keep it as a
  // vector (read once per row instead of walking the diagonal terms).
  bool diag_real = d->has_diag != 0;
  if (diag_real)
    for (uint32_t q = d->groups[0].first; q < d->groups[0].first + d->groups[0].count; ++q)
      if (d->terms[q].wim != 0.0) diag_real = false;
  const bool gen = p->spin && qkd::spin_plan_is_gen(p->spin);
  if ((!p->spin || gen) && diag_real && d->dim > 0) {
    if (cudaMalloc(&p->diag_re, d->dim * 8) == cudaSuccess) {
      p->bytes += d->dim * 8;
      qkd::SpinHandle* keep = p->spin;
      p->spin = nullptr;  // the diagonal kernel walks the terms; the plan is not complete yet
      const int rc = qkd_diagonal(p, QK_F64, p->diag_re, nullptr);
      p->spin = keep;
      if (rc != QKD_OK || cudaStreamSynchronize(nullptr) != cudaSuccess) {
        (void)cudaGetLastError();
        cudaFree(p->diag_re);
        p->diag_re = nullptr;
      }
    } else {
      (void)cudaGetLastError();
      p->diag_re = nullptr;
    }
  }
  if (gen && (!p->diag_re || qkd::spin_plan_set_diag(p->spin, p->diag_re) != QKD_OK)) {
    // without its diagonal vector the two-part kernel cannot run: generic kernel
    qkd::spin_plan_destroy(p->spin);
    p->spin = nullptr;
  }
  if (d->pair_sites && p->diag_re) p->pair = qkd::pair_plan_create(d, p->A, p->B, p->diag_re, &p->bytes);
  *out = p;
  return QKD_OK;
}

int qkd_set_kernel_policy(int policy) {
  if (policy < 0 || policy > 3) return QKD_EINVAL;
  g_kernel_policy = policy == 1 ? 1 : 0;
  qkd::spin_set_die_queues(policy != 2);
  g_pair_path = policy != 3;
  return QKD_OK;
}

int qkd_plan_kernel(const qk_plan* p) {
  if (!p || g_kernel_policy != 0) return 0;
  if (p->pair && g_pair_path) return 3;
  if (!p->spin) return 0;
  return qkd::spin_plan_is_gen(p->spin) ? 2 : 1;
}

int qkd_plan_destroy(qk_plan* p) {
  if (!p) return QKD_OK;
  qkd::pair_plan_destroy(p->pair);
  qkd::spin_plan_destroy(p->spin);
  cudaFree(p->diag_re);
  cudaFree(p->A); cudaFree(p->B); cudaFree(p->llist);
  cudaFree(p->terms); cudaFree(p->groups); cudaFree(p->tiles);
  delete p;
  return QKD_OK;
}

uint64_t qkd_plan_dim(const qk_plan* p) { return p ? p->dim : 0; }
int qkd_plan_all_real(const qk_plan* p) { return p ? p->all_real : 0; }
size_t qkd_plan_device_bytes(const qk_plan* p) { return p ? p->bytes : 0; }

int qkd_apply(const qk_plan* p, qk_dtype t, const void* x, void* y, cudaStream_t s) {
  if (!p || !x || !y || x == y) return QKD_EINVAL;
  if (p->dim == 0 || p->ntiles == 0) return QKD_OK;
  if (!qk_dtype_complex(t) && !p->all_real) return QKD_EINVAL;
  if (p->pair && g_kernel_policy == 0 && g_pair_path) {
    const int rc = qkd::pair_apply(p->pair, t, x, y, s, nullptr, nullptr);
    if (rc != QKD_EINVAL) return rc;
  }
  if (p->spin && g_kernel_policy == 0) return qkd::spin_apply(p->spin, t, x, y, s, nullptr, nullptr);
  if (p->all_real) { QKD_DISPATCH(t, return launch_apply<DT, false>(p, x, y, s, nullptr, nullptr)); }
  QKD_DISPATCH(t, return launch_apply<DT, true>(p, x, y, s, nullptr, nullptr));
  return QKD_OK;
}

// Rows [row_lo, row_hi) of y = H x (x complete; the other rows of y are not
// written).  The bounds must be sector-block boundaries (qkd_plan_shard).
int qkd_apply_range(const qk_plan* p, qk_dtype t, const void* x, void* y, uint64_t row_lo, uint64_t row_hi,
                    cudaStream_t s) {
  if (!p || !x || !y || x == y || row_lo > row_hi || row_hi > p->dim) return QKD_EINVAL;
  if (p->dim == 0 || p->ntiles == 0 || row_lo == row_hi) return QKD_OK;
  if (!qk_dtype_complex(t) && !p->all_real) return QKD_EINVAL;
  if (p->spin && g_kernel_policy == 0) {
    const int rc = qkd::spin_apply_range(p->spin, t, x, y, s, row_lo, row_hi);
    if (rc != QKD_EINVAL) return rc;
  }
  if (p->all_real) { QKD_DISPATCH(t, return launch_apply<DT, false>(p, x, y, s, nullptr, nullptr, row_lo, row_hi)); }
  QKD_DISPATCH(t, return launch_apply<DT, true>(p, x, y, s, nullptr, nullptr, row_lo, row_hi));
  return QKD_OK;
}

// y = H x and out = <x, y> in one pass.
int qkd_apply_dot(const qk_plan* p, qk_workspace* w, qk_dtype t, const void* x, void* y,
                  double* dot_out, cudaStream_t s) {
  if (!p || !w || !x || !y || x == y || !dot_out) return QKD_EINVAL;
  if (p->dim == 0 || p->ntiles == 0) return QKD_OK;
  if (!qk_dtype_complex(t) && !p->all_real) return QKD_EINVAL;
  if (p->pair && g_kernel_policy == 0 && g_pair_path) {
    const int rc = qkd::pair_apply(p->pair, t, x, y, s, w, dot_out);
    if (rc != QKD_EINVAL) return rc;
  }
  if (p->spin && g_kernel_policy == 0) return qkd::spin_apply(p->spin, t, x, y, s, w, dot_out);
  if (p->all_real) { QKD_DISPATCH(t, return launch_apply<DT, false>(p, x, y, s, w, dot_out)); }
  QKD_DISPATCH(t, return launch_apply<DT, true>(p, x, y, s, w, dot_out));
  return QKD_OK;
}

int qkd_apply_block(const qk_plan* p, qk_dtype t, int nvec, const void* X, size_t ldx, void* Y,
                    size_t ldy, cudaStream_t s) {
  if (!p || nvec < 0 || !X || !Y) return QKD_EINVAL;
  const size_t es = qk_dtype_size(t);
  for (int v = 0; v < nvec; ++v) {
    const int rc = qkd_apply(p, t, static_cast<const char*>(X) + v * ldx * es, static_cast<char*>(Y) + v * ldy * es, s);
    if (rc) return rc;
  }
  return QKD_OK;
}

static int apply_rows_shape(const qk_plan* p, qk_workspace* w, qk_dtype t, int R, int lpr, int tilec, const void* X,
                            void* Y, const void* diag, const double* g, double* dots, cudaStream_t s) {
  if (!p || !w || !X || !Y || X == Y || r_index(R) < 0) return QKD_EINVAL;
  if (p->dim == 0 || p->ntiles == 0) return QKD_OK;
  if (!qk_dtype_complex(t) && !p->all_real) return QKD_EINVAL;
  if (g) {
    if (!p->spin || g_kernel_policy != 0) return QKD_EINVAL;  // row-kernel tables only
    return qkd::spin_apply_block(p->spin, t, R, lpr, X, Y, dots, s, w, g, tilec);
  }
  if (p->spin && g_kernel_policy == 0) {  // the row-kernel tables where the operator has them
    const int rc = qkd::spin_apply_block(p->spin, t, R, lpr, X, Y, dots, s, w, nullptr, tilec);
    if (rc != QKD_EINVAL) return rc;
  }
  if (p->all_real) { QKD_DISPATCH(t, return launch_block_shape<DT, false>(p, w, R, lpr, X, Y, diag, dots, s)); }
  if (t == QK_C128) return launch_block_shape<QK_C128, true>(p, w, R, lpr, X, Y, diag, dots, s);
  if (t == QK_C64) return launch_block_shape<QK_C64, true>(p, w, R, lpr, X, Y, diag, dots, s);
  return QKD_EINVAL;
}

int qkd_apply_rows(const qk_plan* p, qk_workspace* w, qk_dtype t, int R, int lanes_per_row, const void* X,
                   void* Y, const void* diag, double* dots, cudaStream_t s) {
  if (!p || r_index(R) < 0 || t < QK_C128 || t > QK_F32) return QKD_EINVAL;
  const int lpr = lanes_per_row ? lanes_per_row : (p->rows_lpr[t][r_index(R)] ? p->rows_lpr[t][r_index(R)] : 32);
  const int tilec = lanes_per_row ? 0 : p->rows_tile[t][r_index(R)];
  return apply_rows_shape(p, w, t, R, lpr, tilec, X, Y, diag, nullptr, dots, s);
}

int qkd_apply_rows_acc(const qk_plan* p, qk_workspace* w, qk_dtype t, int R, int lanes_per_row, const void* X,
                       void* Y, const double* g, double* dots, cudaStream_t s) {
  if (!p || !g || r_index(R) < 0 || t < QK_C128 || t > QK_F32) return QKD_EINVAL;
  const int lpr = lanes_per_row ? lanes_per_row : (p->rows_lpr[t][r_index(R)] ? p->rows_lpr[t][r_index(R)] : 32);
  const int tilec = lanes_per_row ? 0 : p->rows_tile[t][r_index(R)];
  return apply_rows_shape(p, w, t, R, lpr, tilec, X, Y, nullptr, g, dots, s);
}

int qkd_rows_shape(const qk_plan* p, qk_dtype t, int R) {
  if (!p || r_index(R) < 0 || t < QK_C128 || t > QK_F32) return 0;
  return p->rows_lpr[t][r_index(R)];
}

int qkd_rows_timings(const qk_plan* p, qk_dtype t, int R, float* ms9) {
  if (!p || !ms9 || r_index(R) < 0 || t < QK_C128 || t > QK_F32) return QKD_EINVAL;
  for (int i = 0; i < 9; ++i) ms9[i] = p->rows_ms[t][r_index(R)][i];
  return QKD_OK;
}

// The block apply's shape: lanes per row (so vectors per lane R / lanes)
// times tile rows (the rows a CTA takes per fetch: 256, 128 or 512; row
// kernels only), each timed launch by launch in two interleaved rounds of
// three launches after a warm-up; the fastest single launch decides (robust
// to clock drift and to a slow first round) and is kept in the plan per
// dtype and R.  g != NULL tunes the accumulating form Y += diag(g) H X.
static int tune_rows(qk_plan* p, qk_workspace* w, qk_dtype t, int R, const void* X, void* Y, const void* diag,
                     const double* g, cudaStream_t s, int* chosen) {
  if (!p || !w || r_index(R) < 0 || t < QK_C128 || t > QK_F32) return QKD_EINVAL;
  const int lprs[3] = {32, 16, 8};
  const int ntile = (p->spin && g_kernel_policy == 0) ? 3 : 1;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return QKD_ECUDA;
  float fastest[3][3];
  for (auto& r : fastest) for (float& v : r) v = 1e30f;
  for (int round = 0; round < 2; ++round)
    for (int q = 0; q < 3; ++q)
      for (int tc = 0; tc < ntile; ++tc) {
        const int lpr = lprs[q];
        if (R / lpr > 8) continue;
        auto launch = [&]() { return apply_rows_shape(p, w, t, R, lpr, tc, X, Y, diag, g, nullptr, s); };
        if (round == 0 && launch() != QKD_OK) continue;  // warm-up
        for (int i = 0; i < 3; ++i) {
          cudaEventRecord(e0, s);
          if (launch() != QKD_OK) break;
          cudaEventRecord(e1, s);
          float ms = 0.f;
          if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) break;
          fastest[q][tc] = std::min(fastest[q][tc], ms);
        }
      }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  (void)cudaGetLastError();
  float best = 1e30f;
  int pick = 0, pick_tc = 0;
  for (int q = 0; q < 3; ++q)
    for (int tc = 0; tc < ntile; ++tc)
      if (fastest[q][tc] < best) { best = fastest[q][tc]; pick = lprs[q]; pick_tc = tc; }
  if (!pick) return QKD_ECUDA;
  for (int q = 0; q < 3; ++q)
    for (int tc = 0; tc < 3; ++tc)
      p->rows_ms[t][r_index(R)][q * 3 + tc] = (tc < ntile && fastest[q][tc] < 1e29f) ? fastest[q][tc] : 0.f;
  p->rows_lpr[t][r_index(R)] = pick;
  p->rows_tile[t][r_index(R)] = pick_tc;
  if (chosen) *chosen = pick;
  return QKD_OK;
}

int qkd_tune_rows(qk_plan* p, qk_workspace* w, qk_dtype t, int R, const void* X, void* Y, const void* diag,
                  cudaStream_t s, int* chosen) {
  return tune_rows(p, w, t, R, X, Y, diag, nullptr, s, chosen);
}

int qkd_tune_rows_acc(qk_plan* p, qk_workspace* w, qk_dtype t, int R, const void* X, void* Y, const double* g,
                      cudaStream_t s, int* chosen) {
  if (!g) return QKD_EINVAL;
  return tune_rows(p, w, t, R, X, Y, nullptr, g, s, chosen);
}

int qkd_diagonal(const qk_plan* p, qk_dtype t, void* diag, cudaStream_t s) {
  if (!p || !diag) return QKD_EINVAL;
  if (p->dim == 0 || p->ntiles == 0) return QKD_OK;
  if (!qk_dtype_complex(t) && !p->all_real) return QKD_EINVAL;
  const DevPlan d = dev(p);
  if (p->all_real) {
    QKD_DISPATCH(t, { auto k = k_diag<DT, false>; if (set_smem(k, p->smem)) return QKD_EINVAL; k<<<hx_grid(p, k), kTile, p->smem, s>>>(d, diag); });
  } else {
    QKD_DISPATCH(t, { auto k = k_diag<DT, true>; if (set_smem(k, p->smem)) return QKD_EINVAL; k<<<hx_grid(p, k), kTile, p->smem, s>>>(d, diag); });
  }
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

}  // extern "C"
