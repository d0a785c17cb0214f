// H.x specialised for two-site exchange operators in a single-charge sector
// (spin-1/2 fixed Sz, spinless fermions without strings): the Heisenberg,
// XXZ and J1-J2 families.
//
// Every off-diagonal group flips exactly two bits i < j and is conditioned on
// both (Sp_i Sm_j, Sm_i Sp_j ...), every diagonal term is a sign-only
// product (Sz Sz).  Relative to the sector split at bit L a bond is
//   low      (i, j < L):  target rank = A[h] + B[l ^ F]       one smem lookup
//   high     (i, j >= L): target rank = A[h ^ F'] + r         validity and base
//                         depend on h only, so they are computed once per tile
//                         and the warp's gathers are consecutive addresses
//   crossing (i < L <= j): A[h ^ F'] + B[l ^ F], two smem lookups.
// A (u32 offsets) and B (u16 in-class ranks) live in shared memory; the
// state of a row comes from the coalesced low-part list.  One thread per row,
// 512 rows per tile.
#include <algorithm>
#include <mutex>
#include <vector>

#include "reduce.cuh"
#include "../engine/sector.hpp"

namespace qkd {

constexpr int kSpinThreads = 512;
constexpr int kMaxBonds = 64;
constexpr int kMaxDiag = 128;

struct SpinBond {
  uint32_t lo_mask, hi_mask;  // flip split into the low / high part
  double c[4];                // coefficient for (bit_i, bit_j) = 00, 10, 01, 11
  uint8_t bi, bj;             // bit positions
  uint8_t kind;               // 0 low, 1 high, 2 crossing
  uint8_t valid_mask;         // which combos have a valid term
};

struct RowBlock {
  uint32_t base, size, lst, ebeg;  // block offset, rows, llist position, first entry in bent
  uint32_t nh, combo;              // high entries; sign pattern of the crossing Sz Sz terms
  double dh;                       // diagonal terms inside the high part
};

struct SpinPlan {
  int L, H;
  uint64_t dim;
  int nbonds, ndiag;
  // bond classes (host-side, for building the row tables)
  int nlow, nhigh, ncross, ndcross;
  uint32_t low_mask[kMaxBonds], high_mask[kMaxBonds], cross_lo[kMaxBonds], cross_hi[kMaxBonds];
  uint8_t low_i[kMaxBonds], high_i[kMaxBonds], cross_li[kMaxBonds];
  double low_c01[kMaxBonds], low_c10[kMaxBonds], high_c01[kMaxBonds], high_c10[kMaxBonds];
  double cross_c01[kMaxBonds], cross_c10[kMaxBonds];   // c01: low bit 0 / high bit 1
  uint32_t max_block;      // largest block size
  double coef[2 * kMaxBonds];
  int ncoef;
  uint32_t dcross_mask[kMaxDiag];
  double dcross_w[kMaxDiag];
  SpinBond bonds[kMaxBonds];
  uint32_t diag_smask[kMaxDiag];
  double diag_w[kMaxDiag];
  const uint32_t* A32;   // 2^H block offsets (global copy, staged to smem)
  const uint16_t* B16;   // 2^L in-class ranks (global copy, staged to smem)
  const uint16_t* lrow;  // llist as u16
  const qk_tile_t* tiles;
  uint32_t ntiles;
  size_t smem;
  // class and block tables of the row kernel
  const uint2* rrec;     // per llist position: first 4-entry group; groups per low class, 4 bits each
  const uint2* lgrp;     // 4 in-class ranks (u16) per group; padding entries name the zero slot
  const uint16_t* crk;   // [pos][cpad]: (low-side bit << 15) | partner in-class rank
  const double* dtab;    // [combo][pos]: low-part diagonal plus the crossing Sz Sz terms
  const RowBlock* brec;  // per sector block
  const uint2* bent;     // per block: high entries (base, coef) then crossing (base, coef | bit_h << 16)
  double lcls[4];        // coefficient of each low class
  int ncls, cpad, ncombo;
  uint32_t zero_slot, nllist;
  bool rows_ok;
  // two-part operators (any factorisable group, e.g. Hubbard and t-J hops)
  bool gen;
  uint32_t nblocks;       // block records (all 2^H, or only the non-empty ones)
  const uint32_t* crk32;  // [ncross][pos] (coalesced over rows): rank | lv0 << 24 | ls0 << 25 | lv1 << 26 | ls1 << 27
  const uint32_t* crm;    // [pos]: bit q set when a term of crossing group q has its low condition
  const double* diag_full;  // two-part operators: the diagonal per row, summed in term order
  const uint4* btiles;      // block apply: (block record, first row, rows) runs of <= 256 rows
  uint32_t nbtiles;
  const uint32_t* border;   // order in which the row kernel visits the block records (null: record order)
  // per-die work queues of the row kernel: the SMs of die 0 take the visiting
  // positions [0, qsplit), those of die 1 [qsplit, nblocks); a CTA whose
  // queue is empty takes from the other one
  const uint8_t* sm_die;    // die of each SM id (null: one die)
  uint32_t nsmid, qsplit;
};

namespace {

template <int DT, bool DOT>
__global__ void __launch_bounds__(kSpinThreads)
k_hx_spin(const SpinPlan* __restrict__ pp, const void* __restrict__ x, void* __restrict__ y, double* partials,
          unsigned* ticket, double* dot_out, uint64_t row_lo, uint64_t row_hi) {
  using T = VT<DT>;
  using R = typename T::R;
  extern __shared__ __align__(16) unsigned char sm[];
  const SpinPlan& p = *pp;
  const int nA = 1 << p.H, nB = 1 << p.L;
  const int nbonds = p.nbonds, ndiag = p.ndiag;
  const uint64_t dim = p.dim;
  const uint32_t ntiles = p.ntiles;
  uint32_t* sA = reinterpret_cast<uint32_t*>(sm);
  uint16_t* sB = reinterpret_cast<uint16_t*>(sm + size_t(nA) * 4);
  __shared__ SpinBond sbond[kMaxBonds];
  __shared__ uint32_t sdm[kMaxDiag];
  __shared__ R sdw[kMaxDiag];
  __shared__ uint64_t s_hbase[kMaxBonds];
  __shared__ R s_hcoef[kMaxBonds];
  __shared__ int s_hvalid[kMaxBonds];
  for (int i = threadIdx.x; i < nA; i += blockDim.x) sA[i] = p.A32[i];
  for (int i = threadIdx.x; i < nB; i += blockDim.x) sB[i] = p.B16[i];
  for (int i = threadIdx.x; i < nbonds; i += blockDim.x) sbond[i] = p.bonds[i];
  for (int i = threadIdx.x; i < ndiag; i += blockDim.x) { sdm[i] = p.diag_smask[i]; sdw[i] = R(p.diag_w[i]); }
  __syncthreads();
  const int L = p.L;
  double dr = 0.0, di = 0.0;
  for (uint32_t ti = blockIdx.x; ti < ntiles; ti += gridDim.x) {
    const qk_tile_t tile = p.tiles[ti];
    if (tile.row0 < row_lo || tile.row0 >= row_hi) continue;
    const uint32_t h = tile.h;
    if (threadIdx.x < uint32_t(nbonds)) {  // per-tile data of the high bonds
      const SpinBond b = sbond[threadIdx.x];
      if (b.kind == 1) {
        const uint32_t bi = (h >> (b.bi - L)) & 1u, bj = (h >> (b.bj - L)) & 1u;
        const int combo = int(bi | (bj << 1));
        s_hvalid[threadIdx.x] = (b.valid_mask >> combo) & 1;
        s_hcoef[threadIdx.x] = R(b.c[combo]);
        s_hbase[threadIdx.x] = sA[h ^ b.hi_mask];
      }
    }
    __syncthreads();
    if (threadIdx.x < tile.count) {
      const uint64_t row = tile.row0 + threadIdx.x;
      const uint64_t rank_in_block = row - sA[h];
      const uint32_t l = p.lrow[tile.lstart + threadIdx.x];
      const uint32_t s = (h << L) | l;
      R xr0, xi0;
      T::ld(x, row, xr0, xi0);
      R d = R(0);
      for (int q = 0; q < ndiag; ++q) d += (__popc(s & sdm[q]) & 1) ? -sdw[q] : sdw[q];
      R yr = d * xr0, yi = d * xi0;
      const uint64_t base = sA[h];
      for (int q = 0; q < nbonds; ++q) {
        const SpinBond& b = sbond[q];
        uint64_t col;
        R c;
        if (b.kind == 1) {
          if (!s_hvalid[q]) continue;
          col = s_hbase[q] + rank_in_block;
          c = s_hcoef[q];
        } else {
          const uint32_t bi = (s >> b.bi) & 1u, bj = (s >> b.bj) & 1u;
          const int combo = int(bi | (bj << 1));
          if (!((b.valid_mask >> combo) & 1)) continue;
          c = R(b.c[combo]);
          col = (b.kind == 0 ? base : uint64_t(sA[h ^ b.hi_mask])) + sB[l ^ b.lo_mask];
        }
        if (col >= dim) continue;  // cannot happen for conserving bonds; keeps every load in bounds
        R xr, xi;
        T::ld(x, col, xr, xi);
        yr += c * xr;
        if (T::cplx) yi += c * xi;
      }
      T::st(y, row, yr, yi);
      if (DOT) {
        dr += double(xr0) * double(yr) + double(xi0) * double(yi);
        di += double(xr0) * double(yi) - double(xi0) * double(yr);
      }
    }
    __syncthreads();
  }
  if (DOT) {
    __shared__ double sbuf[2 * (kSpinThreads / 32)];
    block_sum2(dr, di, sbuf);
    if (threadIdx.x == 0) { partials[2 * blockIdx.x] = dr; partials[2 * blockIdx.x + 1] = di; }
    grid_finish(partials, ticket, 1, dot_out);
  }
}

// Row kernel.  A CTA owns one sector block h at a time (grid-stride over
// blocks) and stages x_h in shared memory; each thread then walks the rows
// r = tid, tid + 256, ... of the block.  Everything a row needs that does
// not depend on h is precomputed per class position, and everything that
// depends on h only comes from one block record and its entry list, so the
// row body is loads and FMAs:
//   y[r] = (dh + dtab[combo][pos]) x_h[r]                  diagonal
//        + sum_c lc_c sum_j x_h[k_cj]    (u16 row lists)   low bonds
//        + sum_q [bit_l != bit_h] c_q x[cb_q + rk_q]       crossing bonds
//        + sum_e c_e x[hb_e + r]         (coalesced)       high bonds
// The low list of a row is grouped by coefficient class and padded to
// groups of four with the index of a zero slot behind the staged block, so
// a row reads 4 targets per 8-byte load.  The next block's record is loaded
// while the current block runs.
// Index arithmetic is 32-bit (dim < 2^32 is a precondition of the plan).
// All gathers stay in bounds by construction: list ranks are in-class ranks
// of the row's own class, partner blocks of a high bond have the block's
// size, and crossing ranks are in-class ranks of the partner's class; the
// plan builder checks the high-bond sizes.
constexpr int kRowThreads = 256;
constexpr uint32_t kRowStreamY = 1u;  // launch flag: store y with the streaming (evict-first) hint
constexpr int kRowHighC128 = 3;   // complex128: high bonds held in registers (4: 1% slower, 6: 2%)
constexpr int kRowMinCtaC128 = 2; // complex128: CTAs per SM the registers are sized for
constexpr int kRowThreadsC128 = 512;  // complex128: threads per CTA (one staged block shared by 16 warps)
constexpr int kPrefetchAhead = 2; // row chunks of high-bond partner rows prefetched into L2
constexpr int kRowCoef = 32, kRowEnt = 48, kRowCross = 16, kRowCls = 4;
// Rows per thread and pass (K) and CTAs per SM the registers are sized for,
// by vector type and table form.  The kernel is latency-bound, so resident
// warps count for more than the words they spill; measured on Heisenberg
// N=28 (exchange tables), t-J N=20 and Hubbard 4x4 (two-part tables)
// against K = 4 at 4 CTAs: float32 0.576 -> 0.441 ms (K = 1, 8 CTAs),
// float64 0.803 -> 0.580 ms (K = 2, 6 CTAs), complex64 0.620 -> 0.587 ms
// (K = 2, 6 CTAs); two-part float64 t-J 0.414 -> 0.347 ms and Hubbard
// 16.0 -> 13.0 ms (K = 1, 6 CTAs), float32 Hubbard 13.6 -> 8.8 ms (K = 1,
// 8 CTAs).  complex128: one row per thread, 512-thread CTAs, 2 per SM.
template <int DT, bool GEN> constexpr int kRowBatchG = DT == QK_C128 ? 1 : DT == QK_F32 ? 1 : GEN && DT == QK_F64 ? 1 : 2;
template <int DT, bool GEN> constexpr int kRowMinCta = DT == QK_C128 ? kRowMinCtaC128 : DT == QK_F32 ? 8 : 6;
// high bonds held in registers (two-part tables: 4, t-J N=20 float64
// 0.347 -> 0.336 ms and float32 0.275 -> 0.265 ms against 8; exchange
// tables: 8, where 4, 6 and 12 were 1-8% slower)
template <int DT, bool GEN> constexpr int kRowHighRegs = DT == QK_C128 ? kRowHighC128 : GEN ? 4 : 8;
template <int DT> constexpr bool kRowPipe = DT == QK_C128;  // rows pipelined one ahead (one row per thread)
template <int DT> constexpr int kRowNT = DT == QK_C128 ? kRowThreadsC128 : kRowThreads;  // threads per CTA
// two-part crossing groups whose loads are issued together (fewer where a
// thread holds several rows, to stay within its registers)
template <int DT, bool GEN> constexpr int kCrossBatch = kRowBatchG<DT, GEN> == 1 ? 4 : 2;

__device__ __forceinline__ void sld(const double2* s, uint32_t k, double& re, double& im) {
  const double2 v = s[k]; re = v.x; im = v.y;
}
__device__ __forceinline__ void sld(const float2* s, uint32_t k, float& re, float& im) {
  const float2 v = s[k]; re = v.x; im = v.y;
}
__device__ __forceinline__ void sld(const double* s, uint32_t k, double& re, double& im) { re = s[k]; im = 0; }
__device__ __forceinline__ void sld(const float* s, uint32_t k, float& re, float& im) { re = s[k]; im = 0; }
__device__ __forceinline__ void szero(double2& v) { v = make_double2(0.0, 0.0); }
__device__ __forceinline__ void szero(float2& v) { v = make_float2(0.f, 0.f); }
__device__ __forceinline__ void szero(double& v) { v = 0.0; }
__device__ __forceinline__ void szero(float& v) { v = 0.f; }

// L2 prefetch of elements [first, first + count) of a vector of `es`-byte
// elements, rounded inward to 16-byte boundaries (bulk prefetch operands
// must be 16-byte aligned and sized).
__device__ __forceinline__ void l2_prefetch(const void* base, uint32_t es, uint32_t first, uint32_t count) {
  const uintptr_t b = reinterpret_cast<uintptr_t>(base);
  const uintptr_t lo = (b + uintptr_t(first) * es + 15) & ~uintptr_t(15);
  const uintptr_t hi = (b + uintptr_t(first + count) * es) & ~uintptr_t(15);
  if (hi > lo)
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(lo), "r"(uint32_t(hi - lo)) : "memory");
}

// Coefficient of a two-part crossing group in a row: up to two terms, each
// valid when its low condition (row table word `ent`) and its high
// condition (block entry flags `bf`) hold, signed by the parities of both
// parts.  Terms are added in order (first, then second).
template <class R>
__device__ __forceinline__ R cross_coef(uint32_t ent, uint32_t bf, const R* s_coef) {
  R c = R(0);
  if ((ent >> 24) & (bf >> 16) & 1u) {
    const R w = s_coef[bf & 0xFFu];
    c += (((ent >> 25) ^ (bf >> 17)) & 1u) ? -w : w;
  }
  if ((ent >> 26) & (bf >> 18) & 1u) {
    const R w = s_coef[(bf >> 8) & 0xFFu];
    c += (((ent >> 27) ^ (bf >> 19)) & 1u) ? -w : w;
  }
  return c;
}

__device__ __forceinline__ RowBlock load_block(const RowBlock* p) {
  const uint4* q = reinterpret_cast<const uint4*>(p);
  const uint4 a = __ldg(q), b = __ldg(q + 1);
  RowBlock r;
  r.base = a.x; r.size = a.y; r.lst = a.z; r.ebeg = a.w;
  r.nh = b.x; r.combo = b.y;
  r.dh = __hiloint2double(int(b.w), int(b.z));
  return r;
}

// Next visiting position for this CTA from the per-die queues (wq[0], wq[1];
// wq[2] counts CTAs that are done, the last one resets all three for the
// next launch).  Returns nblocks when both queues are empty.
__device__ __forceinline__ uint32_t wq_fetch(const SpinPlan& p, uint32_t* wq, int die) {
  for (int k = 0; k < 2; ++k) {
    const int q = die ^ k;
    const uint32_t beg = q ? p.qsplit : 0u, n = q ? p.nblocks - p.qsplit : p.qsplit;
    const uint32_t i = atomicAdd(wq + q, 1u);
    if (i < n) return beg + i;
  }
  return p.nblocks;
}

__device__ __forceinline__ int sm_die_of(const SpinPlan& p) {
  uint32_t s;
  asm volatile("mov.u32 %0, %%smid;" : "=r"(s));
  return (p.sm_die && s < p.nsmid) ? int(__ldg(p.sm_die + s)) : 0;
}

__device__ __forceinline__ void wq_done(uint32_t* wq) {
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(wq + 2, 1u) == gridDim.x - 1) {
      atomicExch(wq, 0u);
      atomicExch(wq + 1, 0u);
      atomicExch(wq + 2, 0u);
    }
  }
}

template <int DT, bool DOT, bool GEN>
__global__ void __launch_bounds__(kRowNT<DT>, kRowMinCta<DT, GEN>)
k_hx_spin_rows(const SpinPlan* __restrict__ pp, const void* __restrict__ x, void* __restrict__ y,
               double* partials, unsigned* ticket, double* dot_out, uint32_t* wq, uint32_t row_lo,
               uint32_t row_hi, uint32_t flags) {
  using T = VT<DT>;
  using R = typename T::R;
  using E = typename T::E;
  extern __shared__ __align__(16) unsigned char sm[];
  const SpinPlan& p = *pp;
  E* sx = reinterpret_cast<E*>(sm);
  const E* __restrict__ xg = reinterpret_cast<const E*>(x);
  __shared__ R s_coef[kRowCoef], s_lc[kRowCls], s_ec[kRowEnt];
  __shared__ uint32_t s_eb[kRowEnt], s_ebit[kRowCross];
  for (int i = threadIdx.x; i < kRowCoef; i += blockDim.x) s_coef[i] = R(p.coef[i]);
  if (threadIdx.x < kRowCls) s_lc[threadIdx.x] = R(p.lcls[threadIdx.x]);
  if (threadIdx.x == 0) szero(sx[p.zero_slot]);
  const uint32_t nA = p.nblocks;
  const uint32_t nll = p.nllist;
  const int ncross = p.ncross, ncls = p.ncls;
  const uint32_t cw = uint32_t(p.cpad) >> 1;  // crossing words (two u16 each) per row
  double dr = 0.0, di = 0.0;
  RowBlock nxt;
  const uint32_t* __restrict__ bord = p.border;
  // visiting positions: from the per-die queues (wq) or grid-stride
  __shared__ uint32_t s_pos[2];
  const int die = wq ? sm_die_of(p) : 0;
  uint32_t pos = blockIdx.x;
  if (wq) {
    if (threadIdx.x == 0) s_pos[0] = wq_fetch(p, wq, die);
    __syncthreads();
    pos = s_pos[0];
  }
  // DOT: one partial per block record, so the sum does not depend on which
  // CTA took which block
  __shared__ double s_dot[2 * (kRowNT<DT> / 32)];
  uint32_t nrec = pos < nA ? (bord ? __ldg(bord + pos) : pos) : 0u;
  if (pos < nA) nxt = load_block(p.brec + nrec);
  for (uint32_t it = 1; pos < nA; ++it) {
    const RowBlock cur = nxt;
    const uint32_t rec = nrec;
    // the next visiting position (queues: slot it & 1, last read before the
    // previous barrier); one barrier both publishes it and marks the
    // previous block finished with the staging and the entry tables (N=28:
    // c128 1.006 -> 0.989 ms, f32 0.442 -> 0.435 ms; f64 and c64 within
    // 1-2%, either way depending on code generation)
    if (wq && threadIdx.x == 0) s_pos[it & 1] = wq_fetch(p, wq, die);
    __syncthreads();
    const uint32_t pn = wq ? s_pos[it & 1] : pos + gridDim.x;
    if (pn < nA) {
      nrec = bord ? __ldg(bord + pn) : pn;
      nxt = load_block(p.brec + nrec);
    }
    pos = pn;
    if (cur.size == 0 || cur.base < row_lo || cur.base >= row_hi) {
      if (DOT && threadIdx.x == 0) { partials[2 * rec] = 0.0; partials[2 * rec + 1] = 0.0; }
      continue;
    }
    const uint32_t base = cur.base, size = cur.size, nh = cur.nh;
    for (uint32_t r = threadIdx.x; r < size; r += kRowNT<DT>) sx[r] = __ldg(xg + base + r);
    if (threadIdx.x < nh + uint32_t(ncross)) {
      const uint2 e = __ldg(p.bent + cur.ebeg + threadIdx.x);
      s_eb[threadIdx.x] = e.x;
      // crossing entries of two-part operators keep their raw flags
      s_ec[threadIdx.x] = (GEN && threadIdx.x >= nh) ? R(0) : s_coef[e.y & 0xFFFFu];
      if (threadIdx.x >= nh) s_ebit[threadIdx.x - nh] = GEN ? e.y : e.y >> 16;
      else  // high partner rows of the first row chunks into L2
        l2_prefetch(x, sizeof(E), e.x, min(size, uint32_t(kPrefetchAhead) * kRowBatchG<DT, GEN> * kRowNT<DT>));
    }
    __syncthreads();
    const R dh = R(cur.dh);
    const double* __restrict__ dcol = p.dtab + size_t(cur.combo) * nll;
    const uint32_t* __restrict__ ckw = reinterpret_cast<const uint32_t*>(p.crk);
    uint32_t chm = 0u;  // two-part: crossing groups with a term whose high condition holds in this block
    if constexpr (GEN)
      for (int q = 0; q < ncross; ++q) chm |= (((s_ebit[q] >> 16) | (s_ebit[q] >> 18)) & 1u) << q;
    // block-uniform entries in registers: the first NB high bonds, 2 crossing
    constexpr int NB = kRowHighRegs<DT, GEN>;
    const int nh8 = nh < uint32_t(NB) ? int(nh) : NB;
    uint32_t eb[NB];
    R ec[NB];
    #pragma unroll
    for (int e = 0; e < NB; ++e) {
      eb[e] = e < nh8 ? s_eb[e] : 0u;
      ec[e] = e < nh8 ? s_ec[e] : R(0);
    }
    uint32_t cb[2], cbit[2];
    R cc[2];
    const int ncr = GEN ? 0 : ncross;  // crossing bonds of the exchange form (two-part: below)
    #pragma unroll
    for (int u = 0; u < 2; ++u) {
      cb[u] = u < ncr ? s_eb[nh + u] : 0u;
      cbit[u] = u < ncr ? s_ebit[u] : 2u;  // 2: never equal to a low bit, never valid
      cc[u] = u < ncr ? s_ec[nh + u] : R(0);
    }
    constexpr int K = kRowBatchG<DT, GEN>;
    // complex128 exchange tables: the row tables (record, diagonal,
    // crossing ranks) of a thread's next row are loaded while the current row
    // runs, so the loads that depend on them (low groups, crossing partners)
    // start at the top of the row instead of one memory latency into it.
    // (Loading the next row's low groups and crossing values as well was
    // measured: no further gain.)
    constexpr bool PIPE = kRowPipe<DT> && !GEN;
    static_assert(!PIPE || K == 1, "the row pipeline holds one row per thread");
    uint2 nrec = make_uint2(0u, 0u);  // tables of the thread's next row (PIPE)
    double ndt = 0.0;
    uint32_t ntwo = 0u;
    if (PIPE && threadIdx.x < size) {
      const uint32_t pz = cur.lst + threadIdx.x;
      nrec = __ldg(p.rrec + pz);
      ndt = __ldg(dcol + pz);
      ntwo = ncr ? __ldg(ckw + pz * cw) : 0u;
    }
    for (uint32_t r0 = threadIdx.x; r0 < size; r0 += K * kRowNT<DT>) {
      // the high partner rows two chunks ahead go to L2 while this chunk runs
      {
        const uint32_t ahead = r0 - threadIdx.x + uint32_t(kPrefetchAhead) * K * kRowNT<DT>;
        if (threadIdx.x < nh && ahead < size)
          l2_prefetch(x, sizeof(E), s_eb[threadIdx.x] + ahead, min(size - ahead, uint32_t(K * kRowNT<DT>)));
      }
      // K rows r0 + k * 256 per thread.  Loads that do not depend on each
      // other are issued together: row records, diagonals, crossing pairs,
      // then all high-bond values; the shared-memory low groups come last.
      uint32_t rk[K], pos[K];
      bool ok[K];
      uint2 rec[K];
      double dt[K];
      uint32_t two[K];
      #pragma unroll
      for (int k = 0; k < K; ++k) {
        rk[k] = r0 + k * kRowNT<DT>;
        ok[k] = rk[k] < size;
        pos[k] = cur.lst + (ok[k] ? rk[k] : 0u);
        if constexpr (PIPE) {
          rec[k] = nrec; dt[k] = ndt; two[k] = ntwo;
        } else {
          rec[k] = __ldg(p.rrec + pos[k]);
          dt[k] = __ldg(dcol + pos[k]);
          two[k] = ncr ? __ldg(ckw + pos[k] * cw) : 0u;
        }
      }
      if constexpr (PIPE) {
        const uint32_t rn = r0 + kRowNT<DT>;
        if (rn < size) {
          const uint32_t pz = cur.lst + rn;
          nrec = __ldg(p.rrec + pz);
          ndt = __ldg(dcol + pz);
          ntwo = ncr ? __ldg(ckw + pz * cw) : 0u;
        }
      }
      R ar[K], ai[K];
      #pragma unroll
      for (int k = 0; k < K; ++k) { ar[k] = R(0); ai[k] = R(0); }
      #pragma unroll
      for (int e = 0; e < NB; ++e) {
        #pragma unroll
        for (int k = 0; k < K; ++k) {
          if (e < nh8 && ok[k]) {
            R vr, vi;
            T::ld(x, eb[e] + rk[k], vr, vi);
            ar[k] += ec[e] * vr;
            if (T::cplx) ai[k] += ec[e] * vi;
          }
        }
      }
      #pragma unroll
      for (int k = 0; k < K; ++k) {
        #pragma unroll
        for (int u = 0; u < 2; ++u) {
          const uint32_t ent = u ? (two[k] >> 16) : (two[k] & 0xFFFFu);
          if (ok[k] && (ent >> 15) != cbit[u]) {
            R vr, vi;
            T::ld(x, cb[u] + (ent & 0x7FFFu), vr, vi);
            ar[k] += cc[u] * vr;
            if (T::cplx) ai[k] += cc[u] * vi;
          }
        }
      }
      #pragma unroll
      for (int k = 0; k < K; ++k) {
        if (!ok[k]) continue;
        const uint32_t r = rk[k];
        if constexpr (K == 1) {
          // one row per thread: the remaining high bonds four loads at a time
          for (uint32_t e0 = NB; e0 < nh; e0 += 4) {
            R vr[4], vi[4];
            #pragma unroll
            for (int u = 0; u < 4; ++u) {
              vr[u] = R(0);
              vi[u] = R(0);
              if (e0 + u < nh) T::ld(x, s_eb[e0 + u] + r, vr[u], vi[u]);
            }
            #pragma unroll
            for (int u = 0; u < 4; ++u)
              if (e0 + u < nh) {
                ar[k] += s_ec[e0 + u] * vr[u];
                if (T::cplx) ai[k] += s_ec[e0 + u] * vi[u];
              }
          }
        } else {
          for (uint32_t e = NB; e < nh; ++e) {
            R vr, vi;
            T::ld(x, s_eb[e] + r, vr, vi);
            ar[k] += s_ec[e] * vr;
            if (T::cplx) ai[k] += s_ec[e] * vi;
          }
        }
        if constexpr (GEN) {
          // two-part crossing groups: up to two terms, each valid when its
          // low condition (row table) and high condition (block entry) hold,
          // with the sign of both parts' Jordan-Wigner / Sz parities
          // only the groups with a term valid in both parts: the row's low
          // mask and the block's high mask.  Four groups at a time: their
          // table words, then their partner values, are in flight together
          // (sums still in ascending group order).
          for (uint32_t m = __ldg(p.crm + pos[k]) & chm; m;) {
            constexpr int CBAT = kCrossBatch<DT, GEN>;
            int qq[CBAT];
            uint32_t ent[CBAT];
            #pragma unroll
            for (int u = 0; u < CBAT; ++u) {
              qq[u] = m ? __ffs(m) - 1 : -1;
              m &= m - 1u;
              ent[u] = qq[u] >= 0 ? __ldg(p.crk32 + size_t(qq[u]) * nll + pos[k]) : 0u;
            }
            R cq[CBAT], vr[CBAT], vi[CBAT];
            #pragma unroll
            for (int u = 0; u < CBAT; ++u) {
              cq[u] = qq[u] >= 0 ? cross_coef<R>(ent[u], s_ebit[qq[u]], s_coef) : R(0);
              vr[u] = R(0);
              vi[u] = R(0);
              if (cq[u] != R(0)) T::ld(x, s_eb[nh + qq[u]] + (ent[u] & 0xFFFFFFu), vr[u], vi[u]);
            }
            #pragma unroll
            for (int u = 0; u < CBAT; ++u)
              if (cq[u] != R(0)) {
                ar[k] += cq[u] * vr[u];
                if (T::cplx) ai[k] += cq[u] * vi[u];
              }
          }
        }
        for (int q = 2; q < ncr; q += 2) {
          const uint32_t tw = __ldg(ckw + pos[k] * cw + (q >> 1));
          #pragma unroll
          for (int u = 0; u < 2; ++u) {
            const uint32_t ent = u ? (tw >> 16) : (tw & 0xFFFFu);
            if (q + u < ncross && (ent >> 15) != s_ebit[q + u]) {
              R vr, vi;
              T::ld(x, s_eb[nh + q + u] + (ent & 0x7FFFu), vr, vi);
              ar[k] += s_ec[nh + q + u] * vr;
              if (T::cplx) ai[k] += s_ec[nh + q + u] * vi;
            }
          }
        }
        const uint2* __restrict__ g = p.lgrp + rec[k].x;
        for (int c = 0; c < ncls; ++c) {
          const uint32_t ng = (rec[k].y >> (4 * c)) & 0xFu;
          R sr = R(0), si = R(0);
          for (uint32_t j = 0; j < ng; ++j) {
            const uint2 q = __ldg(g + j);
            R vr, vi;
            sld(sx, q.x & 0xFFFFu, vr, vi); sr += vr; if (T::cplx) si += vi;
            sld(sx, q.x >> 16, vr, vi);     sr += vr; if (T::cplx) si += vi;
            sld(sx, q.y & 0xFFFFu, vr, vi); sr += vr; if (T::cplx) si += vi;
            sld(sx, q.y >> 16, vr, vi);     sr += vr; if (T::cplx) si += vi;
          }
          g += ng;
          ar[k] += s_lc[c] * sr;
          if (T::cplx) ai[k] += s_lc[c] * si;
        }
        R x0r, x0i;
        sld(sx, r, x0r, x0i);
        // two-part operators read the full diagonal (summed in term order)
        const R d = GEN ? R(__ldg(p.diag_full + base + r)) : dh + R(dt[k]);
        ar[k] += d * x0r;
        if (T::cplx) ai[k] += d * x0i;
        if (flags & kRowStreamY) T::st_cs(y, base + r, ar[k], ai[k]);  // y is not read again here
        else T::st(y, base + r, ar[k], ai[k]);
        if (DOT) {
          dr += double(x0r) * double(ar[k]) + double(x0i) * double(ai[k]);
          di += double(x0r) * double(ai[k]) - double(x0i) * double(ar[k]);
        }
      }
    }
    if (DOT) {
      block_sum2(dr, di, s_dot);
      if (threadIdx.x == 0) { partials[2 * rec] = dr; partials[2 * rec + 1] = di; }
      dr = 0.0;
      di = 0.0;
    }
  }
  if (wq) wq_done(wq);
  if (DOT) grid_finish_items(partials, ticket, nA, dot_out);
}

// Block form of the row kernel for R vectors stored row-interleaved
// (element (i, r) at i*R + r): LPR lanes share a row and each covers VPL
// consecutive vectors with one vector load per target, so the class
// tables, block entries and crossing flags of a row are read once for all
// R vectors.  Same tables, same sums as k_hx_spin_rows; column dots
// <X_r, Y_r> reduced in a fixed order.
template <class E, int VPL>
struct alignas(sizeof(E) * VPL) BlkPack { E v[VPL]; };

// Registers are sized by the bytes a lane loads per target row: up to 16
// bytes four CTAs per SM (64 registers), up to 32 bytes two, wider one.  The
// kernel is latency-bound, so resident warps count more than the few words
// the narrow shapes spill (t-J N=20, 64 float64 vectors: 12.7 -> 9.5 ms per
// apply against one CTA per SM for every shape).  The tuner times them all.
template <int DT, int VPL>
constexpr int kBlockMinCta = VPL * int(sizeof(typename VT<DT>::E)) <= 16 ? 4
                             : VPL * int(sizeof(typename VT<DT>::E)) <= 32 ? 2 : 1;
template <int DT, bool GEN, int LPR, int VPL>
__global__ void __launch_bounds__(256, kBlockMinCta<DT, VPL>)
k_hx_rows_block(const SpinPlan* __restrict__ pp, const void* __restrict__ X, void* __restrict__ Y,
                double* partials, unsigned* ticket, double* dots, const double* __restrict__ gacc,
                uint32_t* wq, uint32_t nchunks, uint32_t qsplit, double* tile_part, const uint4* __restrict__ tiles) {
  using T = VT<DT>;
  using R = typename T::R;
  using E = typename T::E;
  using Pack = BlkPack<E, VPL>;
  constexpr int RV = LPR * VPL, RPW = 32 / LPR;
  constexpr int NBAT = VPL * sizeof(E) <= 16 ? 4 : 2;  // partner rows in flight per batch
  const SpinPlan& p = *pp;
  __shared__ R s_coef[kRowCoef], s_lc[kRowCls], s_ec[kRowEnt];
  __shared__ uint32_t s_eb[kRowEnt], s_ebit[kRowCross];
  for (int i = threadIdx.x; i < kRowCoef; i += blockDim.x) s_coef[i] = R(p.coef[i]);
  if (threadIdx.x < kRowCls) s_lc[threadIdx.x] = R(p.lcls[threadIdx.x]);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sub = lane / LPR, l = lane % LPR;
  const E* __restrict__ Xe = reinterpret_cast<const E*>(X);
  E* __restrict__ Ye = reinterpret_cast<E*>(Y);
  const uint32_t nll = p.nllist, zs = p.zero_slot;
  const int ncross = p.ncross, ncls = p.ncls;
  const uint32_t cpad = uint32_t(p.cpad);
  double dr[VPL], di[VPL];
  #pragma unroll
  for (int v = 0; v < VPL; ++v) { dr[v] = 0.0; di[v] = 0.0; }
  // gacc != NULL: Y += diag(gacc) (H X) instead of Y = H X (column c = l * VPL + v)
  R gcol[VPL];
  #pragma unroll
  for (int v = 0; v < VPL; ++v) gcol[v] = gacc ? R(gacc[l * VPL + v]) : R(1);
  auto ldrow = [&](uint32_t row, R* re, R* im) {
    const Pack pk = *reinterpret_cast<const Pack*>(Xe + size_t(row) * RV + l * VPL);
    #pragma unroll
    for (int v = 0; v < VPL; ++v) sld(pk.v, v, re[v], im[v]);
  };
  // Tiles of <= 256 rows in block order: the CTAs running at the same time
  // work on a few neighbouring blocks, whose rows (the low-bond targets)
  // then stay in L2 while they are gathered.  The tiles are handed out
  // grid-stride, or (wq) from a queue per die of the GPU, each die taking
  // its own contiguous share; with queues the column dots of every tile go
  // to tile_part and are summed in tile order, so they do not depend on
  // which CTA took which tile (grid-stride: per CTA, in CTA order).
  __shared__ uint32_t s_chunk[2];
  __shared__ double red[2 * (256 / 32) * RV];  // per-warp column sums (also the grid-stride form's scratch)
  int die = 0;
  if (wq) {
    uint32_t sid;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(sid));
    die = (p.sm_die && sid < p.nsmid) ? int(__ldg(p.sm_die + sid)) : 0;
  }
  auto fetch = [&](uint32_t prev) -> uint32_t {
    if (!wq) return prev + gridDim.x;
    for (int k = 0; k < 2; ++k) {
      const int q = die ^ k;
      const uint32_t beg = q ? qsplit : 0u, n = q ? nchunks - qsplit : qsplit;
      const uint32_t i = atomicAdd(wq + q, 1u);
      if (i < n) return beg + i;
    }
    return nchunks;
  };
  uint32_t chunk = blockIdx.x;
  if (wq) {
    if (threadIdx.x == 0) s_chunk[0] = fetch(0);
    __syncthreads();
    chunk = s_chunk[0];
  }
  for (uint32_t it = 1; chunk < nchunks; ++it) {
   {
    const uint32_t ti = chunk;
    const uint4 tile = __ldg(tiles + ti);
    const RowBlock cur = load_block(p.brec + tile.x);
    const uint32_t base = cur.base, size = tile.y + tile.z, nh = cur.nh;
    __syncthreads();
    if (threadIdx.x < nh + uint32_t(ncross)) {
      const uint2 e = __ldg(p.bent + cur.ebeg + threadIdx.x);
      s_eb[threadIdx.x] = e.x;
      s_ec[threadIdx.x] = (GEN && threadIdx.x >= nh) ? R(0) : s_coef[e.y & 0xFFFFu];
      if (threadIdx.x >= nh) s_ebit[threadIdx.x - nh] = GEN ? e.y : e.y >> 16;
    }
    __syncthreads();
    const double* __restrict__ dcol = p.dtab + size_t(cur.combo) * nll;
    uint32_t chm = 0u;
    if constexpr (GEN)
      for (int q = 0; q < ncross; ++q) chm |= (((s_ebit[q] >> 16) | (s_ebit[q] >> 18)) & 1u) << q;
    for (uint32_t r = tile.y + warp * RPW + sub; r < size; r += (256 / 32) * RPW) {
      const uint32_t pos = cur.lst + r, row = base + r;
      R x0r[VPL], x0i[VPL], ar[VPL], ai[VPL];
      ldrow(row, x0r, x0i);
      const R d = GEN ? R(__ldg(p.diag_full + row)) : R(cur.dh) + R(__ldg(dcol + pos));
      #pragma unroll
      for (int v = 0; v < VPL; ++v) { ar[v] = d * x0r[v]; ai[v] = T::cplx ? d * x0i[v] : R(0); }
      // low bonds: the row's target groups, by coefficient class
      const uint2 rec = __ldg(p.rrec + pos);
      const uint2* __restrict__ g = p.lgrp + rec.x;
      for (int c = 0; c < ncls; ++c) {
        const uint32_t ng = (rec.y >> (4 * c)) & 0xFu;
        R sr[VPL], si[VPL];
        #pragma unroll
        for (int v = 0; v < VPL; ++v) { sr[v] = R(0); si[v] = R(0); }
        for (uint32_t j = 0; j < ng; ++j) {
          const uint2 q = __ldg(g + j);
          const uint32_t kk[4] = {q.x & 0xFFFFu, q.x >> 16, q.y & 0xFFFFu, q.y >> 16};
          #pragma unroll
          for (int u = 0; u < 4; ++u) {
            if (kk[u] == zs) continue;  // padding of the group
            R vr[VPL], vi[VPL];
            ldrow(base + kk[u], vr, vi);
            #pragma unroll
            for (int v = 0; v < VPL; ++v) { sr[v] += vr[v]; if (T::cplx) si[v] += vi[v]; }
          }
        }
        g += ng;
        #pragma unroll
        for (int v = 0; v < VPL; ++v) { ar[v] += s_lc[c] * sr[v]; if (T::cplx) ai[v] += s_lc[c] * si[v]; }
      }
      // high bonds: the same row of a partner block, NBAT partner rows in
      // flight at a time
      for (uint32_t e0 = 0; e0 < nh; e0 += NBAT) {
        R vr[NBAT][VPL], vi[NBAT][VPL];
        #pragma unroll
        for (int u = 0; u < NBAT; ++u) {
          #pragma unroll
          for (int v = 0; v < VPL; ++v) { vr[u][v] = R(0); vi[u][v] = R(0); }
          if (e0 + u < nh) ldrow(s_eb[e0 + u] + r, vr[u], vi[u]);
        }
        #pragma unroll
        for (int u = 0; u < NBAT; ++u)
          if (e0 + u < nh) {
            const R c = s_ec[e0 + u];
            #pragma unroll
            for (int v = 0; v < VPL; ++v) { ar[v] += c * vr[u][v]; if (T::cplx) ai[v] += c * vi[u][v]; }
          }
      }
      // crossing bonds (two-part: only the groups the row's low mask and the
      // block's high mask both allow), NBAT groups at a time: their table
      // words, then their partner rows, in flight together
      for (uint32_t m = GEN ? (__ldg(p.crm + pos) & chm) : ((1u << ncross) - 1u); m;) {
        int qq[NBAT];
        uint32_t ent[NBAT];
        #pragma unroll
        for (int u = 0; u < NBAT; ++u) {
          qq[u] = m ? __ffs(m) - 1 : -1;
          m &= m - 1u;
          ent[u] = qq[u] < 0 ? 0u
                   : GEN ? __ldg(p.crk32 + size_t(qq[u]) * p.nllist + pos)
                         : uint32_t(__ldg(p.crk + size_t(pos) * cpad + qq[u]));
        }
        R cq[NBAT], vr[NBAT][VPL], vi[NBAT][VPL];
        #pragma unroll
        for (int u = 0; u < NBAT; ++u) {
          uint32_t rank = 0;
          cq[u] = R(0);
          if (qq[u] >= 0) {
            if constexpr (GEN) {
              cq[u] = cross_coef<R>(ent[u], s_ebit[qq[u]], s_coef);
              rank = ent[u] & 0xFFFFFFu;
            } else {
              if ((ent[u] >> 15) != s_ebit[qq[u]]) cq[u] = s_ec[nh + qq[u]];
              rank = ent[u] & 0x7FFFu;
            }
          }
          #pragma unroll
          for (int v = 0; v < VPL; ++v) { vr[u][v] = R(0); vi[u][v] = R(0); }
          if (cq[u] != R(0)) ldrow(s_eb[nh + qq[u]] + rank, vr[u], vi[u]);
        }
        #pragma unroll
        for (int u = 0; u < NBAT; ++u)
          if (cq[u] != R(0)) {
            #pragma unroll
            for (int v = 0; v < VPL; ++v) { ar[v] += cq[u] * vr[u][v]; if (T::cplx) ai[v] += cq[u] * vi[u][v]; }
          }
      }
      Pack yv;
      if (gacc) {
        const Pack y0 = *reinterpret_cast<const Pack*>(Ye + size_t(row) * RV + l * VPL);
        #pragma unroll
        for (int v = 0; v < VPL; ++v) {
          R y0r, y0i;
          sld(y0.v, v, y0r, y0i);
          ar[v] = y0r + gcol[v] * ar[v];
          if (T::cplx) ai[v] = y0i + gcol[v] * ai[v];
        }
      }
      #pragma unroll
      for (int v = 0; v < VPL; ++v) {
        T::st(yv.v, v, ar[v], ai[v]);
        if (T::cplx) {
          dr[v] += double(x0r[v]) * double(ar[v]) + double(x0i[v]) * double(ai[v]);
          di[v] += double(x0r[v]) * double(ai[v]) - double(x0i[v]) * double(ar[v]);
        } else {
          dr[v] += double(x0r[v]) * double(ar[v]);
        }
      }
      *reinterpret_cast<Pack*>(Ye + size_t(row) * RV + l * VPL) = yv;
    }
   }
    // queues: this tile's column dots in a fixed order (the rows a warp
    // holds by shuffles, then the warps in order), two barriers per tile
    if (tile_part) {
      #pragma unroll
      for (int v = 0; v < VPL; ++v)
        #pragma unroll
        for (int o = LPR; o < 32; o <<= 1) {
          dr[v] += __shfl_xor_sync(0xffffffffu, dr[v], o);
          if (T::cplx) di[v] += __shfl_xor_sync(0xffffffffu, di[v], o);
        }
      __syncthreads();  // the previous tile's sums have been read
      if (lane < LPR) {
        #pragma unroll
        for (int v = 0; v < VPL; ++v) {
          red[(warp * RV + l * VPL + v) * 2] = dr[v];
          red[(warp * RV + l * VPL + v) * 2 + 1] = T::cplx ? di[v] : 0.0;
        }
      }
      __syncthreads();
      for (int c = threadIdx.x; c < RV; c += 256) {
        double sr = 0.0, si = 0.0;
        for (int w = 0; w < 256 / 32; ++w) { sr += red[(w * RV + c) * 2]; si += red[(w * RV + c) * 2 + 1]; }
        tile_part[(size_t(c) * nchunks + chunk) * 2] = sr;
        tile_part[(size_t(c) * nchunks + chunk) * 2 + 1] = si;
      }
      #pragma unroll
      for (int v = 0; v < VPL; ++v) { dr[v] = 0.0; di[v] = 0.0; }
    }
    uint32_t cn = chunk + gridDim.x;
    if (wq) {
      if (threadIdx.x == 0) s_chunk[it & 1] = fetch(chunk);
      __syncthreads();
      cn = s_chunk[it & 1];
    }
    chunk = cn;
  }
  if (wq) wq_done(wq);
  if (tile_part) {
    grid_finish_n(tile_part, ticket, RV, dots, nchunks);
    return;
  }
  for (int v = 0; v < VPL; ++v) {
    __syncthreads();
    red[2 * threadIdx.x] = dr[v];
    red[2 * threadIdx.x + 1] = di[v];
    __syncthreads();
    if (threadIdx.x < LPR) {
      double sr = 0.0, si = 0.0;
      for (int t = threadIdx.x; t < 256; t += LPR) { sr += red[2 * t]; si += red[2 * t + 1]; }
      const int c = threadIdx.x * VPL + v;
      partials[(size_t(c) * gridDim.x + blockIdx.x) * 2] = sr;
      partials[(size_t(c) * gridDim.x + blockIdx.x) * 2 + 1] = si;
    }
  }
  grid_finish(partials, ticket, RV, dots);
}

}  // namespace

constexpr uint32_t kTileRows[3] = {256, 128, 512};  // tile shapes of the block kernel, by tile code

struct SpinHandle {
  SpinPlan host;
  SpinPlan* dev = nullptr;
  void* bufs[20] = {};
  const uint4* bt[3] = {};  // block-kernel tiles of kTileRows[i] rows
  uint32_t nbt[3] = {};
  uint32_t* wq = nullptr;  // per-die work queues (8 u32: row kernel, block kernel; zero between launches)
  int n0 = 0, n1 = 0;      // SMs of each die
  bool lean = false;       // every bond conserves the charge: row kernel
  // per-tile column-dot partials of the queued block kernel, sized on first use
  mutable std::mutex tp_mu;
  mutable double* tile_part = nullptr;
  mutable size_t tp_cap = 0;
};

void spin_plan_destroy(SpinHandle* h) {
  if (!h) return;
  for (void* b : h->bufs) cudaFree(b);
  cudaFree(h->tile_part);
  cudaFree(h->wq);
  cudaFree(h->dev);
  delete h;
}

bool die_map(const uint8_t** dev_map, int* nsmid, int* n0, int* n1);

// Per-die work queues (process-wide switch, for comparisons).
static bool g_die_queues = true;
// Launch flags of the row kernel: y is written once and not read again by
// the kernel, so it is stored with the streaming hint.
constexpr uint32_t g_row_flags = kRowStreamY;

// When the GPU has two dies: split the visiting sequence into a share per
// die in proportion to its SMs (by rows), and allocate the queue counters.
// Without them (one die, or no memory) the row kernel keeps its
// grid-stride order.
static void set_die_queues(SpinHandle* out, SpinPlan& h, const std::vector<RowBlock>& brec,
                           const std::vector<uint32_t>& bord, size_t* dev_bytes) {
  const uint8_t* map = nullptr;
  int nsmid = 0, n0 = 0, n1 = 0;
  if (!die_map(&map, &nsmid, &n0, &n1) || h.nblocks < 2) return;
  uint64_t total = 0;
  for (const RowBlock& b : brec) total += b.size;
  const uint64_t want = total * uint64_t(n0) / uint64_t(n0 + n1);
  uint64_t acc = 0;
  uint32_t split = 0;
  while (split < h.nblocks && acc < want) acc += brec[bord.empty() ? split : bord[split]].size, ++split;
  if (cudaMalloc(&out->wq, 8 * sizeof(uint32_t)) != cudaSuccess ||
      cudaMemset(out->wq, 0, 8 * sizeof(uint32_t)) != cudaSuccess) {
    (void)cudaGetLastError();
    cudaFree(out->wq);
    out->wq = nullptr;
    return;
  }
  *dev_bytes += 8 * sizeof(uint32_t);
  out->n0 = n0;
  out->n1 = n1;
  h.sm_die = map;
  h.nsmid = uint32_t(nsmid);
  h.qsplit = split;
}

// Visiting order of the 2^H sector blocks of a spin plan.  Blocks are
// visited as a counter whose fastest digits are the outer high bits (the
// lowest and highest 2H/7) and whose slowest digits are the middle ones.
// The partners of a block along bonds between neighbouring high bits, and
// along the two bonds that cross the split at either end (block h ^ 1 and
// h ^ 2^(H-1)), then lie within a short stretch of the visiting sequence,
// except for the bonds among the middle bits: for chains this leaves fewer
// partner reads beyond the reach of L2 than the ascending order, whose far
// partners include a crossing bond that every row has.  Heisenberg N=28
// Sz=0: an LRU model of a 100 MB L2 gives 3.2 instead of 3.9 reads of x per
// apply, measured 5-6% less time (complex128 and float64).
static std::vector<uint32_t> block_order(int H) {
  std::vector<int> fast;  // bit of h for each counter digit, fastest first
  const int k = H * 2 / 7;
  for (int b = 0; b < k; ++b) fast.push_back(b);
  for (int b = H - k; b < H; ++b) fast.push_back(b);
  for (int b = k; b < H - k; ++b) fast.push_back(b);
  std::vector<uint32_t> o(size_t(1) << H);
  for (uint32_t c = 0; c < o.size(); ++c) {
    uint32_t hh = 0;
    for (int i = 0; i < H; ++i) if ((c >> i) & 1u) hh |= 1u << fast[i];
    o[c] = hh;
  }
  return o;
}

// Runs of <= `rows` rows of each non-empty block record, in record order or
// in the visiting order `order` (record indices) when given.  The block
// kernel has three tile tables (kTileRows) for its shape tuner.
static std::vector<uint4> block_tiles(const std::vector<RowBlock>& brec,
                                      const std::vector<uint32_t>& order = std::vector<uint32_t>(),
                                      uint32_t rows = 256) {
  std::vector<uint4> t;
  for (uint32_t i = 0; i < uint32_t(brec.size()); ++i) {
    const uint32_t b = order.empty() ? i : order[i];
    for (uint32_t r = 0; r < brec[b].size; r += rows) t.push_back(make_uint4(b, r, std::min(rows, brec[b].size - r), 0));
  }
  if (t.empty()) t.push_back(make_uint4(0, 0, 0, 0));
  return t;
}

// Visiting order of the block records of a two-part plan (records of the
// non-empty blocks, high parts rec_h in ascending order): the counter of
// block_order over units of `unit` bits (2: the up and down bit of one site
// of a pair family), so the blocks reached by hops at either end of the high
// segment and across the split are visited close together.
static std::vector<uint32_t> record_order(const std::vector<uint32_t>& rec_h, int H, int unit) {
  const int nu = std::max(1, H / unit);
  std::vector<int> fast;  // unit of h for each counter digit, fastest first
  const int k = nu * 2 / 7;
  for (int u = 0; u < k; ++u) fast.push_back(u);
  for (int u = nu - k; u < nu; ++u) fast.push_back(u);
  for (int u = k; u < nu - k; ++u) fast.push_back(u);
  const uint32_t umask = (1u << unit) - 1u;
  std::vector<std::pair<uint64_t, uint32_t>> key(rec_h.size());
  for (uint32_t i = 0; i < uint32_t(rec_h.size()); ++i) {
    uint64_t c = 0;
    for (int d = 0; d < nu; ++d) c |= uint64_t((rec_h[i] >> (fast[d] * unit)) & umask) << (d * unit);
    key[i] = {c, i};
  }
  std::sort(key.begin(), key.end());
  std::vector<uint32_t> o(rec_h.size());
  for (size_t i = 0; i < key.size(); ++i) o[i] = key[i].second;
  return o;
}

// Host side: decide eligibility from the compiled plan and build the
// specialised tables.  Returns nullptr when the operator does not qualify.
SpinHandle* spin_plan_create(const qk_plan_desc* d, size_t* dev_bytes) {
  if (!d->all_real || d->nbits > 30 || d->dim >= (1ull << 32) || d->nterms == 0) return nullptr;
  const int L = d->L, H = d->nbits - d->L;
  if (L > 15 || H > 15 || L < 1) return nullptr;
  // single charge: every key is a plain popcount (or 0 without a sector)
  for (uint64_t l = 0; l < d->nB; ++l) {
    const uint32_t key = d->B[l] >> 24;
    if (key == qkb::kInvalidLowKey) return nullptr;
    if (key != uint32_t(__builtin_popcountll(l)) && key != 0) return nullptr;
    if ((d->B[l] & qkb::kRankMask) > 0xFFFF) return nullptr;
  }
  SpinPlan h{};
  h.L = L; h.H = H; h.dim = d->dim;
  uint32_t g0 = 0;
  if (d->has_diag) {
    const qk_group_t& g = d->groups[0];
    if (g.count > uint32_t(kMaxDiag)) return nullptr;
    for (uint32_t q = g.first; q < g.first + g.count; ++q) {
      const qk_term_t& t = d->terms[q];
      if (t.cmask != 0 || (t.smask >> 32)) return nullptr;
      h.diag_smask[h.ndiag] = uint32_t(t.smask);
      h.diag_w[h.ndiag] = t.wre;
      ++h.ndiag;
    }
    g0 = 1;
  }
  if (d->ngroups - g0 > uint32_t(kMaxBonds)) return nullptr;
  for (uint32_t gi = g0; gi < d->ngroups; ++gi) {
    const qk_group_t& g = d->groups[gi];
    if (__builtin_popcountll(g.flip) != 2 || g.check) return nullptr;
    SpinBond b{};
    const int i = __builtin_ctzll(g.flip), j = 63 - __builtin_clzll(g.flip);
    b.bi = uint8_t(i); b.bj = uint8_t(j);
    b.lo_mask = uint32_t(g.flip & ((1ull << L) - 1));
    b.hi_mask = uint32_t(g.flip >> L);
    b.kind = (j < L) ? 0 : (i >= L ? 1 : 2);
    for (uint32_t q = g.first; q < g.first + g.count; ++q) {
      const qk_term_t& t = d->terms[q];
      if (t.cmask != g.flip || (t.smask & ~g.flip)) return nullptr;
      const int combo = int(((t.cval >> i) & 1) | (((t.cval >> j) & 1) << 1));
      const int neg = __builtin_popcountll(t.cval & t.smask) & 1;
      b.c[combo] += neg ? -t.wre : t.wre;
      b.valid_mask |= uint8_t(1u << combo);
    }
    h.bonds[h.nbonds++] = b;
  }
  // Lean classification: only the charge-conserving combinations 01 / 10.
  bool lean = true;
  for (int q = 0; q < h.nbonds && lean; ++q) {
    const SpinBond& b = h.bonds[q];
    if (b.valid_mask & 0b1001) { lean = false; break; }
    const uint32_t mi = 1u << b.bi, mj = 1u << b.bj;
    // c01: bit i = 1, bit j = 0 is combo 1; bit i = 0, bit j = 1 is combo 2
    if (b.kind == 0) {
      h.low_mask[h.nlow] = mi | mj; h.low_i[h.nlow] = b.bi;
      h.low_c10[h.nlow] = b.c[1]; h.low_c01[h.nlow] = b.c[2]; ++h.nlow;
    } else if (b.kind == 1) {
      h.high_mask[h.nhigh] = (mi | mj) >> L; h.high_i[h.nhigh] = uint8_t(b.bi - L);
      h.high_c10[h.nhigh] = b.c[1]; h.high_c01[h.nhigh] = b.c[2]; ++h.nhigh;
    } else {
      h.cross_lo[h.ncross] = mi; h.cross_hi[h.ncross] = mj >> L; h.cross_li[h.ncross] = b.bi;
      // valid when bit i (low) != bit j (high); c10: low bit set
      h.cross_c10[h.ncross] = b.c[1]; h.cross_c01[h.ncross] = b.c[2]; ++h.ncross;
    }
  }
  std::vector<double> dhi(d->nA, 0.0), dlo(d->nllist, 0.0);
  if (lean) {
    const uint32_t lowbits = (1u << L) - 1u;
    for (int q = 0; q < h.ndiag; ++q) {
      const uint32_t m = h.diag_smask[q];
      const double w = h.diag_w[q];
      if ((m & ~lowbits) == 0) {
        for (uint64_t k = 0; k < d->nllist; ++k) dlo[k] += (__builtin_popcount(d->llist[k] & m) & 1) ? -w : w;
      } else if ((m & lowbits) == 0) {
        for (uint64_t k = 0; k < d->nA; ++k) dhi[k] += (__builtin_popcount(uint32_t(k) & (m >> L)) & 1) ? -w : w;
      } else {
        h.dcross_mask[h.ndcross] = m; h.dcross_w[h.ndcross] = w; ++h.ndcross;
      }
    }
  }

  // coefficient table and the per-part target lists the row tables are built from
  std::vector<uint32_t> loff, lent, hoff, hlst;
  std::vector<uint2> hent;
  if (lean) {
    auto coef_index = [&](double c) -> uint32_t {
      for (int k = 0; k < h.ncoef; ++k) if (h.coef[k] == c) return uint32_t(k);
      h.coef[h.ncoef] = c;
      return uint32_t(h.ncoef++);
    };
    loff.assign(d->nllist + 1, 0);
    for (uint64_t pos = 0; pos < d->nllist; ++pos) {
      const uint32_t l = d->llist[pos];
      loff[pos] = uint32_t(lent.size());
      for (int q = 0; q < h.nlow; ++q) {
        const uint32_t m = h.low_mask[q], v = l & m;
        if (v == 0 || v == m) continue;
        const double c = ((v >> h.low_i[q]) & 1u) ? h.low_c10[q] : h.low_c01[q];
        lent.push_back(((d->B[l ^ m] & 0xFFFFu) << 8) | coef_index(c));
      }
    }
    loff[d->nllist] = uint32_t(lent.size());
    hoff.assign(d->nA + 1, 0);
    for (uint64_t hh = 0; hh < d->nA; ++hh) {
      hoff[hh] = uint32_t(hent.size());
      if (uint32_t(d->A[hh] >> 56) == qkb::kEmptyBlockKey) continue;
      for (int q = 0; q < h.nhigh; ++q) {
        const uint32_t m = h.high_mask[q], v = uint32_t(hh) & m;
        if (v == 0 || v == m) continue;
        const double c = ((v >> h.high_i[q]) & 1u) ? h.high_c10[q] : h.high_c01[q];
        hent.push_back(make_uint2(uint32_t(d->A[hh ^ m] & qkb::kOffsetMask), coef_index(c)));
      }
    }
    hoff[d->nA] = uint32_t(hent.size());
    hlst.assign(d->nA, 0);
    for (uint64_t hh = 0; hh < d->nA; ++hh) {
      const uint32_t need = uint32_t(d->A[hh] >> 56);
      if (need == qkb::kEmptyBlockKey) continue;
      hlst[hh] = d->key_off[need];
      h.max_block = std::max<uint32_t>(h.max_block, d->key_off[need + 1] - d->key_off[need]);
    }
    if (lent.empty()) lent.push_back(0);
    if (hent.empty()) hent.push_back(make_uint2(0, 0));
  }

  // Row-kernel tables.  Eligibility: at most kRowCls distinct low-bond
  // coefficients and 15 groups of four per class and row, few enough
  // coefficients and per-block entries for the shared tables, the combined
  // diagonal table at most 16 MB, a free u16 index for the zero slot, and
  // every high-bond partner block of the same size as the block (which is
  // what keeps the coalesced high-bond loads in bounds).
  std::vector<uint2> rrec, lgrp, bent;
  std::vector<uint16_t> crk;
  std::vector<double> dtab;
  std::vector<RowBlock> brec;
  if (lean) {
    const uint32_t lowbits = (1u << L) - 1u;
    h.cpad = h.ncross ? (h.ncross + 1) & ~1 : 0;
    h.ncombo = 1 << h.ndcross;
    h.nllist = uint32_t(d->nllist);
    h.zero_slot = h.max_block;
    h.rows_ok = h.nhigh + h.ncross <= kRowEnt && h.ncross <= kRowCross && h.ndcross <= 6 &&
                d->nllist * uint64_t(h.ncombo) * 8 <= (16ull << 20) && h.max_block < 0xFFFFu;
    // low coefficient classes (by coefficient index of the list entries)
    int cls_of[2 * kMaxBonds];
    for (int k = 0; k < 2 * kMaxBonds; ++k) cls_of[k] = -1;
    for (uint32_t e = 0; e < loff[d->nllist] && h.rows_ok; ++e) {
      const uint32_t ci = lent[e] & 0xFFu;
      if (cls_of[ci] >= 0) continue;
      if (h.ncls == kRowCls) { h.rows_ok = false; break; }
      cls_of[ci] = h.ncls;
      h.lcls[h.ncls++] = h.coef[ci];
    }
    for (uint64_t hh = 0; hh < d->nA && h.rows_ok; ++hh) {
      if (uint32_t(d->A[hh] >> 56) == qkb::kEmptyBlockKey) continue;
      const uint32_t need = uint32_t(d->A[hh] >> 56), size = d->key_off[need + 1] - d->key_off[need];
      for (int q = 0; q < h.nhigh; ++q) {
        const uint32_t m = h.high_mask[q], v = uint32_t(hh) & m;
        if (v == 0 || v == m) continue;
        const uint32_t need2 = uint32_t(d->A[hh ^ m] >> 56);
        if (need2 == qkb::kEmptyBlockKey || d->key_off[need2 + 1] - d->key_off[need2] != size) h.rows_ok = false;
      }
    }
    if (h.rows_ok) {
      rrec.resize(d->nllist);
      std::vector<uint16_t> bucket[kRowCls];
      for (uint64_t pos = 0; pos < d->nllist && h.rows_ok; ++pos) {
        for (auto& b : bucket) b.clear();
        for (uint32_t e = loff[pos]; e < loff[pos + 1]; ++e)
          bucket[cls_of[lent[e] & 0xFFu]].push_back(uint16_t(lent[e] >> 8));
        uint32_t counts = 0;
        rrec[pos].x = uint32_t(lgrp.size());
        for (int c = 0; c < h.ncls; ++c) {
          auto& b = bucket[c];
          while (b.size() % 4) b.push_back(uint16_t(h.zero_slot));
          const uint32_t ng = uint32_t(b.size() / 4);
          if (ng > 15) { h.rows_ok = false; break; }
          counts |= ng << (4 * c);
          for (uint32_t k = 0; k < ng; ++k)
            lgrp.push_back(make_uint2(uint32_t(b[4 * k]) | (uint32_t(b[4 * k + 1]) << 16),
                                      uint32_t(b[4 * k + 2]) | (uint32_t(b[4 * k + 3]) << 16)));
        }
        rrec[pos].y = counts;
      }
      if (lgrp.empty()) lgrp.push_back(make_uint2(0, 0));
    }
    if (h.rows_ok) {
      crk.assign(std::max<uint64_t>(2, d->nllist * uint64_t(h.cpad)), 0);
      for (uint64_t pos = 0; pos < d->nllist; ++pos) {
        const uint32_t l = d->llist[pos];
        for (int q = 0; q < h.ncross; ++q) {
          const uint32_t bl = (l >> h.cross_li[q]) & 1u;
          crk[pos * h.cpad + q] = uint16_t((bl << 15) | (d->B[l ^ h.cross_lo[q]] & 0x7FFFu));
        }
      }
      dtab.assign(d->nllist * uint64_t(h.ncombo), 0.0);
      for (int c = 0; c < h.ncombo; ++c)
        for (uint64_t pos = 0; pos < d->nllist; ++pos) {
          const uint32_t l = d->llist[pos];
          double v = dlo[pos];
          for (int q = 0; q < h.ndcross; ++q) {
            const uint32_t par = ((c >> q) ^ __builtin_popcount(l & h.dcross_mask[q] & lowbits)) & 1u;
            v += par ? -h.dcross_w[q] : h.dcross_w[q];
          }
          dtab[c * d->nllist + pos] = v;
        }
      auto coef_index = [&](double c) -> uint32_t {
        for (int k = 0; k < h.ncoef; ++k) if (h.coef[k] == c) return uint32_t(k);
        h.coef[h.ncoef] = c;
        return uint32_t(h.ncoef++);
      };
      h.nblocks = uint32_t(d->nA);
      brec.resize(d->nA);
      for (uint64_t hh = 0; hh < d->nA; ++hh) {
        RowBlock& b = brec[hh];
        const uint32_t need = uint32_t(d->A[hh] >> 56);
        b.base = uint32_t(d->A[hh] & qkb::kOffsetMask);
        b.size = need == qkb::kEmptyBlockKey ? 0 : d->key_off[need + 1] - d->key_off[need];
        b.lst = hlst[hh];
        b.ebeg = uint32_t(bent.size());
        b.nh = hoff[hh + 1] - hoff[hh];
        b.dh = dhi[hh];
        b.combo = 0;
        for (int q = 0; q < h.ndcross; ++q)
          b.combo |= uint32_t(__builtin_popcount(uint32_t(hh) & (h.dcross_mask[q] >> L)) & 1) << q;
        for (uint32_t e = hoff[hh]; e < hoff[hh + 1]; ++e) bent.push_back(hent[e]);
        for (int q = 0; q < h.ncross; ++q) {
          const uint32_t bh = (uint32_t(hh) & h.cross_hi[q]) ? 1u : 0u;
          // valid rows have the opposite low bit: c01 (low 0, high 1) or c10
          const uint32_t ci = coef_index(bh ? h.cross_c01[q] : h.cross_c10[q]);
          bent.push_back(make_uint2(uint32_t(d->A[hh ^ h.cross_hi[q]] & qkb::kOffsetMask), ci | (bh << 16)));
        }
      }
      if (bent.empty()) bent.push_back(make_uint2(0, 0));
      if (h.ncoef > kRowCoef) h.rows_ok = false;
    }
  }

  std::vector<uint32_t> A32(d->nA);
  std::vector<uint16_t> B16(d->nB), l16(d->nllist);
  for (uint64_t k = 0; k < d->nA; ++k) A32[k] = uint32_t(d->A[k] & qkb::kOffsetMask);
  for (uint64_t k = 0; k < d->nB; ++k) B16[k] = uint16_t(d->B[k] & 0xFFFF);
  for (uint64_t k = 0; k < d->nllist; ++k) l16[k] = uint16_t(d->llist[k]);
  std::vector<qk_tile_t> tiles;
  for (uint64_t hh = 0; hh < d->nA; ++hh) {
    const uint32_t need = uint32_t(d->A[hh] >> 56);
    if (need == qkb::kEmptyBlockKey) continue;
    const uint32_t start = d->key_off[need], size = d->key_off[need + 1] - start;
    const uint64_t off = d->A[hh] & qkb::kOffsetMask;
    for (uint32_t r = 0; r < size; r += kSpinThreads)
      tiles.push_back(qk_tile_t{off + r, uint32_t(hh), start + r, std::min<uint32_t>(kSpinThreads, size - r), 0});
  }
  h.ntiles = uint32_t(tiles.size());
  h.smem = size_t(d->nA) * 4 + size_t(d->nB) * 2;
  if (h.smem > 160 * 1024) return nullptr;
  auto* out = new SpinHandle;
  out->lean = lean;
  auto up = [&](int slot, const void* src, size_t bytes) {
    if (cudaMalloc(&out->bufs[slot], bytes) != cudaSuccess) return false;
    *dev_bytes += bytes;
    return cudaMemcpy(out->bufs[slot], src, bytes, cudaMemcpyHostToDevice) == cudaSuccess;
  };
  bool ok = up(0, A32.data(), A32.size() * 4) && up(1, B16.data(), B16.size() * 2) &&
            up(2, l16.data(), l16.size() * 2) && up(3, tiles.data(), tiles.size() * sizeof(qk_tile_t)) &&
            (!h.rows_ok || (up(11, rrec.data(), rrec.size() * sizeof(uint2)) &&
                            up(12, lgrp.data(), lgrp.size() * sizeof(uint2)) && up(13, crk.data(), crk.size() * 2) &&
                            up(14, dtab.data(), dtab.size() * 8) &&
                            up(15, brec.data(), brec.size() * sizeof(RowBlock)) &&
                            up(16, bent.data(), bent.size() * sizeof(uint2))));
  const std::vector<uint4> btl = h.rows_ok ? block_tiles(brec) : std::vector<uint4>();
  ok = ok && (!h.rows_ok || up(18, btl.data(), btl.size() * sizeof(uint4)));
  std::vector<uint4> bt1, bt2;
  if (h.rows_ok) {
    bt1 = block_tiles(brec, std::vector<uint32_t>(), kTileRows[1]);
    bt2 = block_tiles(brec, std::vector<uint32_t>(), kTileRows[2]);
    ok = ok && up(6, bt1.data(), bt1.size() * sizeof(uint4)) && up(7, bt2.data(), bt2.size() * sizeof(uint4));
  }
  const std::vector<uint32_t> bord = h.rows_ok ? block_order(H) : std::vector<uint32_t>();
  ok = ok && (bord.empty() || up(19, bord.data(), bord.size() * 4));
  if (ok) {
    h.border = bord.empty() ? nullptr : static_cast<const uint32_t*>(out->bufs[19]);
    h.A32 = static_cast<const uint32_t*>(out->bufs[0]);
    h.B16 = static_cast<const uint16_t*>(out->bufs[1]);
    h.lrow = static_cast<const uint16_t*>(out->bufs[2]);
    h.tiles = static_cast<const qk_tile_t*>(out->bufs[3]);
    h.rrec = static_cast<const uint2*>(out->bufs[11]);
    h.lgrp = static_cast<const uint2*>(out->bufs[12]);
    h.crk = static_cast<const uint16_t*>(out->bufs[13]);
    h.dtab = static_cast<const double*>(out->bufs[14]);
    h.brec = static_cast<const RowBlock*>(out->bufs[15]);
    h.bent = static_cast<const uint2*>(out->bufs[16]);
    h.btiles = static_cast<const uint4*>(out->bufs[18]);
    h.nbtiles = uint32_t(btl.size());
    if (h.rows_ok) {
      out->bt[0] = h.btiles; out->nbt[0] = h.nbtiles;
      out->bt[1] = static_cast<const uint4*>(out->bufs[6]); out->nbt[1] = uint32_t(bt1.size());
      out->bt[2] = static_cast<const uint4*>(out->bufs[7]); out->nbt[2] = uint32_t(bt2.size());
      set_die_queues(out, h, brec, bord, dev_bytes);
    }
    out->host = h;
    ok = cudaMalloc(reinterpret_cast<void**>(&out->dev), sizeof(SpinPlan)) == cudaSuccess &&
         cudaMemcpy(out->dev, &h, sizeof(SpinPlan), cudaMemcpyHostToDevice) == cudaSuccess;
    if (ok) *dev_bytes += sizeof(SpinPlan);
  }
  if (!ok) {
    (void)cudaGetLastError();
    spin_plan_destroy(out);
    return nullptr;
  }
  return out;
}

// Two-part operators.  Every compiled term factorises over the sector
// split: its condition (s & cmask) == cval and its sign parity
// popcount(s & smask) are a condition and a parity of the low part times a
// condition and a parity of the high part.  Groups whose flip and terms lie
// in the low part become the class tables of the row kernel (their
// coefficient is a function of l), groups inside the high part become
// block entries (a function of h), and groups whose flip spans both parts
// (at most two terms) keep per-row low flags and per-block high flags that
// the kernel combines.  The diagonal is read from the plan's diagonal
// vector (summed in term order, as the reference sums it), set with
// spin_plan_set_diag.  This covers the Hubbard and t-J hops with their
// Jordan-Wigner signs, U Nupdn, the t-J spin-flip and density terms, and
// the spin models.
SpinHandle* gen_plan_create(const qk_plan_desc* d, size_t* dev_bytes) {
  if (!d->all_real || d->dim == 0 || d->dim >= (1ull << 32) || d->nterms == 0) return nullptr;
  const int L = d->L, H = d->nbits - d->L;
  if (L < 1 || L > 24 || H < 0 || H > 24 || d->nbits > 48) return nullptr;
  const uint64_t lowbits = (1ull << L) - 1;
  auto lo = [&](uint64_t v) { return uint32_t(v & lowbits); };
  auto hi = [&](uint64_t v) { return uint32_t(v >> L); };
  auto par = [](uint32_t v) { return uint32_t(__builtin_popcount(v) & 1); };
  SpinPlan h{};
  h.L = L; h.H = H; h.dim = d->dim; h.gen = true;
  for (uint32_t k = 0; k < d->nkeys; ++k) h.max_block = std::max(h.max_block, d->key_off[k + 1] - d->key_off[k]);
  if (h.max_block >= 0xFFFFu || size_t(h.max_block + 1) * 16 > 200 * 1024) return nullptr;
  auto coef_index = [&](double c) -> int {
    for (int k = 0; k < h.ncoef; ++k) if (h.coef[k] == c) return k;
    if (h.ncoef >= kRowCoef) return -1;
    h.coef[h.ncoef] = c;
    return h.ncoef++;
  };
  // classify the groups
  std::vector<uint32_t> lowg, highg, crossg;
  uint32_t g0 = 0;
  if (d->has_diag) g0 = 1;  // the diagonal comes from the plan's diagonal vector
  for (uint32_t gi = g0; gi < d->ngroups; ++gi) {
    const qk_group_t& g = d->groups[gi];
    if (g.check) return nullptr;  // targets must stay in the sector
    uint64_t m = g.flip;
    for (uint32_t q = g.first; q < g.first + g.count; ++q) m |= d->terms[q].cmask | d->terms[q].smask;
    if ((g.flip >> L) == 0 && (m >> L) == 0) lowg.push_back(gi);
    else if ((g.flip & lowbits) == 0 && (m & lowbits) == 0) highg.push_back(gi);
    else if ((g.flip & lowbits) != 0 && (g.flip >> L) != 0 && g.count <= 2) crossg.push_back(gi);
    else return nullptr;
  }
  h.ncross = int(crossg.size());
  if (h.ncross > kRowCross || highg.size() + crossg.size() > size_t(kRowEnt)) return nullptr;
  auto group_value = [&](const qk_group_t& g, uint32_t part, bool low) {
    double c = 0.0;
    for (uint32_t q = g.first; q < g.first + g.count; ++q) {
      const qk_term_t& t = d->terms[q];
      const uint32_t cm = low ? lo(t.cmask) : hi(t.cmask), cv = low ? lo(t.cval) : hi(t.cval);
      const uint32_t sm = low ? lo(t.smask) : hi(t.smask);
      if ((part & cm) == cv) c += par(part & sm) ? -t.wre : t.wre;
    }
    return c;
  };
  // class tables over llist positions
  const uint64_t nll = d->nllist;
  h.nllist = uint32_t(nll);
  h.zero_slot = h.max_block;
  h.ncombo = 1;
  std::vector<uint2> rrec(nll), lgrp;
  std::vector<double> dtab(nll, 0.0);
  std::vector<uint32_t> crk32(std::max<uint64_t>(1, nll * crossg.size()), 0);
  std::vector<uint32_t> crm(std::max<uint64_t>(1, nll), 0);
  std::vector<double> cls;
  std::vector<uint16_t> bucket[kRowCls];
  for (uint64_t pos = 0; pos < nll; ++pos) {
    const uint32_t l = d->llist[pos];
    const uint32_t key = d->B[l] >> 24;
    for (auto& b : bucket) b.clear();
    for (uint32_t gi : lowg) {
      const qk_group_t& g = d->groups[gi];
      const double c = group_value(g, l, true);
      if (c == 0.0) continue;
      const uint32_t lt = l ^ lo(g.flip);
      if ((d->B[lt] >> 24) != key) return nullptr;  // low groups must keep the low part's charges
      int ci = -1;
      for (int k = 0; k < int(cls.size()); ++k) if (cls[k] == c) ci = k;
      if (ci < 0) {
        if (int(cls.size()) == kRowCls) return nullptr;
        cls.push_back(c);
        ci = int(cls.size()) - 1;
      }
      bucket[ci].push_back(uint16_t(d->B[lt] & 0xFFFFu));
    }
    rrec[pos].x = uint32_t(lgrp.size());
    uint32_t counts = 0;
    for (int c = 0; c < kRowCls; ++c) {
      auto& b = bucket[c];
      if (b.empty()) continue;
      while (b.size() % 4) b.push_back(uint16_t(h.zero_slot));
      const uint32_t ng = uint32_t(b.size() / 4);
      if (ng > 15) return nullptr;
      counts |= ng << (4 * c);
      for (uint32_t k = 0; k < ng; ++k)
        lgrp.push_back(make_uint2(uint32_t(b[4 * k]) | (uint32_t(b[4 * k + 1]) << 16),
                                  uint32_t(b[4 * k + 2]) | (uint32_t(b[4 * k + 3]) << 16)));
    }
    rrec[pos].y = counts;
    for (size_t q = 0; q < crossg.size(); ++q) {
      const qk_group_t& g = d->groups[crossg[q]];
      const uint32_t lt = l ^ lo(g.flip);
      uint32_t e = (d->B[lt] & qkb::kRankMask) & 0xFFFFFFu;
      if ((d->B[lt] & qkb::kRankMask) > 0xFFFFFFu) return nullptr;
      for (uint32_t k = 0; k < g.count; ++k) {
        const qk_term_t& t = d->terms[g.first + k];
        const uint32_t lv = (l & lo(t.cmask)) == lo(t.cval), ls = par(l & lo(t.smask));
        e |= (lv << (24 + 2 * k)) | (ls << (25 + 2 * k));
      }
      crk32[q * nll + pos] = e;
      if (e & ((1u << 24) | (1u << 26))) crm[pos] |= 1u << q;
    }
  }
  if (lgrp.empty()) lgrp.push_back(make_uint2(0, 0));
  h.ncls = int(cls.size());
  for (int c = 0; c < h.ncls; ++c) h.lcls[c] = cls[c];
  // block records of the non-empty blocks
  std::vector<RowBlock> brec;
  std::vector<uint2> bent;
  std::vector<uint32_t> rec_h;
  for (uint64_t hh = 0; hh < d->nA; ++hh) {
    const uint32_t need = uint32_t(d->A[hh] >> 56);
    if (need == qkb::kEmptyBlockKey) continue;
    const uint32_t size = d->key_off[need + 1] - d->key_off[need];
    if (size == 0) continue;
    rec_h.push_back(uint32_t(hh));
    RowBlock b{};
    b.base = uint32_t(d->A[hh] & qkb::kOffsetMask);
    b.size = size;
    b.lst = d->key_off[need];
    b.ebeg = uint32_t(bent.size());
    b.dh = 0.0;
    for (uint32_t gi : highg) {
      const qk_group_t& g = d->groups[gi];
      const double c = group_value(g, uint32_t(hh), false);
      if (c == 0.0) continue;
      const uint64_t hp = hh ^ hi(g.flip);
      const uint32_t need2 = uint32_t(d->A[hp] >> 56);
      if (need2 != need) return nullptr;  // high groups must keep the high part's charges
      const int ci = coef_index(c);
      if (ci < 0) return nullptr;
      bent.push_back(make_uint2(uint32_t(d->A[hp] & qkb::kOffsetMask), uint32_t(ci)));
      ++b.nh;
    }
    for (uint32_t gi : crossg) {
      const qk_group_t& g = d->groups[gi];
      const uint64_t hp = hh ^ hi(g.flip);
      const bool pempty = uint32_t(d->A[hp] >> 56) == qkb::kEmptyBlockKey;
      uint32_t f = 0;
      for (uint32_t k = 0; k < g.count; ++k) {
        const qk_term_t& t = d->terms[g.first + k];
        const int ci = coef_index(t.wre);
        if (ci < 0) return nullptr;
        const uint32_t hv = !pempty && (uint32_t(hh) & hi(t.cmask)) == hi(t.cval), hs = par(uint32_t(hh) & hi(t.smask));
        f |= (uint32_t(ci) << (8 * k)) | (hv << (16 + 2 * k)) | (hs << (17 + 2 * k));
      }
      bent.push_back(make_uint2(uint32_t(d->A[hp] & qkb::kOffsetMask), f));
    }
    brec.push_back(b);
  }
  if (brec.empty()) return nullptr;
  if (bent.empty()) bent.push_back(make_uint2(0, 0));
  h.nblocks = uint32_t(brec.size());
  h.rows_ok = true;
  std::vector<uint16_t> crk_dummy(2, 0);
  auto* out = new SpinHandle;
  out->lean = true;
  auto up = [&](int slot, const void* src, size_t bytes) {
    if (cudaMalloc(&out->bufs[slot], bytes) != cudaSuccess) return false;
    *dev_bytes += bytes;
    return cudaMemcpy(out->bufs[slot], src, bytes, cudaMemcpyHostToDevice) == cudaSuccess;
  };
  bool ok = up(11, rrec.data(), rrec.size() * sizeof(uint2)) && up(12, lgrp.data(), lgrp.size() * sizeof(uint2)) &&
            up(13, crk_dummy.data(), 4) && up(14, dtab.data(), dtab.size() * 8) &&
            up(15, brec.data(), brec.size() * sizeof(RowBlock)) && up(16, bent.data(), bent.size() * sizeof(uint2)) &&
            up(17, crk32.data(), crk32.size() * 4) && up(19, crm.data(), crm.size() * 4);
  // the row kernel visits the records in the two-bit-unit order (sites of a
  // pair family: t-J N=20 0.47 -> 0.41 ms per apply); the block kernel keeps
  // record order, where its tiles of neighbouring blocks gather better
  // (batched FTLM on the same chain: 0.86 s in record order, 0.92 s in the
  // visiting order)
  const std::vector<uint32_t> rord = record_order(rec_h, H, (L % 2 == 0 && H % 2 == 0) ? 2 : 1);
  const std::vector<uint4> tiles = block_tiles(brec);
  const std::vector<uint4> t1 = block_tiles(brec, std::vector<uint32_t>(), kTileRows[1]);
  const std::vector<uint4> t2 = block_tiles(brec, std::vector<uint32_t>(), kTileRows[2]);
  ok = ok && up(18, tiles.data(), tiles.size() * sizeof(uint4)) && up(10, rord.data(), rord.size() * 4) &&
       up(6, t1.data(), t1.size() * sizeof(uint4)) && up(7, t2.data(), t2.size() * sizeof(uint4));
  if (ok) {
    h.rrec = static_cast<const uint2*>(out->bufs[11]);
    h.lgrp = static_cast<const uint2*>(out->bufs[12]);
    h.crk = static_cast<const uint16_t*>(out->bufs[13]);
    h.dtab = static_cast<const double*>(out->bufs[14]);
    h.brec = static_cast<const RowBlock*>(out->bufs[15]);
    h.bent = static_cast<const uint2*>(out->bufs[16]);
    h.crk32 = static_cast<const uint32_t*>(out->bufs[17]);
    h.crm = static_cast<const uint32_t*>(out->bufs[19]);
    h.border = static_cast<const uint32_t*>(out->bufs[10]);
    h.btiles = static_cast<const uint4*>(out->bufs[18]);
    h.nbtiles = uint32_t(tiles.size());
    out->bt[0] = h.btiles; out->nbt[0] = h.nbtiles;
    out->bt[1] = static_cast<const uint4*>(out->bufs[6]); out->nbt[1] = uint32_t(t1.size());
    out->bt[2] = static_cast<const uint4*>(out->bufs[7]); out->nbt[2] = uint32_t(t2.size());
    set_die_queues(out, h, brec, rord, dev_bytes);
    out->host = h;
    ok = cudaMalloc(reinterpret_cast<void**>(&out->dev), sizeof(SpinPlan)) == cudaSuccess &&
         cudaMemcpy(out->dev, &h, sizeof(SpinPlan), cudaMemcpyHostToDevice) == cudaSuccess;
    if (ok) *dev_bytes += sizeof(SpinPlan);
  }
  if (!ok) {
    (void)cudaGetLastError();
    spin_plan_destroy(out);
    return nullptr;
  }
  return out;
}

int spin_apply_rows(const SpinHandle* h, qk_dtype t, const void* x, void* y, cudaStream_t s,
                    qk_workspace* w, double* dot_out, uint64_t row_lo = 0, uint64_t row_hi = ~0ull) {
  if (!h->host.rows_ok || (h->host.gen && !h->host.diag_full)) return QKD_EINVAL;
  const size_t es = (t == QK_C128) ? 16 : (t == QK_F32 ? 4 : 8);
  const size_t smem = es * (h->host.max_block + 1);  // staged block and the zero slot
  if (smem > 200 * 1024) return QKD_EINVAL;
  uint32_t* const wq = g_die_queues ? h->wq : nullptr;
  if (dot_out && size_t(h->host.nblocks) > size_t(kMaxK) * kMaxG) return QKD_EINVAL;  // one partial per block
  const uint32_t rlo = uint32_t(std::min<uint64_t>(row_lo, 0xFFFFFFFFull));
  const uint32_t rhi = uint32_t(std::min<uint64_t>(row_hi, 0xFFFFFFFFull));
#define QKD_ROWS_LAUNCH1(DT, G)                                                                           \
  {                                                                                                       \
    auto kd = k_hx_spin_rows<DT, true, G>;                                                                \
    auto kn = k_hx_spin_rows<DT, false, G>;                                                               \
    if (cudaFuncSetAttribute(kd, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess ||  \
        cudaFuncSetAttribute(kn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)    \
      return QKD_EINVAL;                                                                                  \
    const unsigned cap = std::max(1u, h->host.nblocks);                                                   \
    if (dot_out) kd<<<resident_grid(kd, kRowNT<DT>, smem, std::min<unsigned>(cap, kMaxG)), kRowNT<DT>, smem, s>>>( \
        h->dev, x, y, w->partials, w->ticket, dot_out, wq, rlo, rhi, g_row_flags);                        \
    else kn<<<resident_grid(kn, kRowNT<DT>, smem, cap), kRowNT<DT>, smem, s>>>(h->dev, x, y, nullptr, nullptr, \
                                                                                 nullptr, wq, rlo, rhi,   \
                                                                                 g_row_flags);            \
  }
#define QKD_ROWS_LAUNCH(DT) { if (h->host.gen) QKD_ROWS_LAUNCH1(DT, true) else QKD_ROWS_LAUNCH1(DT, false) }
  switch (t) {
    case QK_C128: QKD_ROWS_LAUNCH(QK_C128); break;
    case QK_C64: QKD_ROWS_LAUNCH(QK_C64); break;
    case QK_F64: QKD_ROWS_LAUNCH(QK_F64); break;
    case QK_F32: QKD_ROWS_LAUNCH(QK_F32); break;
    default: return QKD_EINVAL;
  }
#undef QKD_ROWS_LAUNCH
#undef QKD_ROWS_LAUNCH1
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

template <int DT, bool GEN, int LPR, int VPL>
int launch_rows_block(const SpinHandle* h, qk_workspace* w, const void* X, void* Y, double* dots, cudaStream_t s,
                      const double* gacc, int tilec) {
  auto k = k_hx_rows_block<DT, GEN, LPR, VPL>;
  constexpr uint32_t RV = uint32_t(LPR * VPL);
  if (tilec < 0 || tilec > 2 || !h->bt[tilec]) tilec = 0;
  const uint4* tiles = h->bt[tilec] ? h->bt[tilec] : h->host.btiles;
  const uint32_t nt = std::max(1u, h->bt[tilec] ? h->nbt[tilec] : h->host.nbtiles);
  const unsigned g = resident_grid(k, 256, 0, std::min<unsigned>(nt, kMaxG));
  uint32_t* wq = nullptr;
  uint32_t qsplit = nt;
  double* tp = nullptr;
  if (g_die_queues && h->wq && h->host.sm_die) {
    // per-tile dot partials for the queued form (RV columns, 2 doubles each)
    std::lock_guard<std::mutex> lk(h->tp_mu);
    const size_t need = size_t(nt) * RV * 2;
    cudaStreamCaptureStatus cap_st = cudaStreamCaptureStatusNone;
    const bool capturing = cudaStreamIsCapturing(s, &cap_st) != cudaSuccess || cap_st != cudaStreamCaptureStatusNone;
    if (h->tp_cap < need && !capturing) {  // (a graph keeps the grid-stride form unless sized before capture)
      cudaFree(h->tile_part);
      h->tile_part = nullptr;
      h->tp_cap = 0;
      if (cudaMalloc(&h->tile_part, need * sizeof(double)) == cudaSuccess) h->tp_cap = need;
      else (void)cudaGetLastError();
    }
    if (h->tile_part && h->tp_cap >= need) {
      tp = h->tile_part;
      wq = h->wq + 4;
      qsplit = uint32_t(uint64_t(nt) * h->n0 / std::max(1, h->n0 + h->n1));
    }
  }
  k<<<g, 256, 0, s>>>(h->dev, X, Y, w->partials, w->ticket, dots ? dots : qkd_workspace_results(w), gacc, wq, nt,
                      qsplit, tp, tiles);
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

template <int DT, bool GEN>
int rows_block_shape(const SpinHandle* h, qk_workspace* w, int R, int lpr, const void* X, void* Y, double* dots,
                     cudaStream_t s, const double* gacc, int tilec) {
#define QKD_RB(RR, L, V) if (R == RR && lpr == L) return launch_rows_block<DT, GEN, L, V>(h, w, X, Y, dots, s, gacc, tilec);
  QKD_RB(32, 32, 1) QKD_RB(32, 16, 2) QKD_RB(32, 8, 4)
  QKD_RB(64, 32, 2) QKD_RB(64, 16, 4) QKD_RB(64, 8, 8)
  QKD_RB(128, 32, 4) QKD_RB(128, 16, 8)
#undef QKD_RB
  return QKD_EINVAL;
}

// Block apply with the row-kernel tables; QKD_EINVAL when this plan has none.
// gacc != NULL (R device doubles): Y += diag(gacc) (H X) instead of Y = H X.
int spin_apply_block(const SpinHandle* h, qk_dtype t, int R, int lpr, const void* X, void* Y, double* dots,
                     cudaStream_t s, qk_workspace* w, const double* gacc, int tilec) {
  if (!h || !h->host.rows_ok || !h->host.btiles || (h->host.gen && !h->host.diag_full)) return QKD_EINVAL;
  if (h->host.gen) { QKD_DISPATCH(t, return rows_block_shape<DT, true>(h, w, R, lpr, X, Y, dots, s, gacc, tilec)); }
  QKD_DISPATCH(t, return rows_block_shape<DT, false>(h, w, R, lpr, X, Y, dots, s, gacc, tilec));
  return QKD_EINVAL;
}

bool spin_plan_is_gen(const SpinHandle* h) { return h && h->host.gen; }

// Two-part plans read the operator's diagonal vector (device, dim doubles);
// without one they cannot run (spin_apply_rows reports QKD_EINVAL).
int spin_plan_set_diag(SpinHandle* h, const double* diag) {
  if (!h) return QKD_EINVAL;
  h->host.diag_full = diag;
  return cudaMemcpy(h->dev, &h->host, sizeof(SpinPlan), cudaMemcpyHostToDevice) == cudaSuccess ? QKD_OK : QKD_ECUDA;
}

static int spin_apply_impl(const SpinHandle* h, qk_dtype t, const void* x, void* y, cudaStream_t s, qk_workspace* w,
                           double* dot_out, uint64_t row_lo, uint64_t row_hi) {
  if (h->host.gen) return spin_apply_rows(h, t, x, y, s, w, dot_out, row_lo, row_hi);
  if (h->lean) {  // the row kernel where its tables exist; otherwise the bond kernel below
    const int rc = spin_apply_rows(h, t, x, y, s, w, dot_out, row_lo, row_hi);
    if (rc != QKD_EINVAL) return rc;
  }
  const size_t smem = h->host.smem;
  const unsigned grid = std::max(1u, std::min<unsigned>(h->host.ntiles, unsigned(sm_count(0)) * 1));
#define QKD_SPIN_LAUNCH(DT)                                                                             \
  {                                                                                                     \
    if (dot_out) {                                                                                      \
      auto k = k_hx_spin<DT, true>;                                                                     \
      if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess) \
        return QKD_EINVAL;                                                                              \
      k<<<std::min<unsigned>(grid, kMaxG), kSpinThreads, smem, s>>>(h->dev, x, y, w->partials, w->ticket, \
                                                                     dot_out, row_lo, row_hi);          \
    } else {                                                                                            \
      auto k = k_hx_spin<DT, false>;                                                                    \
      if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess) \
        return QKD_EINVAL;                                                                              \
      k<<<grid, kSpinThreads, smem, s>>>(h->dev, x, y, nullptr, nullptr, nullptr, row_lo, row_hi);      \
    }                                                                                                   \
  }
  switch (t) {
    case QK_C128: QKD_SPIN_LAUNCH(QK_C128); break;
    case QK_C64: QKD_SPIN_LAUNCH(QK_C64); break;
    case QK_F64: QKD_SPIN_LAUNCH(QK_F64); break;
    case QK_F32: QKD_SPIN_LAUNCH(QK_F32); break;
    default: return QKD_EINVAL;
  }
#undef QKD_SPIN_LAUNCH
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

int spin_apply(const SpinHandle* h, qk_dtype t, const void* x, void* y, cudaStream_t s, qk_workspace* w,
               double* dot_out) {
  return spin_apply_impl(h, t, x, y, s, w, dot_out, 0, ~0ull);
}

// Rows [row_lo, row_hi) only (block-aligned bounds); no fused dot.
int spin_apply_range(const SpinHandle* h, qk_dtype t, const void* x, void* y, cudaStream_t s, uint64_t row_lo,
                     uint64_t row_hi) {
  return spin_apply_impl(h, t, x, y, s, nullptr, nullptr, row_lo, row_hi);
}

void spin_set_die_queues(bool on) { g_die_queues = on; }

}  // namespace qkd

