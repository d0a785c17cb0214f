// H.x for operators with the spin-product structure of the Hubbard model:
// two bits per site (up at bit 2i, down at 2i+1), N_up and N_dn conserved,
// every off-diagonal term a hop of one spin species.  In the basis ordered by
// (up configuration, down configuration), with the sign
//   S(u, d) = (-1)^(number of pairs (down at site i, up at site j > i)),
// the reference's matrix is exactly
//   S H S = T_up (x) 1 + 1 (x) T_dn + D
// (the Jordan-Wigner strings of one species no longer see the other): a
// sparse matrix over the up configurations acting on whole rows of the
// product-ordered vector, one over the down configurations acting inside each
// row, and the diagonal.  The plan builder derives T_up and T_dn from the
// compiled terms and checks the structure before it is used (any failure:
// no plan, the two-part row kernel stays in charge).
//
// One apply is three passes over the vector:
//   k_pair_in   x_p[u][d] = S(u, d) x[rank(u, d)]       (reference -> product order)
//   k_pair_up   y_p[u][:] = sum_u' T_up[u][u'] x_p[u'][:]  (rows of the product
//               order; CTAs sweep column slabs so the partner rows of a slab
//               stay in L2)
//   k_pair_dn   y[rank(u, d)] = S(u, d) (y_p[u][d] + D[u][d] x_p[u][d]
//               + sum_d' T_dn[d][d'] x_p[u][d'])  (row u staged in shared memory;
//               fused column dot <x, y> when asked)
// rank(u, d) is the reference's index of the interleaved state, from the
// sector's two-level tables (offset of the high part + rank of the low part).
#include <algorithm>
#include <mutex>
#include <vector>

#include "reduce.cuh"
#include "../engine/sector.hpp"

namespace qkd {

struct PairPlan {
  uint32_t Du, Dd;         // up and down configurations
  int L;                   // low bits of the sector tables
  uint32_t lmask;
  const uint64_t* A;       // sector tables (device copies owned by the qk_plan)
  const uint32_t* B;
  const uint32_t* ulist;   // up configurations (compressed site bits), ascending
  const uint32_t* dlist;
  const uint32_t* up_ptr;  // CSR of T_up over configuration indices (Du + 1)
  const uint32_t* up_col;
  const double* up_val;
  const uint32_t* dn_ptr;  // CSR of T_dn (Dd + 1)
  const uint16_t* dn_ent;  // column | (sign << 15) when every |T_dn| equals dn_mag
  const uint32_t* dn_col;  // otherwise columns and values
  const double* dn_val;
  double dn_mag;
  const double* diag;      // D in product order (Du * Dd)
  const uint32_t* perm;    // rank(u, d) in product order (Du * Dd), or null: computed from A, B
};

namespace {

constexpr int kPT = 256;  // threads per CTA; k_pair_up takes row slabs of 2 * kPT elements
constexpr int kDT = 1024; // k_pair_dn: one staged row shared by 32 warps (two CTAs per SM)

__device__ __forceinline__ uint32_t spread16(uint32_t x) {  // bit i -> bit 2i (16 -> 32 bits)
  x &= 0xFFFFu;
  x = (x | (x << 8)) & 0x00FF00FFu;
  x = (x | (x << 4)) & 0x0F0F0F0Fu;
  x = (x | (x << 2)) & 0x33333333u;
  x = (x | (x << 1)) & 0x55555555u;
  return x;
}

// S(u, d): parity of the pairs (down at i, up at j > i) = parity(u & P) with
// P_j = XOR of d's bits below j
__device__ __forceinline__ double pair_sign(uint32_t u, uint32_t d) {
  uint32_t p = d << 1;
  p ^= p << 1; p ^= p << 2; p ^= p << 4; p ^= p << 8; p ^= p << 16;
  return (__popc(u & p) & 1) ? -1.0 : 1.0;
}

__device__ __forceinline__ uint32_t pair_rank(const PairPlan& p, uint32_t u, uint32_t d) {
  const uint32_t s = spread16(u) | (spread16(d) << 1);
  return uint32_t(__ldg(p.A + (s >> p.L)) & qkb::kOffsetMask) + (__ldg(p.B + (s & p.lmask)) & qkb::kRankMask);
}

// SIGN false: the plain gather (the diagonal, on which S acts twice)
template <int DT, bool SIGN>
__global__ void __launch_bounds__(kPT) k_pair_in(const PairPlan* __restrict__ pp, const void* __restrict__ x,
                                                 void* __restrict__ xp) {
  using T = VT<DT>;
  using R = typename T::R;
  const PairPlan& p = *pp;
  const uint64_t n = uint64_t(p.Du) * p.Dd;
  for (uint64_t i = blockIdx.x * uint64_t(kPT) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * kPT) {
    const uint32_t iu = uint32_t(i / p.Dd), id = uint32_t(i - uint64_t(iu) * p.Dd);
    const uint32_t u = __ldg(p.ulist + iu), d = __ldg(p.dlist + id);
    R re, im;
    T::ld(x, p.perm ? __ldg(p.perm + i) : pair_rank(p, u, d), re, im);
    const R sg = SIGN ? R(pair_sign(u, d)) : R(1);
    T::st(xp, i, sg * re, sg * im);
  }
}

// perm[i] = rank(u, d) for the product index i = iu * Dd + id
__global__ void __launch_bounds__(kPT) k_pair_perm(const PairPlan* __restrict__ pp, uint32_t* __restrict__ perm) {
  const PairPlan& p = *pp;
  const uint64_t n = uint64_t(p.Du) * p.Dd;
  for (uint64_t i = blockIdx.x * uint64_t(kPT) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * kPT) {
    const uint32_t iu = uint32_t(i / p.Dd), id = uint32_t(i - uint64_t(iu) * p.Dd);
    perm[i] = pair_rank(p, __ldg(p.ulist + iu), __ldg(p.dlist + id));
  }
}

// y_p[u][c0 .. c0 + 2 kPT) = sum_u' T_up[u][u'] x_p[u'][...]: work item
// (slab, u) in slab-major order, two elements per thread
template <int DT>
__global__ void __launch_bounds__(kPT) k_pair_up(const PairPlan* __restrict__ pp, const void* __restrict__ xp,
                                                 void* __restrict__ yp) {
  using T = VT<DT>;
  using R = typename T::R;
  const PairPlan& p = *pp;
  const uint32_t slab_elems = 2 * kPT;
  const uint32_t nslab = (p.Dd + slab_elems - 1) / slab_elems;
  const uint64_t items = uint64_t(nslab) * p.Du;
  for (uint64_t it = blockIdx.x; it < items; it += gridDim.x) {
    const uint32_t slab = uint32_t(it / p.Du), iu = uint32_t(it - uint64_t(slab) * p.Du);
    const uint32_t c0 = slab * slab_elems + threadIdx.x, c1 = c0 + kPT;
    const uint32_t k0 = __ldg(p.up_ptr + iu), k1 = __ldg(p.up_ptr + iu + 1);
    R a0r = R(0), a0i = R(0), a1r = R(0), a1i = R(0);
    const bool in0 = c0 < p.Dd, in1 = c1 < p.Dd;
    uint32_t k = k0;
    for (; k + 4 <= k1; k += 4) {  // four partner rows in flight
      uint32_t col[4];
      R w[4], v0r[4], v0i[4], v1r[4], v1i[4];
      #pragma unroll
      for (int j = 0; j < 4; ++j) {
        col[j] = __ldg(p.up_col + k + j);
        w[j] = R(__ldg(p.up_val + k + j));
        const uint64_t rb = uint64_t(col[j]) * p.Dd;
        v0r[j] = v0i[j] = v1r[j] = v1i[j] = R(0);
        if (in0) T::ld(xp, rb + c0, v0r[j], v0i[j]);
        if (in1) T::ld(xp, rb + c1, v1r[j], v1i[j]);
      }
      #pragma unroll
      for (int j = 0; j < 4; ++j) {
        a0r += w[j] * v0r[j]; a1r += w[j] * v1r[j];
        if (T::cplx) { a0i += w[j] * v0i[j]; a1i += w[j] * v1i[j]; }
      }
    }
    for (; k < k1; ++k) {
      const uint64_t rb = uint64_t(__ldg(p.up_col + k)) * p.Dd;
      const R w = R(__ldg(p.up_val + k));
      R vr = R(0), vi = R(0);
      if (in0) { T::ld(xp, rb + c0, vr, vi); a0r += w * vr; if (T::cplx) a0i += w * vi; }
      if (in1) { T::ld(xp, rb + c1, vr, vi); a1r += w * vr; if (T::cplx) a1i += w * vi; }
    }
    const uint64_t ob = uint64_t(iu) * p.Dd;
    if (in0) T::st(yp, ob + c0, a0r, a0i);
    if (in1) T::st(yp, ob + c1, a1r, a1i);
  }
}

// NR rows u of the product order staged in shared memory; per column d the
// down hops' table words are read once and serve all NR rows; per element
// the hops and the diagonal are added to y_p and the result goes to its
// reference-order slot with the sign S.  DOT: <x, y> summed per CTA in a
// fixed order, then over CTAs (deterministic for a given grid).
template <class E, int NR>
struct alignas(sizeof(E) * NR) RowPack { E v[NR]; };

template <int DT, bool DOT, int NR>
__global__ void __launch_bounds__(kDT) k_pair_dn(const PairPlan* __restrict__ pp, const void* __restrict__ xp,
                                                 const void* __restrict__ yp, void* __restrict__ y,
                                                 double* partials, unsigned* ticket, double* dot_out) {
  using T = VT<DT>;
  using R = typename T::R;
  using E = typename T::E;
  extern __shared__ __align__(16) unsigned char smraw[];
  // the NR rows interleaved: element (r, d) at d * NR + r, so one vector
  // load fetches a column of all NR rows
  using Pack = RowPack<E, NR>;
  E* xs = reinterpret_cast<E*>(smraw);
  const Pack* xsp = reinterpret_cast<const Pack*>(smraw);
  __shared__ double s_red[2 * (kDT / 32)];
  const PairPlan& p = *pp;
  const uint32_t Dd = p.Dd;
  double dr = 0.0, di = 0.0;
  const bool packed = p.dn_ent != nullptr;
  const R mag = R(p.dn_mag);
  auto split = [](const E& v, R& re, R& im) {
    if constexpr (T::cplx) { re = v.x; im = v.y; } else { re = v; im = R(0); }
  };
  for (uint32_t iu0 = blockIdx.x * NR; iu0 < p.Du; iu0 += gridDim.x * NR) {
    const uint32_t nr = min(uint32_t(NR), p.Du - iu0);
    __syncthreads();  // the previous rows are finished with the staging
    for (uint32_t i = threadIdx.x; i < nr * Dd; i += kDT) {
      const uint32_t r = i / Dd, c = i - r * Dd;
      xs[c * NR + r] = reinterpret_cast<const E*>(xp)[uint64_t(iu0) * Dd + i];
    }
    __syncthreads();
    for (uint32_t c = threadIdx.x; c < Dd; c += kDT) {
      const uint32_t k0 = __ldg(p.dn_ptr + c), k1 = __ldg(p.dn_ptr + c + 1);
      R sr[NR], si[NR];
      #pragma unroll
      for (int r = 0; r < NR; ++r) { sr[r] = R(0); si[r] = R(0); }
      if (packed) {
        // four hops at a time: their table words, then their row values
        auto hop = [&](uint32_t e) {
          const Pack pk = xsp[e & 0x7FFFu];
          #pragma unroll
          for (int r = 0; r < NR; ++r) {
            R vr, vi;
            split(pk.v[r], vr, vi);
            if (e & 0x8000u) { sr[r] -= vr; if (T::cplx) si[r] -= vi; }
            else { sr[r] += vr; if (T::cplx) si[r] += vi; }
          }
        };
        uint32_t k = k0;
        for (; k + 4 <= k1; k += 4) {
          uint32_t e[4];
          #pragma unroll
          for (int j = 0; j < 4; ++j) e[j] = __ldg(p.dn_ent + k + j);
          #pragma unroll
          for (int j = 0; j < 4; ++j) hop(e[j]);
        }
        for (; k < k1; ++k) hop(__ldg(p.dn_ent + k));
        #pragma unroll
        for (int r = 0; r < NR; ++r) { sr[r] *= mag; si[r] *= mag; }
      } else {
        for (uint32_t k = k0; k < k1; ++k) {
          const Pack pk = xsp[__ldg(p.dn_col + k)];
          const R w = R(__ldg(p.dn_val + k));
          #pragma unroll
          for (int r = 0; r < NR; ++r) {
            R vr, vi;
            split(pk.v[r], vr, vi);
            sr[r] += w * vr;
            if (T::cplx) si[r] += w * vi;
          }
        }
      }
      const uint32_t d = __ldg(p.dlist + c);
      #pragma unroll
      for (int r = 0; r < NR; ++r) {
        if (uint32_t(r) >= nr) break;
        const uint64_t i = uint64_t(iu0 + r) * Dd + c;
        R ar, ai, xr, xi;
        T::ld(yp, i, ar, ai);
        split(xs[c * NR + r], xr, xi);
        const R dg = R(__ldg(p.diag + i));
        ar += dg * xr + sr[r];
        if (T::cplx) ai += dg * xi + si[r];
        const uint32_t u = __ldg(p.ulist + iu0 + r);
        const R sg = R(pair_sign(u, d));
        T::st(y, p.perm ? __ldg(p.perm + i) : pair_rank(p, u, d), sg * ar, sg * ai);
        if (DOT) {  // <x, y> = <x_p, y_p> (S^2 = 1)
          dr += double(xr) * double(ar) + double(xi) * double(ai);
          di += double(xr) * double(ai) - double(xi) * double(ar);
        }
      }
    }
  }
  if (DOT) {
    block_sum2(dr, di, s_red);
    if (threadIdx.x == 0) { partials[2 * blockIdx.x] = dr; partials[2 * blockIdx.x + 1] = di; }
    grid_finish(partials, ticket, 1, dot_out);
  }
}

}  // namespace

struct PairHandle {
  PairPlan host{};
  PairPlan* dev = nullptr;
  std::vector<void*> bufs;
  mutable std::mutex mu;
  mutable void* scr = nullptr;  // x_p and y_p, sized on first use
  mutable size_t scr_bytes = 0;
};

void pair_plan_destroy(PairHandle* h) {
  if (!h) return;
  for (void* b : h->bufs) cudaFree(b);
  cudaFree(h->scr);
  cudaFree(h->dev);
  delete h;
}

namespace {
uint32_t compress(uint64_t s, int shift, int nsites) {  // the bits of one species
  uint32_t v = 0;
  for (int i = 0; i < nsites; ++i) v |= uint32_t((s >> (2 * i + shift)) & 1u) << i;
  return v;
}
uint64_t interleave(uint32_t u, uint32_t d, int nsites) {
  uint64_t s = 0;
  for (int i = 0; i < nsites; ++i) s |= (uint64_t((u >> i) & 1u) << (2 * i)) | (uint64_t((d >> i) & 1u) << (2 * i + 1));
  return s;
}
int host_pair_sign(uint32_t u, uint32_t d, int nsites) {
  int c = 0;
  for (int i = 0; i < nsites; ++i)
    if ((d >> i) & 1u) c += __builtin_popcount(u >> (i + 1));
  return (c & 1) ? -1 : 1;
}
}  // namespace

// Host side: eligibility, T_up / T_dn from the compiled terms (the matrix
// element of row s is the term's coefficient with its parity sign, target
// s ^ flip; products with S on both sides), a check that they do not depend
// on the other species' configuration, and the device tables.  Returns
// nullptr when the operator does not have the structure.  A, B: the plan's
// device copies of the sector tables.  diag_ref: the operator's diagonal
// (device, reference order, dim doubles).
PairHandle* pair_plan_create(const qk_plan_desc* d, const uint64_t* A_dev, const uint32_t* B_dev,
                             const double* diag_ref, size_t* dev_bytes) {
  if (!d->pair_sites || !d->all_real || d->nbits > 32 || (d->nbits & 1) || d->dim == 0 || d->dim >= (1ull << 32))
    return nullptr;
  const int ns = d->nbits / 2;
  if (ns > 16 || d->L <= 0 || d->L > 16) return nullptr;
  // the first state fixes N_up and N_dn; the sector must hold every
  // combination of those (its size is the product)
  uint64_t s0 = ~0ull;
  for (uint64_t h = 0; h < d->nA && s0 == ~0ull; ++h) {
    const uint32_t need = uint32_t(d->A[h] >> 56);
    if (need == qkb::kEmptyBlockKey) continue;
    if (d->key_off[need + 1] == d->key_off[need]) continue;
    s0 = (h << d->L) | d->llist[d->key_off[need]];
  }
  if (s0 == ~0ull) return nullptr;
  const int nu = __builtin_popcount(compress(s0, 0, ns)), nd = __builtin_popcount(compress(s0, 1, ns));
  std::vector<uint32_t> ul, dl;
  for (uint32_t v = 0; v < (1u << ns); ++v) {
    if (__builtin_popcount(v) == nu) ul.push_back(v);
    if (__builtin_popcount(v) == nd) dl.push_back(v);
  }
  if (uint64_t(ul.size()) * dl.size() != d->dim || dl.size() >= 32768) return nullptr;
  auto in_sector = [&](uint64_t s) {
    const uint64_t a = d->A[s >> d->L];
    const uint32_t b = d->B[s & ((1ull << d->L) - 1)];
    return uint32_t(a >> 56) == (b >> 24);
  };
  if (!in_sector(interleave(ul.back(), dl.back(), ns)) || !in_sector(interleave(ul[0], dl.back(), ns))) return nullptr;
  // off-diagonal groups: hops of one species (flip within the even or the odd bits)
  const uint64_t even = 0x5555555555555555ull & ((ns >= 32) ? ~0ull : ((1ull << (2 * ns)) - 1));
  std::vector<uint32_t> gup, gdn;
  for (uint32_t gi = d->has_diag ? 1u : 0u; gi < d->ngroups; ++gi) {
    const qk_group_t& g = d->groups[gi];
    if (g.flip == 0) return nullptr;
    if ((g.flip & ~even) == 0) gup.push_back(gi);
    else if ((g.flip & even) == 0) gdn.push_back(gi);
    else return nullptr;
    for (uint32_t q = g.first; q < g.first + g.count; ++q)
      if (d->terms[q].wim != 0.0) return nullptr;
  }
  std::vector<uint32_t> uidx(size_t(1) << ns, ~0u), didx(size_t(1) << ns, ~0u);
  for (uint32_t i = 0; i < ul.size(); ++i) uidx[ul[i]] = i;
  for (uint32_t i = 0; i < dl.size(); ++i) didx[dl[i]] = i;
  // row `a` of T_species at a fixed configuration `o` of the other species:
  // (column index, value) pairs in term order
  auto row = [&](bool up, uint32_t a, uint32_t o, std::vector<std::pair<uint32_t, double>>& out) -> bool {
    out.clear();
    const uint64_t s = up ? interleave(a, o, ns) : interleave(o, a, ns);
    const int ss = up ? host_pair_sign(a, o, ns) : host_pair_sign(o, a, ns);
    for (uint32_t gi : (up ? gup : gdn)) {
      const qk_group_t& g = d->groups[gi];
      const uint64_t t = s ^ g.flip;
      double c = 0.0;
      for (uint32_t q = g.first; q < g.first + g.count; ++q) {
        const qk_term_t& tm = d->terms[q];
        if ((s & tm.cmask) != tm.cval) continue;
        c += (__builtin_popcountll(s & tm.smask) & 1) ? -tm.wre : tm.wre;
      }
      if (c == 0.0) continue;
      const uint32_t a2 = up ? compress(t, 0, ns) : compress(t, 1, ns);
      const uint32_t o2 = up ? compress(t, 1, ns) : compress(t, 0, ns);
      if (o2 != o) return false;
      const uint32_t idx = up ? uidx[a2] : didx[a2];
      if (idx == ~0u) return false;
      const int ts = up ? host_pair_sign(a2, o, ns) : host_pair_sign(o, a2, ns);
      out.push_back({idx, double(ss * ts) * c});
    }
    return true;
  };
  std::vector<uint32_t> uptr(1, 0), ucol, dptr(1, 0), dcol;
  std::vector<double> uval, dval;
  std::vector<std::pair<uint32_t, double>> r, r2;
  const uint32_t o_chk[2][2] = {{dl[dl.size() / 2], dl.back()}, {ul[ul.size() / 2], ul.back()}};
  for (int sp = 0; sp < 2; ++sp) {
    const bool up = sp == 0;
    const std::vector<uint32_t>& own = up ? ul : dl;
    const uint32_t o0 = up ? dl[0] : ul[0];
    for (uint32_t a : own) {
      if (!row(up, a, o0, r)) return nullptr;
      for (int k = 0; k < 2; ++k) {  // the row must not depend on the other species
        if (!row(up, a, o_chk[sp][k], r2) || r2 != r) return nullptr;
      }
      for (auto& e : r) {
        (up ? ucol : dcol).push_back(e.first);
        (up ? uval : dval).push_back(e.second);
      }
      (up ? uptr : dptr).push_back(uint32_t((up ? ucol : dcol).size()));
    }
  }
  // down hops packed as column | sign when they share one magnitude
  double mag = dval.empty() ? 1.0 : std::abs(dval[0]);
  bool uniform = true;
  for (double v : dval) uniform = uniform && std::abs(v) == mag;
  std::vector<uint16_t> dent;
  if (uniform)
    for (size_t k = 0; k < dcol.size(); ++k) dent.push_back(uint16_t(dcol[k] | (dval[k] < 0 ? 0x8000u : 0u)));
  auto* out = new PairHandle;
  bool ok = true;
  auto up_ = [&](const void* src, size_t bytes) -> void* {
    void* p = nullptr;
    if (!ok) return nullptr;
    bytes = std::max<size_t>(bytes, 8);
    if (cudaMalloc(&p, bytes) != cudaSuccess) { ok = false; return nullptr; }
    out->bufs.push_back(p);
    *dev_bytes += bytes;
    if (src && cudaMemcpy(p, src, bytes, cudaMemcpyHostToDevice) != cudaSuccess) ok = false;
    return p;
  };
  PairPlan& h = out->host;
  h.Du = uint32_t(ul.size()); h.Dd = uint32_t(dl.size());
  h.L = d->L; h.lmask = uint32_t((1ull << d->L) - 1);
  h.A = A_dev; h.B = B_dev;
  h.ulist = static_cast<const uint32_t*>(up_(ul.data(), ul.size() * 4));
  h.dlist = static_cast<const uint32_t*>(up_(dl.data(), dl.size() * 4));
  h.up_ptr = static_cast<const uint32_t*>(up_(uptr.data(), uptr.size() * 4));
  h.up_col = static_cast<const uint32_t*>(up_(ucol.data(), ucol.size() * 4));
  h.up_val = static_cast<const double*>(up_(uval.data(), uval.size() * 8));
  h.dn_ptr = static_cast<const uint32_t*>(up_(dptr.data(), dptr.size() * 4));
  if (uniform) {
    h.dn_ent = static_cast<const uint16_t*>(up_(dent.data(), dent.size() * 2));
  } else {
    h.dn_col = static_cast<const uint32_t*>(up_(dcol.data(), dcol.size() * 4));
    h.dn_val = static_cast<const double*>(up_(dval.data(), dval.size() * 8));
  }
  h.dn_mag = mag;
  double* dp = static_cast<double*>(up_(nullptr, d->dim * 8));
  h.diag = dp;
  if (ok) {
    out->dev = nullptr;
    ok = cudaMalloc(reinterpret_cast<void**>(&out->dev), sizeof(PairPlan)) == cudaSuccess &&
         cudaMemcpy(out->dev, &h, sizeof(PairPlan), cudaMemcpyHostToDevice) == cudaSuccess;
    if (ok) *dev_bytes += sizeof(PairPlan);
  }
  if (ok) {  // the diagonal in product order (no sign: S D S = D)
    const unsigned g = resident_grid(k_pair_in<QK_F64, false>, kPT, 0, 4096);
    k_pair_in<QK_F64, false><<<g, kPT>>>(out->dev, diag_ref, dp);
    ok = cudaGetLastError() == cudaSuccess && cudaDeviceSynchronize() == cudaSuccess;
  }
  if (ok) {
    // the reference rank of every product index, read coalesced by the
    // gather and the scatter instead of two scattered table lookups per
    // element (4 bytes per state; without the memory the kernels compute it)
    uint32_t* pm = nullptr;
    if (cudaMalloc(&pm, d->dim * 4) == cudaSuccess) {
      out->bufs.push_back(pm);
      *dev_bytes += d->dim * 4;
      k_pair_perm<<<resident_grid(k_pair_perm, kPT, 0, 4096), kPT>>>(out->dev, pm);
      ok = cudaGetLastError() == cudaSuccess && cudaDeviceSynchronize() == cudaSuccess;
      h.perm = pm;
      ok = ok && cudaMemcpy(out->dev, &h, sizeof(PairPlan), cudaMemcpyHostToDevice) == cudaSuccess;
    } else {
      (void)cudaGetLastError();
    }
  }
  if (!ok) {
    (void)cudaGetLastError();
    pair_plan_destroy(out);
    return nullptr;
  }
  return out;
}

// y = H x (and <x, y> into dot_out when given) through the product order.
// QKD_EINVAL when the scratch is missing and cannot be allocated now (during
// a stream capture): the caller then takes the row kernel.
int pair_apply(const PairHandle* h, qk_dtype t, const void* x, void* y, cudaStream_t s, qk_workspace* w,
               double* dot_out) {
  if (!h || !x || !y || x == y) return QKD_EINVAL;
  const size_t es = qk_dtype_size(t), n = size_t(h->host.Du) * h->host.Dd;
  void* scr = nullptr;
  {
    std::lock_guard<std::mutex> lk(h->mu);
    if (h->scr_bytes < 2 * n * es) {
      cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
      if (cudaStreamIsCapturing(s, &st) != cudaSuccess || st != cudaStreamCaptureStatusNone) return QKD_EINVAL;
      cudaFree(h->scr);
      h->scr = nullptr;
      h->scr_bytes = 0;
      if (cudaMalloc(&h->scr, 2 * n * es) != cudaSuccess) {
        (void)cudaGetLastError();
        return QKD_EINVAL;
      }
      h->scr_bytes = 2 * n * es;
    }
    scr = h->scr;
  }
  void* xp = scr;
  void* yp = static_cast<char*>(scr) + n * es;
  // rows staged per pass of the down-hop kernel: as many as 220 KB hold (1, 2
  // or 4; a CTA may use up to 227 KB of shared memory)
  constexpr size_t kStage = 220 * 1024;
  const size_t row_bytes = es * h->host.Dd;
  if (row_bytes > kStage) return QKD_EINVAL;
  const int nr = row_bytes * 4 <= kStage ? 4 : row_bytes * 2 <= kStage ? 2 : 1;
  const size_t smem = row_bytes * nr;
#define QKD_PAIR_DN(DT, DOT, NR)                                                                           \
  {                                                                                                        \
    auto k = k_pair_dn<DT, DOT, NR>;                                                                       \
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)     \
      return QKD_EINVAL;                                                                                   \
    const unsigned rows = (h->host.Du + NR - 1) / NR;                                                      \
    const unsigned g = resident_grid(k, kDT, smem, DOT ? std::min<unsigned>(rows, kMaxG) : rows);          \
    k<<<g, kDT, smem, s>>>(h->dev, xp, yp, y, DOT ? w->partials : nullptr, DOT ? w->ticket : nullptr, dot_out); \
  }
#define QKD_PAIR(DT)                                                                                       \
  {                                                                                                        \
    k_pair_in<DT, true><<<resident_grid(k_pair_in<DT, true>, kPT, 0, 1u << 20), kPT, 0, s>>>(h->dev, x, xp); \
    k_pair_up<DT><<<resident_grid(k_pair_up<DT>, kPT, 0, 1u << 20), kPT, 0, s>>>(h->dev, xp, yp);       \
    if (dot_out) {                                                                                         \
      if (nr == 4) QKD_PAIR_DN(DT, true, 4) else if (nr == 2) QKD_PAIR_DN(DT, true, 2) else QKD_PAIR_DN(DT, true, 1) \
    } else {                                                                                               \
      if (nr == 4) QKD_PAIR_DN(DT, false, 4) else if (nr == 2) QKD_PAIR_DN(DT, false, 2) else QKD_PAIR_DN(DT, false, 1) \
    }                                                                                                      \
  }
  switch (t) {
    case QK_C128: QKD_PAIR(QK_C128); break;
    case QK_C64: QKD_PAIR(QK_C64); break;
    case QK_F64: QKD_PAIR(QK_F64); break;
    case QK_F32: QKD_PAIR(QK_F32); break;
    default: return QKD_EINVAL;
  }
#undef QKD_PAIR
#undef QKD_PAIR_DN
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}

}  // namespace qkd
