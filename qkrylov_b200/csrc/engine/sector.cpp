#include "sector.hpp"

#include <algorithm>

namespace qkb {

namespace {
uint64_t even_bits(int nbits) {  // up-spin positions 0, 2, 4, ...
  uint64_t m = 0;
  for (int b = 0; b < nbits; b += 2) m |= 1ULL << b;
  return m;
}
}  // namespace

uint32_t SectorTable::part_key(uint64_t p, int width) const {
  int nu, nd;
  if (is_pair(family)) {
    const uint64_t um = even_bits(width), dm = um << 1;
    if (family == Family::TJ && ((p & um) & ((p & dm) >> 1))) return kInvalidLowKey;
    nu = popc64(p & um);
    nd = popc64(p & dm);
  } else {
    nu = popc64(p);
    nd = 0;
  }
  return uint32_t((con_u ? nu : 0) * KD + (con_d ? nd : 0));
}

SectorTable::SectorTable(Family fam, int ns, const SectorSpec& spec) : family(fam), nsites(ns) {
  // Site-count limits and messages of the reference constructors
  // (spinhalf_basis.cpp:17-23, fermion_basis.cpp:17-23,
  //  hubbard_basis.cpp:17-23, tj_basis.cpp:17-23).
  if (!is_pair(fam) && (ns <= 0 || ns > 63))
    throw std::runtime_error(fam == Family::Spin ? "SpinHalfBasis: N must satisfy 1 <= N <= 63"
                                                 : "FermionBasis: N must satisfy 1 <= N <= 63");
  if (is_pair(fam) && (ns <= 0 || ns > 31))
    throw std::runtime_error(fam == Family::Hubbard ? "HubbardBasis: N must satisfy 1 <= N <= 31"
                                                    : "TJBasis: N must satisfy 1 <= N <= 31");
  nbits = is_pair(fam) ? 2 * ns : ns;
  if (nbits > kMaxBits)
    throw std::runtime_error("qkrylov_b200: bases wider than " + std::to_string(kMaxBits) +
                             " bits are not supported");

  // Conserved charges and their targets, exactly the membership tests of the
  // reference builders.
  bool empty = false;
  switch (fam) {
    case Family::Spin:
      if (spec.use_sz) {  // nup - (N - nup) == sz2  (spinhalf_basis.cpp:60-72)
        con_u = true;
        if ((spec.sz2 + ns) % 2 != 0) empty = true;
        tu = (spec.sz2 + ns) / 2;
        if (tu < 0 || tu > ns) empty = true;
      }
      break;
    case Family::Fermion:
      if (spec.use_n) { con_u = true; tu = spec.n; if (tu < 0 || tu > ns) empty = true; }
      break;
    case Family::Hubbard:
    case Family::TJ:
      if (spec.use_nup) { con_u = true; tu = spec.nup; if (tu < 0 || tu > ns) empty = true; }
      if (spec.use_ndn) { con_d = true; td = spec.ndn; if (td < 0 || td > ns) empty = true; }
      break;
  }
  L = nbits / 2;
  if (is_pair(fam)) L &= ~1;
  H = nbits - L;
  // A part of H (>= L) bits holds at most `part` particles of each species.
  const int part = is_pair(fam) ? H / 2 : H;
  KD = con_d ? (part + 1) : 1;
  const uint64_t nlow = 1ULL << L, nhigh = 1ULL << H;
  const int nkeys = (con_u ? part + 1 : 1) * KD;
  if (nkeys >= int(kInvalidLowKey)) throw std::runtime_error("qkrylov_b200: too many sector keys");

  // Low parts: key, rank within key, grouped list.
  B.assign(nlow, 0);
  std::vector<uint32_t> cnt(nkeys, 0);
  for (uint64_t l = 0; l < nlow; ++l) {
    const uint32_t k = part_key(l, L);
    if (k == kInvalidLowKey) { B[l] = kInvalidLowKey << 24; continue; }
    B[l] = (k << 24) | cnt[k]++;
  }
  key_off.assign(nkeys + 1, 0);
  for (int k = 0; k < nkeys; ++k) key_off[k + 1] = key_off[k] + cnt[k];
  llist.assign(key_off[nkeys], 0);
  for (uint64_t l = 0; l < nlow; ++l) {
    const uint32_t k = B[l] >> 24;
    if (k == kInvalidLowKey) continue;
    llist[key_off[k] + (B[l] & kRankMask)] = uint32_t(l);
  }

  // High parts: required low key and running offset.
  A.assign(nhigh, 0);
  uint64_t off = 0;
  for (uint64_t h = 0; h < nhigh; ++h) {
    uint32_t need = kEmptyBlockKey;
    uint64_t size = 0;
    const uint32_t kh = empty ? kInvalidLowKey : part_key(h, H);
    if (kh != kInvalidLowKey) {
      const int nu_h = con_u ? int(kh) / KD : 0, nd_h = con_d ? int(kh) % KD : 0;
      const int ru = tu - nu_h, rd = td - nd_h;
      if (ru >= 0 && rd >= 0 && (!con_u || ru <= part) && (!con_d || rd < KD)) {
        need = uint32_t((con_u ? ru : 0) * KD + (con_d ? rd : 0));
        if (need < uint32_t(nkeys)) size = cnt[need]; else need = kEmptyBlockKey;
        if (size == 0) need = kEmptyBlockKey;
      }
    }
    A[h] = (uint64_t(need) << 56) | off;
    off += size;
  }
  dim = off;
}

uint64_t SectorTable::block_size(uint64_t h) const {
  const uint32_t need = block_need(h);
  if (need == kEmptyBlockKey) return 0;
  return key_off[need + 1] - key_off[need];
}

int64_t SectorTable::index(uint64_t s) const {
  if (nbits < 64 && (s >> nbits) != 0) return -1;
  const uint64_t h = s >> L, l = s & lmask();
  const uint64_t a = A[h];
  const uint32_t b = B[l];
  if (uint32_t(a >> 56) != (b >> 24)) return -1;
  return int64_t((a & kOffsetMask) + (b & kRankMask));
}

uint64_t SectorTable::state(uint64_t i) const {
  if (i >= dim) throw std::out_of_range("qkrylov_b200: basis index out of range");
  // Last block whose offset is <= i (offsets are non-decreasing in h).
  uint64_t lo = 0, hi = A.size() - 1;
  while (lo < hi) {
    const uint64_t mid = (lo + hi + 1) / 2;
    if ((A[mid] & kOffsetMask) <= i) lo = mid; else hi = mid - 1;
  }
  // The last block starting at or before i is the non-empty block holding i
  // (empty blocks share the offset of the next block and sort before it).
  const uint64_t h = lo;
  if (block_need(h) == kEmptyBlockKey || (A[h] & kOffsetMask) + block_size(h) <= i)
    throw std::logic_error("qkrylov_b200: inconsistent sector table");
  const uint64_t r = i - (A[h] & kOffsetMask);
  return (h << L) | llist[key_off[block_need(h)] + r];
}

std::vector<uint64_t> SectorTable::shard_bounds(int nshards) const {
  if (nshards < 1) throw std::invalid_argument("qkrylov_b200: shard count must be at least 1");
  std::vector<uint64_t> starts;  // block starts in ascending row order
  for (uint64_t h = 0; h < A.size(); ++h)
    if (block_need(h) != kEmptyBlockKey && block_size(h) > 0) starts.push_back(block_offset(h));
  starts.push_back(dim);
  std::vector<uint64_t> b(size_t(nshards) + 1, 0);
  b[nshards] = dim;
  size_t j = 0;
  for (int k = 1; k < nshards; ++k) {
    const double want = double(dim) * k / nshards;
    while (j + 1 < starts.size() && double(starts[j + 1]) <= want) ++j;
    uint64_t pick = starts[j];
    if (j + 1 < starts.size() && double(starts[j + 1]) - want < want - double(starts[j])) pick = starts[j + 1];
    b[k] = std::max(pick, b[k - 1]);
  }
  return b;
}

bool SectorTable::is_block_start(uint64_t r) const {
  if (r == dim || r == 0) return true;
  // block offsets ascend with h: binary search over the high parts
  uint64_t lo = 0, hi = A.size();
  while (lo < hi) {
    const uint64_t mid = (lo + hi) / 2;
    if (block_offset(mid) < r) lo = mid + 1;
    else hi = mid;
  }
  for (uint64_t h = lo; h < A.size() && block_offset(h) == r; ++h)
    if (block_need(h) != kEmptyBlockKey && block_size(h) > 0) return true;
  return false;
}

}  // namespace qkb
