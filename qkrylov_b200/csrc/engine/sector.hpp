// Sector tables: the ordered list of basis states of one U(1) sector, held as
// two-level ranking tables instead of an explicit state list.
//
// Order.  qkrylov's bases list every valid state in ascending integer order
// (src/basis/spinhalf_basis.cpp:86-104, fermion_basis.cpp:72-89,
// hubbard_basis.cpp:72-100, tj_basis.cpp:56-96).  A state s of `nbits` bits
// is split into a high part h = s >> L and a low part l = s & (2^L - 1).  In
// ascending order all states sharing h are contiguous, and inside that block
// the low parts appear in ascending order.  So
//
//     index(s) = A[h] + B[l]
//
// where A[h] is the number of sector states with a smaller high part and B[l]
// is the rank of l among the valid low parts carrying the same conserved
// charges ("key").  Membership is a key check: a block h needs low parts of
// key need(h), which is packed into the top byte of A[h]; the key of l is
// packed into the top byte of B[l].  One lookup into each table ranks a state
// and tests membership, with no hashing and no 2^N enumeration.
//
// For pair families (Hubbard, t-J: up at bit 2i, down at bit 2i+1,
// hubbard_site.cpp:11-29) L is even so no site straddles the split, and the
// t-J no-double-occupancy rule is a per-part validity test.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace qkb {

enum class Family : int { Spin = 0, Fermion = 1, Hubbard = 2, TJ = 3 };

inline bool is_pair(Family f) { return f == Family::Hubbard || f == Family::TJ; }
inline int popc64(uint64_t x) { return __builtin_popcountll(x); }

// Field-for-field copy of qkrylov's Sector (include/qkrylov/symmetry/sector.hpp:10-41).
struct SectorSpec {
  bool use_sz = false; int sz2 = 0;
  bool use_nup = false; bool use_ndn = false; int nup = 0; int ndn = 0;
  bool use_n = false; int n = 0;
  bool use_nb = false; int nb = 0;
};

constexpr uint64_t kOffsetMask = (1ULL << 56) - 1;
constexpr uint32_t kRankMask = (1u << 24) - 1;
constexpr uint32_t kEmptyBlockKey = 0xFF;  // need(h) of a block with no states
constexpr uint32_t kInvalidLowKey = 0xFE;  // key of a low part that is never valid
constexpr int kMaxBits = 48;               // two-level tables up to 2^24 entries each

class SectorTable {
 public:
  SectorTable(Family family, int nsites, const SectorSpec& spec);

  Family family;
  int nsites;
  int nbits;      // N (spin, fermion) or 2N (Hubbard, t-J)
  int L, H;       // low / high split, L + H = nbits
  bool con_u = false, con_d = false;  // which charges are conserved
  int tu = 0, td = 0;                 // their required totals
  int KD = 1;                         // key = nu * KD + nd over conserved charges
  uint64_t dim = 0;

  std::vector<uint64_t> A;       // 2^H entries: (need(h) << 56) | offset
  std::vector<uint32_t> B;       // 2^L entries: (key(l) << 24) | rank
  std::vector<uint32_t> key_off; // per key: start of its low parts in llist
  std::vector<uint32_t> llist;   // valid low parts grouped by key, ascending

  uint64_t state(uint64_t i) const;      // throws std::out_of_range past dim
  int64_t index(uint64_t s) const;       // -1 when s is not in the sector
  bool contains(uint64_t s) const { return index(s) >= 0; }
  uint32_t part_key(uint64_t part, int width_bits) const;  // kInvalidLowKey if invalid

  uint64_t lmask() const { return (L == 64) ? ~0ULL : ((1ULL << L) - 1); }
  uint64_t block_offset(uint64_t h) const { return A[h] & kOffsetMask; }
  uint32_t block_need(uint64_t h) const { return uint32_t(A[h] >> 56); }
  uint64_t block_size(uint64_t h) const;
  // nshards + 1 row bounds at sector-block boundaries (0 and dim at the
  // ends), each as close as a block boundary gets to k * dim / nshards:
  // contiguous row ranges for a row-sharded H.x.
  std::vector<uint64_t> shard_bounds(int nshards) const;
  // true when row r starts a sector block (or is dim)
  bool is_block_start(uint64_t r) const;
};

}  // namespace qkb
