// OpSum compiler: turns each term's factor chain into bit masks.
//
// The reference evaluates a term on a ket |s> by applying its factors in list
// order (factors[0] first), each through Site::apply on the intermediate
// state, multiplying the matrix elements into amp = coeff * prod(me), and
// stores conj(amp) at (row = s, column = final state)
// (src/hamiltonian/matrix_free_hamiltonian.cpp:45-91).
//
// Every single-site operator of the four sites (spinhalf_site.cpp:18-121,
// fermion_site.cpp:59-111, hubbard_site.cpp:48-125, tj_site.cpp:47-113) is
// one of: a required bit value, an unconditional bit flip, a Jordan-Wigner
// parity over the bits below the target, or a constant from {0.5, i/2, 1}
// with a sign that depends on one bit.  Because the intermediate state is
// always s XOR (flips so far), the whole chain reduces to
//
//   valid(s)   <=>  (s & cmask) == cval
//   target     =    s ^ flip
//   conj(amp)  =    w * (-1)^popcount(s & smask)
//
// with w = conj(coeff * K) for an exact constant K (products of +-1, +-1/2,
// +-i/2 are exact in binary floating point).  Operators whose element is 0
// on an empty site (N, Nup, Ndn, Nupdn) become conditions: the reference
// keeps those zero-valued entries, which add 0 * x[col] to the row.
//
// Terms are grouped by flip mask so that one target rank and one gather of
// x serve every term with the same target.
#pragma once

#include <complex>
#include <cstdint>
#include <string>
#include <vector>

#include "sector.hpp"

namespace qkb {

struct FactorIn { std::string op; int site; };
struct TermIn { std::complex<double> coeff; std::vector<FactorIn> factors; };

struct CTerm {
  uint64_t cmask, cval, smask;
  double wre, wim;
};
struct CGroup {
  uint64_t flip;
  uint32_t first, count;  // terms [first, first + count)
  uint32_t check;         // 1: the target may fall outside the sector
  uint32_t pad;
};

struct CompiledOp {
  std::vector<CTerm> terms;
  std::vector<CGroup> groups;  // the diagonal group (flip 0), if any, comes first
  bool has_diag = false;
  bool all_real = true;
  size_t n_input_terms = 0;
  size_t n_dropped = 0;  // terms that can never contribute
};

// Compile `terms` for operators of `site_family` acting on `basis`.
// Throws std::runtime_error for unknown operator names (message as the
// reference's sites) and std::invalid_argument for site indices that do not
// map to a bit of a 64-bit state.
CompiledOp compile_opsum(Family site_family, const SectorTable& basis,
                         const std::vector<TermIn>& terms);

// Single operator on one state: the Site::apply contract.
struct FactorAction { bool valid; uint64_t new_state; std::complex<double> me; };
FactorAction apply_factor(Family site_family, const std::string& op, int site, uint64_t state);

}  // namespace qkb
