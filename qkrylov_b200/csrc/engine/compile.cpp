#include "compile.hpp"

#include <map>
#include <stdexcept>

namespace qkb {

namespace {

using cd = std::complex<double>;

enum class Op {
  Sz, Sp, Sm, Sx, Sy,                       // spin-1/2
  N, Id, C, Cdag,                           // spinless fermion
  Nup, Ndn, Nupdn, CUp, CdagUp, CDn, CdagDn  // Hubbard, t-J
};

const char* family_word(Family f) {
  switch (f) {
    case Family::Spin: return "spin";
    case Family::Fermion: return "fermion";
    case Family::Hubbard: return "Hubbard";
    case Family::TJ: return "TJ";
  }
  return "?";
}

// Operator names each site accepts; anything else is the reference's
// "Unknown <family> operator: <name>" runtime_error.
Op parse(Family f, const std::string& s) {
  switch (f) {
    case Family::Spin:
      if (s == "Sz") return Op::Sz;
      if (s == "Sp") return Op::Sp;
      if (s == "Sm") return Op::Sm;
      if (s == "Sx") return Op::Sx;
      if (s == "Sy") return Op::Sy;
      break;
    case Family::Fermion:
      if (s == "N") return Op::N;
      if (s == "Id") return Op::Id;
      if (s == "C") return Op::C;
      if (s == "Cdag") return Op::Cdag;
      break;
    case Family::Hubbard:
    case Family::TJ:
      if (s == "Nup") return Op::Nup;
      if (s == "Ndn") return Op::Ndn;
      if (s == "Nupdn" && f == Family::Hubbard) return Op::Nupdn;
      if (s == "CUp") return Op::CUp;
      if (s == "CdagUp") return Op::CdagUp;
      if (s == "CDn") return Op::CDn;
      if (s == "CdagDn") return Op::CdagDn;
      break;
  }
  throw std::runtime_error(std::string("Unknown ") + family_word(f) + " operator: " + s);
}

int bit_of(Family f, Op op, int site) {
  if (site < 0) throw std::invalid_argument("qkrylov_b200: negative site index");
  const bool pair = is_pair(f);
  const bool dn = (op == Op::Ndn || op == Op::CDn || op == Op::CdagDn);
  const long b = pair ? 2L * site + (dn ? 1 : 0) : site;
  if (b > 63 || (pair && 2L * site + 1 > 63))
    throw std::invalid_argument("qkrylov_b200: site index " + std::to_string(site) +
                                " does not fit a 64-bit state");
  return int(b);
}

// Symbolic evaluation of a factor chain on an unknown ket s.
struct Chain {
  uint64_t F = 0, cmask = 0, cval = 0, smask = 0;
  cd K = 1.0;
  bool dead = false;

  void require(int b, unsigned v_inter) {  // intermediate bit b must equal v_inter
    const uint64_t bit = 1ULL << b;
    const uint64_t orig = (v_inter ^ ((F >> b) & 1ULL)) & 1ULL;
    if (cmask & bit) {
      if (((cval >> b) & 1ULL) != orig) dead = true;
      return;
    }
    cmask |= bit;
    cval |= orig << b;
  }
  void parity_below(int b) {  // (-1)^popcount(intermediate & (2^b - 1))
    const uint64_t m = (b >= 64) ? ~0ULL : ((1ULL << b) - 1);
    smask ^= m;
    if (popc64(F & m) & 1) K = -K;
  }
  void sign_of_bit(int b) {  // (-1)^(intermediate bit b)
    smask ^= 1ULL << b;
    if ((F >> b) & 1ULL) K = -K;
  }
  void flip(int b) { F ^= 1ULL << b; }
};

void step(Chain& c, Family f, Op op, int site) {
  const bool tj = (f == Family::TJ);
  switch (op) {
    case Op::Sz: { const int b = bit_of(f, op, site); c.sign_of_bit(b); c.K *= -0.5; break; }
    case Op::Sp: { const int b = bit_of(f, op, site); c.require(b, 0); c.flip(b); break; }
    case Op::Sm: { const int b = bit_of(f, op, site); c.require(b, 1); c.flip(b); break; }
    case Op::Sx: { const int b = bit_of(f, op, site); c.K *= 0.5; c.flip(b); break; }
    case Op::Sy: { const int b = bit_of(f, op, site); c.sign_of_bit(b); c.K *= cd(0.0, 0.5); c.flip(b); break; }
    case Op::N: { const int b = bit_of(f, op, site); c.require(b, 1); break; }
    case Op::Id: { (void)bit_of(f, op, site); break; }
    case Op::C: { const int b = bit_of(f, op, site); c.require(b, 1); c.parity_below(b); c.flip(b); break; }
    case Op::Cdag: { const int b = bit_of(f, op, site); c.require(b, 0); c.parity_below(b); c.flip(b); break; }
    case Op::Nup: c.require(bit_of(f, op, site), 1); break;
    case Op::Ndn: c.require(bit_of(f, op, site), 1); break;
    case Op::Nupdn: { const int b = bit_of(f, op, site); c.require(b, 1); c.require(b + 1, 1); break; }
    case Op::CUp: { const int b = bit_of(f, op, site); c.require(b, 1); c.parity_below(b); c.flip(b); break; }
    case Op::CdagUp: {
      const int b = bit_of(f, op, site);
      c.require(b, 0);
      if (tj) c.require(b + 1, 0);
      c.parity_below(b); c.flip(b); break;
    }
    case Op::CDn: { const int b = bit_of(f, op, site); c.require(b, 1); c.parity_below(b); c.flip(b); break; }
    case Op::CdagDn: {
      const int b = bit_of(f, op, site);
      c.require(b, 0);
      if (tj) c.require(b - 1, 0);
      c.parity_below(b); c.flip(b); break;
    }
  }
}

// Is the target of a surviving term always / never / maybe in the sector?
enum class Member { Always, Never, Maybe };

Member target_membership(const Chain& c, const SectorTable& B) {
  const bool pair = is_pair(B.family);
  int du = 0, dd = 0;
  bool unknown_u = false, unknown_d = false;
  for (int b = 0; b < 64; ++b) {
    if (!((c.F >> b) & 1ULL)) continue;
    const bool is_dn = pair && (b & 1);
    if (c.cmask & (1ULL << b)) {
      const int delta = ((c.cval >> b) & 1ULL) ? -1 : +1;
      (is_dn ? dd : du) += delta;
    } else {
      (is_dn ? unknown_d : unknown_u) = true;
    }
  }
  if (B.con_u && !unknown_u && du != 0) return Member::Never;
  if (B.con_d && !unknown_d && dd != 0) return Member::Never;
  bool maybe = (B.con_u && unknown_u) || (B.con_d && unknown_d);
  if (B.family == Family::TJ) {
    // A site may end doubly occupied unless its other bit is known empty.
    for (int b = 0; b < 64; ++b) {
      if (!((c.F >> b) & 1ULL)) continue;
      const int p = b ^ 1;
      const uint64_t bb = 1ULL << b, pb = 1ULL << p;
      const bool b_known = c.cmask & bb;
      const bool b_final_one = b_known && !((c.cval >> b) & 1ULL);  // flipped from 0
      const bool p_known = c.cmask & pb;
      const bool p_final_one = p_known && (((c.cval >> p) ^ (c.F >> p)) & 1ULL);
      const bool p_final_zero = p_known && !p_final_one;
      if (b_final_one && p_final_one) return Member::Never;
      if (!(b_known && !b_final_one) && !p_final_zero) maybe = true;
    }
  }
  return maybe ? Member::Maybe : Member::Always;
}

}  // namespace

CompiledOp compile_opsum(Family site_family, const SectorTable& basis,
                         const std::vector<TermIn>& terms) {
  CompiledOp out;
  out.n_input_terms = terms.size();
  const uint64_t inside = (basis.nbits >= 64) ? ~0ULL : ((1ULL << basis.nbits) - 1);

  struct Pending { uint64_t flip; CTerm t; uint32_t check; };
  std::vector<Pending> pend;
  for (const auto& term : terms) {
    Chain c;
    for (const auto& f : term.factors) {
      const Op op = parse(site_family, f.op);  // always validated, like a first evaluation
      if (!c.dead) step(c, site_family, op, f.site);
      else (void)bit_of(site_family, op, f.site);
    }
    if (c.dead || term.coeff == cd(0.0, 0.0)) { ++out.n_dropped; continue; }
    // Bits above the basis are 0 in every basis state.
    if (c.F & ~inside) { ++out.n_dropped; continue; }
    if (c.cval & ~inside) { ++out.n_dropped; continue; }
    c.cmask &= inside;
    c.smask &= inside;
    const Member m = target_membership(c, basis);
    if (m == Member::Never) { ++out.n_dropped; continue; }
    const cd w = std::conj(term.coeff * c.K);
    pend.push_back({c.F, CTerm{c.cmask, c.cval, c.smask, w.real(), w.imag()},
                    m == Member::Maybe ? 1u : 0u});
  }

  // Group by flip mask: diagonal first, then first-appearance order.
  std::vector<uint64_t> order;
  std::map<uint64_t, std::vector<size_t>> by_flip;
  for (size_t i = 0; i < pend.size(); ++i) {
    auto it = by_flip.find(pend[i].flip);
    if (it == by_flip.end()) { order.push_back(pend[i].flip); by_flip[pend[i].flip] = {i}; }
    else it->second.push_back(i);
  }
  auto emit = [&](uint64_t flip) {
    CGroup g{flip, uint32_t(out.terms.size()), 0, 0, 0};
    for (size_t i : by_flip[flip]) {
      out.terms.push_back(pend[i].t);
      g.check |= pend[i].check;
      if (pend[i].t.wim != 0.0) out.all_real = false;
    }
    g.count = uint32_t(out.terms.size()) - g.first;
    out.groups.push_back(g);
  };
  if (by_flip.count(0)) { out.has_diag = true; emit(0); }
  for (uint64_t f : order) if (f != 0) emit(f);
  return out;
}

FactorAction apply_factor(Family f, const std::string& name, int site, uint64_t st) {
  const Op op = parse(f, name);
  Chain c;
  step(c, f, op, site);
  FactorAction a{false, 0, cd(0.0, 0.0)};  // LocalAction's defaults (local_action.hpp:9-16)
  if (c.dead || (st & c.cmask) != c.cval) {
    // The density operators are valid with element 0 on an empty site.
    if (op == Op::N || op == Op::Nup || op == Op::Ndn || op == Op::Nupdn) { a.valid = true; a.new_state = st; }
    return a;
  }
  a.valid = true;
  a.new_state = st ^ c.F;
  a.me = (popc64(st & c.smask) & 1) ? -c.K : c.K;
  return a;
}

}  // namespace qkb
