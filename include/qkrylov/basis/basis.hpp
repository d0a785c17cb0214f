// Hilbert-space basis of one sector (qkrylov's include/qkrylov/basis/basis.hpp:11-24).
// States are listed in ascending integer order, exactly as the reference
// enumerates them; they are ranked by two-level sector tables instead of
// a stored list and a hash map, so no basis is ever enumerated state by
// state.
#pragma once

#include <memory>

#include "qkrylov/core/types.hpp"
#include "qkrylov/symmetry/sector.hpp"

namespace qkb { class SectorTable; }

namespace qkrylov {
namespace QKRYLOV_PRECISION_NAMESPACE {

class Basis {
 public:
  virtual ~Basis() = default;
  virtual Index size() const = 0;
  virtual StateID state(Index i) const = 0;   // std::out_of_range past size()
  virtual Index index(StateID s) const = 0;   // std::runtime_error if absent
  virtual bool contains(StateID s) const = 0;
  // Sector tables behind the bases of this library (nullptr otherwise).
  virtual std::shared_ptr<const qkb::SectorTable> table() const { return nullptr; }
};

namespace detail {
// family: 0 spin-1/2, 1 fermion, 2 Hubbard, 3 t-J
std::shared_ptr<const qkb::SectorTable> make_table(int family, int N, const Sector& sector);
Index table_size(const qkb::SectorTable& t);
StateID table_state(const qkb::SectorTable& t, Index i);
long long table_index(const qkb::SectorTable& t, StateID s);
}  // namespace detail

#define QKRYLOV_DECLARE_BASIS(NAME, FAMILY)                                                   \
  class NAME : public Basis {                                                                 \
   public:                                                                                    \
    NAME(int N, const Sector& sector = Sector{})                                              \
        : N_(N), sector_(sector), table_(detail::make_table(FAMILY, N, sector)) {}            \
    Index size() const override { return detail::table_size(*table_); }                       \
    StateID state(Index i) const override { return detail::table_state(*table_, i); }         \
    Index index(StateID s) const override {                                                   \
      const long long r = detail::table_index(*table_, s);                                    \
      if (r < 0) throw std::runtime_error("State not present in basis");                      \
      return Index(r);                                                                        \
    }                                                                                         \
    bool contains(StateID s) const override { return detail::table_index(*table_, s) >= 0; } \
    int nsites() const noexcept { return N_; }                                                \
    const Sector& sector() const noexcept { return sector_; }                                 \
    std::shared_ptr<const qkb::SectorTable> table() const override { return table_; }         \
                                                                                              \
   private:                                                                                   \
    int N_;                                                                                   \
    Sector sector_;                                                                           \
    std::shared_ptr<const qkb::SectorTable> table_;                                           \
  };

}  // namespace QKRYLOV_PRECISION_NAMESPACE
}  // namespace qkrylov
