// Objects behind the opaque C-ABI handles.  They hold the engine's
// precision-independent objects; a Hamiltonian handle carries the vector
// precision it was created with (32: the reference C ABI's complex float).
#pragma once

#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "engine/compile.hpp"
#include "engine/operator.hpp"
#include "engine/sector.hpp"

struct qkrylov_sector_t {
  qkb::SectorSpec s;
};
struct qkrylov_basis_t {
  qkb::Family family;
  int nsites;
  std::shared_ptr<const qkb::SectorTable> table;
};
struct qkrylov_site_t {
  qkb::Family family;
};
struct qkrylov_opsum_t {
  std::vector<qkb::TermIn> terms;
};
struct qkrylov_hamiltonian_t {
  std::shared_ptr<qkb::Operator> op;
  int precision;  // 32 or 64
  // Device staging of the host-pointer entry points, kept between calls
  // (calls on one handle are serialised by `mu`).
  std::mutex mu;
  qkb::DevVec sx, sy;
  void stage(qk_dtype t) {
    const uint64_t n = op->dim();
    if (sx.size() != n || sx.dtype() != t) {
      sx = qkb::DevVec(n, t, op->device(), false);
      sy = qkb::DevVec(n, t, op->device(), false);
    }
  }
};

namespace qkapi {
void set_error(const std::string& msg);
}
