// U(1) sector selection (fields as qkrylov's include/qkrylov/symmetry/sector.hpp:10-41).
#pragma once

#include "qkrylov/core/types.hpp"

namespace qkrylov {
namespace QKRYLOV_PRECISION_NAMESPACE {

struct Sector {
  bool use_sz = false;   // spin-1/2: conserve 2*Sz
  int sz2 = 0;
  bool use_nup = false;  // Hubbard / t-J: conserve N_up, N_dn
  bool use_ndn = false;
  int nup = 0;
  int ndn = 0;
  bool use_n = false;    // spinless fermions: conserve N
  int n = 0;
  bool use_nb = false;   // bosons (accepted, unused, as in qkrylov)
  int nb = 0;
};

}  // namespace QKRYLOV_PRECISION_NAMESPACE
}  // namespace qkrylov
