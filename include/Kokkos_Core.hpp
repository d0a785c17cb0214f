// Compatibility header for callers of the qkrylov C++ API that include
// <Kokkos_Core.hpp> only to bracket their program with Kokkos::initialize /
// Kokkos::finalize and to name Kokkos::DefaultExecutionSpace (the
// reference's own tests do: tests/test_vector_ops.cpp:4-11 of qkrylov).
// This library has no Kokkos: the names resolve to the single CUDA
// execution-space tag of qkrylov/core/kokkos_types.hpp.  A program that
// uses the real Kokkos for other work puts the real header first on its
// include path; kokkos_types.hpp then leaves the Kokkos namespace alone.
#pragma once

#include "qkrylov/core/kokkos_types.hpp"
