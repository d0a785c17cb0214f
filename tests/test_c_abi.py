"""The C-ABI boundary without a GPU: every entry point declared in
include/*.h is exported by libqkrylov_b200.so, and argument checks return
the reference's status codes and sentinels (src/c_api.cpp)."""
import ctypes
import glob
import os
import re

import pytest

import qkrylov_b200 as qk
from qkrylov_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(qkrylov_\w+)\s*\(", src):
            names.add(m.group(1))
    return sorted(names)


def test_every_declared_symbol_is_exported():
    L = qk.lib()
    names = declared()
    assert len(names) >= 60
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # the loader declares prototypes for all of them
    assert not [n for n in names if n not in _lib.PROTOTYPES]


def test_reference_entry_points_all_present():
    # the 43 functions of the reference C ABI (include/qkrylov/c_api.h:30-168)
    ref = """sector_create sector_destroy sector_set_sz sector_set_hubbard_particles sector_set_n sector_set_nb
    sector_get_sz sector_get_hubbard_particles sector_get_n sector_get_nb spinhalf_basis_create fermion_basis_create
    hubbard_basis_create tj_basis_create basis_destroy basis_dimension basis_nsites basis_state basis_index
    basis_contains spinhalf_site_create fermion_site_create hubbard_site_create tj_site_create site_destroy
    opsum_create opsum_destroy opsum_clear opsum_add_term_1body opsum_add_term_2body opsum_add_term_nbody
    hamiltonian_create hamiltonian_destroy hamiltonian_dimension hamiltonian_apply hamiltonian_apply_complex
    hamiltonian_diagonal lanczos_ground_state lanczos_ground_state_complex davidson_lowest_complex
    continued_fraction_coeffs_complex evaluate_spectral_function ftlm""".split()
    assert len(ref) == 43
    L = qk.lib()
    assert all(hasattr(L, "qkrylov_" + n) for n in ref)


def test_null_arguments_and_sentinels():
    L = qk.lib()
    assert L.qkrylov_sector_set_sz(None, 0) == -1
    assert L.qkrylov_sector_get_n(None, None, None) == -1
    assert L.qkrylov_basis_dimension(None) == 0
    assert L.qkrylov_basis_nsites(None) == 0
    assert L.qkrylov_basis_index(None, 3) == -1
    assert L.qkrylov_basis_contains(None, 3) == 0
    assert L.qkrylov_opsum_clear(None) == -1
    assert L.qkrylov_opsum_add_term_1body(None, 1.0, 0.0, b"Sz", 0) == -1
    assert L.qkrylov_hamiltonian_create(None, None, None) is None
    assert L.qkrylov_hamiltonian_dimension(None) == 0
    assert L.qkrylov_hamiltonian_apply(None, None, None, None, None) == -1
    assert L.qkrylov_hamiltonian_apply_complex(None, None, None) == -1
    assert L.qkrylov_hamiltonian_diagonal(None, None) == -1
    assert L.qkrylov_lanczos_ground_state(None, 10, ctypes.c_float(1e-6), None) == -1
    assert L.qkrylov_davidson_lowest_complex(None, 1, 10, ctypes.c_float(1e-6), None, None, None) == -1
    assert L.qkrylov_continued_fraction_coeffs_complex(None, None, 5, None, None, None, None) == -1
    assert L.qkrylov_ftlm(None, ctypes.c_float(1.0), 2, 2, None) == -1
    a = (ctypes.c_float * 2)(1.0, 2.0)
    assert L.qkrylov_evaluate_spectral_function(a, a, 0, 1.0, 0.5, 0.0, 0.1) == 0.0
    assert L.qkrylov_evaluate_spectral_function(None, a, 2, 1.0, 0.5, 0.0, 0.1) == 0.0


def test_sector_roundtrip_and_basis_queries():
    L = qk.lib()
    s = L.qkrylov_sector_create()
    assert L.qkrylov_sector_set_sz(s, 0) == 0
    v, act = ctypes.c_int(), ctypes.c_int()
    assert L.qkrylov_sector_get_sz(s, ctypes.byref(v), ctypes.byref(act)) == 0 and (v.value, act.value) == (0, 1)
    b = L.qkrylov_spinhalf_basis_create(4, s)
    assert L.qkrylov_basis_dimension(b) == 6 and L.qkrylov_basis_nsites(b) == 4
    s0 = L.qkrylov_basis_state(b, 0)
    assert L.qkrylov_basis_contains(b, s0) == 1 and L.qkrylov_basis_index(b, s0) == 0
    assert L.qkrylov_basis_index(b, 0b0111) == -1
    assert L.qkrylov_basis_state(b, 6) == 0          # out of range -> 0, as the reference's try/catch
    # test_c_api.cpp:32-33: setting n / nb on the same sector is accepted
    assert L.qkrylov_sector_set_n(s, 2) == 0 and L.qkrylov_sector_set_nb(s, 1) == 0
    L.qkrylov_basis_destroy(b)
    assert L.qkrylov_spinhalf_basis_create(0, s) is None   # constructor error -> NULL
    L.qkrylov_sector_destroy(s)


def test_opsum_nbody_validation():
    L = qk.lib()
    o = L.qkrylov_opsum_create()
    ops = (ctypes.c_char_p * 3)(b"Sz", b"Sz", b"Sz")
    sites = (ctypes.c_int * 3)(0, 1, 2)
    assert L.qkrylov_opsum_add_term_nbody(o, 0.1, 0.0, 3, ops, sites) == 0
    assert L.qkrylov_opsum_add_term_nbody(o, 0.1, 0.0, 0, ops, sites) == -1
    bad = (ctypes.c_char_p * 2)(b"Sz", None)
    assert L.qkrylov_opsum_add_term_nbody(o, 0.1, 0.0, 2, bad, sites) == -1
    assert L.qkrylov_opsum_size(o) == 1
    L.qkrylov_opsum_destroy(o)


def test_extension_entry_points_reject_bad_arguments():
    # the batched entry points check their arguments before touching a GPU
    L = qk.lib()
    g = (ctypes.c_double * 2)(0.1, 0.2)
    e = (ctypes.c_double * 2)()
    assert L.qkrylov_b200_lanczos_sweep(None, None, 2, g, 64, 16, 1e-10, 1, None, e, None, None, None) == -1
    assert L.qkrylov_b200_cf_block(None, 64, 0, 32, 10, g, 0, 1, e, e, None, None, None) == -1
    assert L.qkrylov_b200_ftlm_block(None, 64, 32, 10, 1, 1, g, None, None, None, 1, None) == -1
    assert L.qkrylov_b200_davidson_block(None, 64, 1, 8, 64, 1e-6, 1, 10, e, None, None, None) == -1
