"""Loader for libqkrylov_b200.so with the C prototypes of its entry points.

The library is built in-tree (python -m qkrylov_b200.build); if it is
missing it is built on first use.  There is no fallback: without the CUDA
library nothing in this package runs.
"""
from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqkrylov_b200.so")


class LibraryError(RuntimeError):
    pass


_vp, _i, _u64, _i64, _d, _f, _cp, _sz = (ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64, ctypes.c_int64,
                                         ctypes.c_double, ctypes.c_float, ctypes.c_char_p, ctypes.c_size_t)

# name: (restype, argtypes)
PROTOTYPES = {
    # qkrylov_c_api.h
    "qkrylov_sector_create": (_vp, []),
    "qkrylov_sector_destroy": (None, [_vp]),
    "qkrylov_sector_set_sz": (_i, [_vp, _i]),
    "qkrylov_sector_set_hubbard_particles": (_i, [_vp, _i, _i]),
    "qkrylov_sector_set_n": (_i, [_vp, _i]),
    "qkrylov_sector_set_nb": (_i, [_vp, _i]),
    "qkrylov_sector_get_sz": (_i, [_vp, _vp, _vp]),
    "qkrylov_sector_get_hubbard_particles": (_i, [_vp, _vp, _vp, _vp]),
    "qkrylov_sector_get_n": (_i, [_vp, _vp, _vp]),
    "qkrylov_sector_get_nb": (_i, [_vp, _vp, _vp]),
    "qkrylov_spinhalf_basis_create": (_vp, [_i, _vp]),
    "qkrylov_fermion_basis_create": (_vp, [_i, _vp]),
    "qkrylov_hubbard_basis_create": (_vp, [_i, _vp]),
    "qkrylov_tj_basis_create": (_vp, [_i, _vp]),
    "qkrylov_basis_destroy": (None, [_vp]),
    "qkrylov_basis_dimension": (_u64, [_vp]),
    "qkrylov_basis_nsites": (_i, [_vp]),
    "qkrylov_basis_state": (_u64, [_vp, _u64]),
    "qkrylov_basis_index": (_i64, [_vp, _u64]),
    "qkrylov_basis_contains": (_i, [_vp, _u64]),
    "qkrylov_spinhalf_site_create": (_vp, []),
    "qkrylov_fermion_site_create": (_vp, []),
    "qkrylov_hubbard_site_create": (_vp, []),
    "qkrylov_tj_site_create": (_vp, []),
    "qkrylov_site_destroy": (None, [_vp]),
    "qkrylov_opsum_create": (_vp, []),
    "qkrylov_opsum_destroy": (None, [_vp]),
    "qkrylov_opsum_clear": (_i, [_vp]),
    "qkrylov_opsum_add_term_1body": (_i, [_vp, _f, _f, _cp, _i]),
    "qkrylov_opsum_add_term_2body": (_i, [_vp, _f, _f, _cp, _i, _cp, _i]),
    "qkrylov_opsum_add_term_nbody": (_i, [_vp, _f, _f, _i, _vp, _vp]),
    "qkrylov_hamiltonian_create": (_vp, [_vp, _vp, _vp]),
    "qkrylov_hamiltonian_destroy": (None, [_vp]),
    "qkrylov_hamiltonian_dimension": (_u64, [_vp]),
    "qkrylov_hamiltonian_apply": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "qkrylov_hamiltonian_apply_complex": (_i, [_vp, _vp, _vp]),
    "qkrylov_hamiltonian_diagonal": (_i, [_vp, _vp]),
    "qkrylov_lanczos_ground_state": (_i, [_vp, _i, _f, _vp]),
    "qkrylov_lanczos_ground_state_complex": (_i, [_vp, _i, _f, _vp, _vp]),
    "qkrylov_davidson_lowest_complex": (_i, [_vp, _i, _i, _f, _vp, _vp, _vp]),
    "qkrylov_continued_fraction_coeffs_complex": (_i, [_vp, _vp, _i, _vp, _vp, _vp, _vp]),
    "qkrylov_evaluate_spectral_function": (_f, [_vp, _vp, _sz, _f, _f, _f, _f]),
    "qkrylov_ftlm": (_i, [_vp, _f, _i, _i, _vp]),
    # qkrylov_b200.h
    "qkrylov_b200_last_error": (_cp, []),
    "qkrylov_b200_launch_count": (_u64, []),
    "qkrylov_b200_device_count": (_i, []),
    "qkrylov_b200_sector_set_species": (_i, [_vp, _i, _i]),
    "qkrylov_b200_set_kernel_policy": (_i, [_i]),
    "qkrylov_b200_die_count": (_i, [_vp, _vp]),
    "qkrylov_hamiltonian_kernel": (_i, [_vp]),
    "qkrylov_b200_site_apply": (_i, [_vp, _cp, _i, _u64, _vp, _vp, _vp]),
    "qkrylov_basis_states": (_i, [_vp, _u64, _u64, _vp]),
    "qkrylov_basis_index_many": (_i, [_vp, _vp, _u64, _vp]),
    "qkrylov_opsum_add_term_nbody_f64": (_i, [_vp, _d, _d, _i, _vp, _vp]),
    "qkrylov_opsum_size": (_u64, [_vp]),
    "qkrylov_opsum_compile": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "qkrylov_hamiltonian_create_ex": (_vp, [_vp, _vp, _vp, _i, _i]),
    "qkrylov_hamiltonian_precision": (_i, [_vp]),
    "qkrylov_hamiltonian_all_real": (_i, [_vp]),
    "qkrylov_hamiltonian_device_bytes": (_u64, [_vp]),
    "qkrylov_hamiltonian_stream": (_vp, [_vp]),
    "qkrylov_hamiltonian_apply_complex_f64": (_i, [_vp, _vp, _vp]),
    "qkrylov_hamiltonian_diagonal_complex_f64": (_i, [_vp, _vp]),
    "qkrylov_hamiltonian_apply_device": (_i, [_vp, _i, _vp, _vp, _vp]),
    "qkrylov_hamiltonian_diagonal_device": (_i, [_vp, _i, _vp, _vp]),
    "qkrylov_b200_multi_dot": (_i, [_i, _i, _sz, _i, _vp, _vp, _vp]),
    "qkrylov_b200_multi_dot_noalloc": (_i, [_i, _i, _sz, _i, _vp, _vp, _vp, _vp]),
    "qkrylov_lanczos_ground_state_f64": (_i, [_vp, _i, _d, _vp, _vp, _vp, _vp, _vp]),
    "qkrylov_davidson_lowest_f64": (_i, [_vp, _i, _i, _d, _vp, _vp, _vp]),
    "qkrylov_continued_fraction_coeffs_f64": (_i, [_vp, _vp, _i, _vp, _vp, _vp, _vp, _vp]),
    "qkrylov_evaluate_spectral_function_f64": (_d, [_vp, _vp, _sz, _d, _d, _d, _d]),
    "qkrylov_b200_spectral_function_batch": (_i, [_i, _i, _i, _vp, _vp, _vp, _vp, _sz, _vp, _d, _d, _vp]),
    "qkrylov_b200_apply_operator": (_i, [_vp, _vp, _vp, _i, _i, _vp, _vp, _vp]),
    "qkrylov_b200_cf_checkpointed": (_i, [_vp, _vp, _cp, _i, _cp, _vp, _vp, _vp, _vp, _vp]),
    "qkrylov_b200_basis_shard_bounds": (_i, [_vp, _i, _vp]),
    "qkrylov_hamiltonian_apply_range_device": (_i, [_vp, _i, _vp, _vp, _u64, _u64, _vp]),
    "qkrylov_b200_block_shape_timings": (_i, [_vp, _i, _i, _vp]),
    "qkrylov_b200_apply_block_device": (_i, [_vp, _i, _i, _i, _vp, _vp, _vp, _vp]),
    "qkrylov_ftlm_sweep_f64": (_i, [_vp, _i, _vp, _i, _i, _vp, _vp, _vp]),
    "qkrylov_b200_lanczos_mixed": (_i, [_vp, _u64, _vp, _i, _i, _d, _vp, _vp, _i, _vp, _vp, _vp]),
    "qkrylov_b200_lanczos_mixed_full": (_i, [_vp, _u64, _vp, _i, _i, _d, _vp, _vp, _i, _vp, _vp, _vp]),
    "qkrylov_b200_lanczos_fp64": (_i, [_vp, _u64, _vp, _i, _i, _d, _vp, _vp, _i, _vp, _vp, _vp]),
    "qkrylov_b200_ftlm_block": (_i, [_vp, _i, _i, _i, _u64, _i, _vp, _vp, _vp, _vp, _i, _vp]),
    "qkrylov_b200_ftlm_loop": (_i, [_vp, _i, _i, _i, _u64, _i, _i, _vp, _vp, _vp, _vp, _vp]),
    "qkrylov_b200_mlp_create": (_vp, [_vp, _i, _u64]),
    "qkrylov_b200_mlp_destroy": (None, [_vp]),
    "qkrylov_b200_mlp_num_params": (_sz, [_vp]),
    "qkrylov_b200_mlp_get_params": (_i, [_vp, _vp]),
    "qkrylov_b200_mlp_set_params": (_i, [_vp, _vp]),
    "qkrylov_b200_mlp_add_target": (_i, [_vp, _d, _vp]),
    "qkrylov_b200_mlp_set_tensor_cores": (_i, [_vp, _i]),
    "qkrylov_b200_mlp_train": (_i, [_vp, _i, _i, _d, _u64, _d, _vp]),
    "qkrylov_b200_mlp_start_vector": (_i, [_vp, _d, _vp, _i]),
    "qkrylov_b200_mlp_loss_grad": (_i, [_vp, _i, _vp, _vp, _vp, _d, _vp, _vp]),
    "qkrylov_b200_lanczos_warm": (_i, [_vp, _vp, _d, _i, _d, _vp, _vp]),
    "qkrylov_b200_davidson_block": (_i, [_vp, _i, _i, _i, _i, _d, _u64, _i, _vp, _vp, _vp, _vp]),
    "qkrylov_b200_cf_block": (_i, [_vp, _i, _i, _i, _i, _vp, _i, _i, _vp, _vp, _vp, _vp, _vp]),
    "qkrylov_b200_lanczos_sweep": (_i, [_vp, _vp, _i, _vp, _i, _i, _d, _u64, _vp, _vp, _vp, _vp, _vp]),
}

_lock = threading.Lock()
_lib = None


def _declare(L):
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(L, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    return L


def lib():
    """The loaded CUDA library (built in-tree on first use if missing)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                from . import build
                build.build()
            if not os.path.exists(LIB_PATH):
                raise LibraryError(f"{LIB_PATH} is missing and could not be built")
            _lib = _declare(ctypes.CDLL(LIB_PATH))
    return _lib


def exported_symbols():
    """Names of the declared entry points present in the loaded library."""
    L = lib()
    return [n for n in PROTOTYPES if hasattr(L, n)]
