"""qkrylov_b200_multi_dot_noalloc: the multi-vector dot for callers that
cannot let a library allocate device memory (memory owned by another
allocator's pool, or loops where an allocation or free would stall their
streams).  Its scratch is a fixed device array inside the library, so it
must agree with the allocating qkrylov_b200_multi_dot on the same inputs,
twice in a row (the array keeps the previous call's contents), and reject
more vectors than the array holds.

This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import qkrylov_b200 as qk

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _call(fn, k, V, x, code, n, extra=()):
    ptrs = (ctypes.c_void_p * k)(*[v.data_ptr() for v in V])
    out = np.zeros(2 * k)
    rc = fn(torch.cuda.current_device(), code, n, k, ptrs, ctypes.c_void_p(x.data_ptr()), out.ctypes.data, *extra)
    return rc, out


def _vec(rng, n, tdt):
    v = rng.standard_normal(n)
    if tdt.is_complex:
        v = v + 1j * rng.standard_normal(n)
    return torch.tensor(v, device="cuda").to(tdt)


@pytest.mark.parametrize("code,tdt,tol", [(qk.DTYPE_C128, torch.complex128, 1e-13), (qk.DTYPE_C64, torch.complex64, 1e-6),
                                          (qk.DTYPE_F64, torch.float64, 1e-13), (qk.DTYPE_F32, torch.float32, 1e-6)])
def test_noalloc_matches_allocating_entry_point(code, tdt, tol):
    L = qk.lib()
    rng = np.random.default_rng(11)
    # consecutive calls on the shared array: a full-size call, a smaller k,
    # one vector shorter than one 2048-element tile
    for n, k in [(1_000_003, 16), (77_777, 5), (100, 1)]:
        V = [_vec(rng, n, tdt) for _ in range(k)]
        x = _vec(rng, n, tdt)
        rc0, ref = _call(L.qkrylov_b200_multi_dot, k, V, x, code, n)
        rc1, got = _call(L.qkrylov_b200_multi_dot_noalloc, k, V, x, code, n, (None,))
        assert rc0 == 0 and rc1 == 0, L.qkrylov_b200_last_error()
        scale = np.abs(ref).max()
        assert np.abs(got - ref).max() <= tol * scale


def test_noalloc_empty_vectors_give_zeros():
    L = qk.lib()
    k = 3
    V = [torch.ones(4, dtype=torch.float64, device="cuda") for _ in range(k)]
    x = torch.ones(4, dtype=torch.float64, device="cuda")
    rc, out = _call(L.qkrylov_b200_multi_dot_noalloc, k, V, x, qk.DTYPE_F64, 0, (None,))
    assert rc == 0 and np.all(out == 0.0)


def test_noalloc_rejects_a_device_that_does_not_exist():
    L = qk.lib()
    n, k = 10, 1
    V = [torch.zeros(n, dtype=torch.float64, device="cuda")]
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    ptrs = (ctypes.c_void_p * k)(*[v.data_ptr() for v in V])
    out = np.zeros(2 * k)
    rc = L.qkrylov_b200_multi_dot_noalloc(torch.cuda.device_count(), qk.DTYPE_F64, n, k, ptrs,
                                          ctypes.c_void_p(x.data_ptr()), out.ctypes.data, None)
    assert rc == -1 and b"invalid argument" in L.qkrylov_b200_last_error()


def test_noalloc_rejects_too_many_vectors():
    L = qk.lib()
    n, k = 1000, 17
    V = [torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(k)]
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    rc, _ = _call(L.qkrylov_b200_multi_dot_noalloc, k, V, x, qk.DTYPE_F64, n, (None,))
    assert rc == -1
    assert b"exceeds the static scratch maximum of 16" in L.qkrylov_b200_last_error()
