"""Row-range H.x on the GPU (the building block of the row-sharded apply):
the rows of every shard, computed separately from the complete x, put
together give the full H.x bit for bit (row kernel, two-part kernel and
generic kernel); bounds that are not sector-block boundaries are rejected;
the sharded Lanczos on one GPU through the range apply matches the
library's Lanczos.  The exchange step between GPUs (NCCL all-gather) is
covered with gloo ranks on the CPU (tests/test_sharded.py)."""
import ctypes

import numpy as np
import pytest
import torch

import oracle as O
import qkrylov_b200 as qk
from qkrylov_b200 import sharded
from test_gpu_hx import ham

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,N,sec,terms,basis", [
    ("spin", 18, dict(use_sz=1, sz2=0), O.heisenberg_chain(18), lambda: qk.SpinHalfBasis(18, sz=0)),
    ("tj", 12, dict(use_nup=1, nup=5, use_ndn=1, ndn=5), O.tj_chain(12, 1.0, 0.4),
     lambda: qk.TJBasis(12, conserve_nup=True, nup=5, conserve_ndn=True, ndn=5)),
    ("spin", 10, dict(use_sz=1, sz2=0), [(1.0, [("Sx", 0), ("Sx", 3)])] + O.heisenberg_chain(10),
     lambda: qk.SpinHalfBasis(10, sz=0)),
])
def test_shards_reassemble_the_full_apply(kind, N, sec, terms, basis):
    H = ham(kind, N, sec, terms)
    B = basis()
    D = H.dimension
    x = torch.randn(D, dtype=torch.complex128, device="cuda", generator=torch.Generator("cuda").manual_seed(1))
    y_full = torch.empty_like(x)
    H.apply_device(x.data_ptr(), y_full.data_ptr(), qk.DTYPE_C128)
    for n in (1, 2, 3, 7):
        b = sharded.shard_bounds(B, n)
        y = torch.full_like(x, complex(float("nan"), 0.0))
        for k in range(n):
            rc = qk.lib().qkrylov_hamiltonian_apply_range_device(H._h, qk.DTYPE_C128, ctypes.c_void_p(x.data_ptr()),
                                                                 ctypes.c_void_p(y.data_ptr()), int(b[k]),
                                                                 int(b[k + 1]), None)
            assert rc == 0, qk.lib().qkrylov_b200_last_error()
        torch.cuda.synchronize()
        assert torch.equal(y, y_full), (kind, n)


def test_range_bounds_must_be_block_boundaries():
    H = ham("spin", 12, dict(use_sz=1, sz2=0), O.heisenberg_chain(12))
    st = qk.SpinHalfBasis(12, sz=0).states()
    # a row inside a sector block: its state shares every bit above bit 1
    # with the previous row's, so no split of the 12 bits separates them
    r = int(next(i for i in range(1, len(st)) if (int(st[i]) >> 2) == (int(st[i - 1]) >> 2)))
    x = torch.zeros(H.dimension, dtype=torch.float64, device="cuda")
    y = torch.zeros_like(x)
    rc = qk.lib().qkrylov_hamiltonian_apply_range_device(H._h, qk.DTYPE_F64, ctypes.c_void_p(x.data_ptr()),
                                                         ctypes.c_void_p(y.data_ptr()), r, H.dimension, None)
    assert rc == -1 and b"block" in qk.lib().qkrylov_b200_last_error()


def test_sharded_lanczos_on_one_gpu_matches_lanczos():
    N = 16
    H = ham("spin", N, dict(use_sz=1, sz2=0), O.heisenberg_chain(N))
    B = qk.SpinHalfBasis(N, sz=0)
    b = sharded.shard_bounds(B, 1)
    x0 = torch.rand(H.dimension, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(3))
    r = sharded.lanczos_sharded(sharded.gpu_apply_rows(H, qk.DTYPE_F64), H.dimension, b, x0 - 0.5, 200, 1e-12,
                                want_vector=True)
    ref = qk.lanczos_fp64(H, seed=1, tol=1e-12)
    assert r.converged and abs(r.energy - ref.energy) < 1e-11
