"""Block H.X through the public entry point qkrylov_b200_apply_block_device:
R row-interleaved vectors (element (i, r) at X[i*R + r]) against the CPU
oracle's one-vector apply, column by column, for every shape (lanes per
row 8 / 16 / 32 and the tuned one), each kernel family (exchange row
tables, two-part tables, the generic term walk) and both real precisions,
with the fused column dots <X_r, Y_r>; and the tuner's timing table."""
import numpy as np
import pytest
import torch

import oracle as O
import qkrylov_b200 as qk
from test_gpu_hx import ham

pytestmark = pytest.mark.gpu

MODELS = [
    ("spin", 16, dict(use_sz=1, sz2=0), O.j1j2_chain(16, 1.0, 0.3)),
    ("tj", 12, dict(use_nup=1, nup=5, use_ndn=1, ndn=5), O.tj_chain(12)),
    ("hubbard", 8, dict(use_nup=1, nup=4, use_ndn=1, ndn=4), O.hubbard_square(4, 2)),
    ("fermion", 12, dict(use_n=1, n=5), [(-1.0, [("C", (i + 1) % 12), ("Cdag", i)]) for i in range(12)]
     + [(-1.0, [("C", i), ("Cdag", (i + 1) % 12)]) for i in range(12)]
     + [(0.4, [("N", i), ("N", (i + 2) % 12)]) for i in range(12)]),
]


@pytest.mark.parametrize("kind,N,sec,terms", MODELS, ids=[m[0] for m in MODELS])
@pytest.mark.parametrize("prec", [64, 32])
def test_block_apply_matches_oracle(kind, N, sec, terms, prec):
    H = ham(kind, N, sec, terms)
    Po = O.port().hamiltonian(kind, N, sec, terms)
    n = H.dimension
    tdt, code, tol = (torch.float64, qk.DTYPE_F64, 1e-12) if prec == 64 else (torch.float32, qk.DTYPE_F32, 2e-5)
    for R in (32, 64):
        rng = np.random.default_rng(R + N)
        Xh = rng.standard_normal((n, R))
        X = torch.tensor(Xh, dtype=tdt, device="cuda").contiguous()
        ref = np.stack([Po.apply(Xh[:, r].astype(np.complex128)).real for r in range(R)], axis=1)
        scale = np.abs(ref).max()
        for lpr in (0, 32, 16, 8):
            if lpr and R // lpr > 8:
                continue
            Y = torch.full_like(X, float("nan"))
            torch.cuda.synchronize()  # the fill runs on torch's stream, the apply on the library's
            dots = H.apply_block_device(X.data_ptr(), Y.data_ptr(), code, R, lanes_per_row=lpr, dots=True)
            torch.cuda.synchronize()
            Yh = Y.double().cpu().numpy()
            assert np.abs(Yh - ref).max() <= tol * scale, (R, lpr)
            d_ref = np.einsum("ir,ir->r", Xh, ref)
            assert np.abs(dots[0::2] - d_ref).max() <= tol * np.abs(d_ref).max() * 10, (R, lpr)
            assert np.all(dots[1::2] == 0.0)
        t = H.block_shape_timings(prec, R)
        assert t.shape == (3, 3) and t.max() > 0.0


def test_block_apply_rejects_bad_arguments():
    H = ham("spin", 10, dict(use_sz=1, sz2=0), O.heisenberg_chain(10))
    X = torch.zeros(H.dimension * 32, dtype=torch.float64, device="cuda")
    Y = torch.zeros_like(X)
    with pytest.raises(Exception):
        H.apply_block_device(X.data_ptr(), Y.data_ptr(), qk.DTYPE_F64, 48)  # R not 32/64/128
    with pytest.raises(Exception):
        H.apply_block_device(X.data_ptr(), X.data_ptr(), qk.DTYPE_F64, 32)  # aliased
    with pytest.raises(Exception):
        H.apply_block_device(X.data_ptr(), Y.data_ptr(), qk.DTYPE_F64, 32, lanes_per_row=12)
    with pytest.raises(Exception):
        H.apply_block_device(X.data_ptr() + 8, Y.data_ptr(), qk.DTYPE_F64, 32)  # misaligned
