"""Batched FTLM on the GPU: R Rademacher vectors advanced as one block
(block H.X, column updates, CUDA graph) against the same vectors run one at
a time through the single-vector kernels, and against exact
thermodynamics of a small spectrum."""
import numpy as np
import pytest

import oracle as O
import qkrylov_b200 as qk
from test_gpu_hx import ham

pytestmark = pytest.mark.gpu

TEMPS = 0.05 * 200.0 ** (np.arange(40) / 39.0)   # 0.05 .. 10


def tj(N, holes=2):
    ne = N - holes
    return ham("tj", N, dict(use_nup=1, nup=ne // 2, use_ndn=1, ndn=ne - ne // 2), O.tj_chain(N, 1.0, 0.4))


def rel(a, b):
    return np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))


@pytest.mark.parametrize("R", [32, 64])
def test_block_fp64_equals_one_vector_loop(R):
    H = tj(10)
    b = qk.ftlm_block(H, TEMPS, n_random=R, n_steps=60, seed=7, precision=64)
    l = qk.ftlm_loop(H, TEMPS, n_random=R, n_steps=60, seed=7, precision=64)
    assert b.graph and b.lanes_per_row in (8, 16, 32)
    assert rel(b.U, l.U) < 1e-10
    assert rel(b.Cv, l.Cv) < 1e-9
    assert np.max(np.abs(b.logZ - l.logZ)) < 1e-10


def test_block_fp32_close_to_fp64_loop():
    H = tj(10)
    b = qk.ftlm_block(H, TEMPS, n_random=64, n_steps=60, seed=3, precision=32)
    l = qk.ftlm_loop(H, TEMPS, n_random=64, n_steps=60, seed=3, precision=64)
    # FP32 vectors, FP64 dots and tridiagonals: agreement at the FP32 level
    assert rel(b.U, l.U) < 1e-4
    assert np.max(np.abs(b.logZ - l.logZ)) < 1e-4
    assert rel(b.Cv, l.Cv) < 1e-3


def test_graph_and_stream_launches_agree():
    H = tj(8)
    a = qk.ftlm_block(H, TEMPS, n_random=32, n_steps=40, seed=1, precision=64, graph=True)
    b = qk.ftlm_block(H, TEMPS, n_random=32, n_steps=40, seed=1, precision=64, graph=False)
    assert a.graph and not b.graph
    assert np.array_equal(a.U, b.U) and np.array_equal(a.Cv, b.Cv) and np.array_equal(a.logZ, b.logZ)


def test_against_exact_spectrum():
    # Heisenberg N=10 Sz=0 (dim 252): with 120 steps every Lanczos run has
    # converged its Krylov space, so what remains is the statistical error of
    # the Rademacher trace estimate, a few per cent of Z at T = 1 for R = 128
    # and shrinking as T grows.
    N = 10
    H = ham("spin", N, dict(use_sz=1, sz2=0), O.heisenberg_chain(N))
    dim = H.dimension
    M = np.zeros((dim, dim))
    for j in range(dim):
        e = np.zeros(dim, np.complex128)
        e[j] = 1.0
        M[:, j] = H.apply(e).real
    ev = np.linalg.eigvalsh(M)
    T = np.array([1.0, 2.0, 5.0, 10.0])
    Ze = np.array([np.exp(-ev / t).sum() for t in T])
    Ue = np.array([(ev * np.exp(-ev / t)).sum() for t in T]) / Ze
    r = qk.ftlm_block(H, T, n_random=128, n_steps=120, seed=11, precision=64)
    assert np.max(np.abs(r.logZ - np.log(Ze))) < 0.06
    assert abs(r.logZ[-1] - np.log(Ze[-1])) < 0.01
    assert np.max(np.abs(r.U - Ue)) < 0.05 * np.max(np.abs(Ue)) + 0.05


def test_argument_checks():
    H = tj(6)
    with pytest.raises((ValueError, RuntimeError)):
        qk.ftlm_block(H, TEMPS, n_random=48)
    with pytest.raises((ValueError, RuntimeError)):
        qk.ftlm_block(H, [0.0, 1.0], n_random=32)
    with pytest.raises((ValueError, RuntimeError)):
        qk.ftlm_block(H, TEMPS, n_random=32, precision=16)
