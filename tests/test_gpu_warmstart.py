"""Learned warm start on the GPU: the network's loss, gradient and start
vector against the CPU oracle (oracle/mlp.py), training on ground states
from plain Lanczos, and what the trained network gains over a random start
at couplings it was not trained on (same residual acceptance)."""
import numpy as np
import pytest

import oracle as O
from oracle import mlp
import qkrylov_b200 as qk
from test_gpu_hx import ham

pytestmark = pytest.mark.gpu


def j1j2(N, J2):
    return ham("spin", N, dict(use_sz=1, sz2=0), O.j1j2_chain(N, 1.0, J2))


def test_loss_and_gradient_match_oracle():
    N = 12
    B = qk.SpinHalfBasis(N, sz=0)
    net = qk.WarmStartMLP(B, seed=4)
    p = net.params
    assert p.size == mlp.n_params(N) == 128 * 13 + 128 * 128 + 256 + 258
    rng = np.random.default_rng(1)
    states = B.states()[rng.integers(0, B.size, 257)]
    j2 = rng.uniform(0, 1, 257)
    tg = np.stack([rng.standard_normal(257), rng.choice([-1.0, 1.0], 257), rng.uniform(0.5, 1.5, 257)], 1)
    loss, g = net.loss_grad(states, j2, tg, c_sign=0.8)
    lo, go = mlp.loss_grad(p, states, j2, tg, N, 0.8)
    assert abs(loss - lo) <= 1e-5 * abs(lo)
    # FP32 accumulation over 257 samples against FP64
    assert np.max(np.abs(g - go)) <= 2e-4 * np.max(np.abs(go))
    for blk in (slice(0, 128 * 13), slice(128 * 13, 128 * 13 + 128 * 128), slice(-258, None)):
        assert np.max(np.abs(g[blk] - go[blk])) <= 2e-4 * np.max(np.abs(go[blk])) + 1e-7


def test_start_vector_matches_oracle():
    N = 10
    B = qk.SpinHalfBasis(N, sz=0)
    net = qk.WarmStartMLP(B, seed=9)
    net.set_tensor_cores(False)   # CUDA cores: FP32 activations, as in training
    phi = net.start_vector(0.37)
    ref = mlp.start_vector(net.params, B.states(), 0.37, N)
    assert phi.dtype == np.float32
    assert np.max(np.abs(phi - ref)) <= 1e-4 * np.max(np.abs(ref))


@pytest.mark.parametrize("N,j2", [(10, 0.37), (16, 0.81), (24, 0.05)])
def test_tensor_core_inference_matches_oracle(N, j2):
    # tcgen05 MMAs: BF16 weights and activations, FP32 accumulation in TMEM;
    # the oracle rounds the same operands to BF16 and accumulates in FP64
    B = qk.SpinHalfBasis(N, sz=0)
    net = qk.WarmStartMLP(B, seed=2)
    p = net.params
    p[-258:] = np.random.default_rng(0).standard_normal(258).astype(np.float32) * 0.3  # non-zero biases
    net.params = p
    phi = net.start_vector(j2).astype(np.float64)
    st = B.states()
    idx = np.random.default_rng(1).choice(st.size, min(st.size, 4000), replace=False)
    # the start vector is shifted by the largest log-amplitude over the whole basis
    ref_all = mlp.start_vector(net.params, st, j2, N, act_bf16=True) if st.size <= 20000 else None
    if ref_all is not None:
        assert np.max(np.abs(phi - ref_all)) <= 2e-3 * np.max(np.abs(ref_all))
    else:
        X = mlp.inputs(st[idx], j2, N)
        O = mlp.forward(net.params, X, N, act_bf16=True)["O"]
        m = np.where(np.array([bin(int(v)).count("1") & 1 for v in (st[idx] & np.uint64(mlp.marshall_mask(N)))]) == 1,
                     -1.0, 1.0)
        ratio = phi[idx] / (m * np.exp(O[:, 0]) * np.tanh(O[:, 1]))   # exp(-shift), the same for every state
        assert np.max(np.abs(ratio / np.median(ratio) - 1)) < 5e-3
    net.set_tensor_cores(False)
    phi32 = net.start_vector(j2).astype(np.float64)
    cos = abs(phi @ phi32) / (np.linalg.norm(phi) * np.linalg.norm(phi32))
    assert cos > 0.999


def test_training_and_warm_start_gain():
    N = 16
    train_j2 = [0.0, 0.15, 0.3, 0.45]
    net = qk.WarmStartMLP(qk.SpinHalfBasis(N, sz=0), seed=0)
    for j in train_j2:
        r = qk.lanczos_fp64(j1j2(N, j), seed=1, tol=1e-10, eigenvector=True)
        net.add_target(j, r.eigenvector)
    loss = net.train(steps=400, batch=4096, lr=2e-3, seed=3)
    assert loss[-20:].mean() < 0.5 * loss[:20].mean()
    for j in (0.075, 0.375):   # couplings not trained on
        H = j1j2(N, j)
        ref = qk.lanczos_fp64(H, seed=2, tol=1e-10, eigenvector=True)
        phi = net.start_vector(j).astype(np.float64)
        ov = abs(phi @ ref.eigenvector) / np.linalg.norm(phi)
        assert ov > 0.9, (j, ov)             # a random start has overlap ~ 1/sqrt(dim) = 0.01
        w = qk.lanczos_warm(H, net, j, tol=1e-10)
        c = qk.lanczos_mixed(H, seed=2, tol=1e-10)
        assert w.converged and w.residual <= 1e-10
        assert abs(w.energy - ref.energy) < 1e-10
        assert w.iterations_low + w.iterations_high < c.iterations_low + c.iterations_high
        assert w.seconds_inference > 0
