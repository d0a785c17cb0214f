"""Operator application and batched spectral evaluation on the GPU.

* qkrylov_b200_apply_operator: y = O x for an OpSum without a Hamiltonian
  handle (Sz(q)|psi>, correlation functions <psi|Sz_i Sz_j|psi>), against
  numpy and the CPU oracle;
* qkrylov_b200_spectral_function_batch: S(omega) of many continued
  fractions at many frequencies in one call, against the one-frequency
  evaluate_spectral_function (the reference's semantics, itself pinned to
  the reference's golden S(omega)) and the golden values directly."""
import numpy as np
import pytest

import oracle as O
import qkrylov_b200 as qk
from test_gpu_hx import ham

pytestmark = pytest.mark.gpu


def test_spectral_batch_matches_per_frequency_and_golden(golden, golden_vecs):
    m = golden["models"]["heis12_sz0"]
    H = ham("spin", 12, m["sector"], O.heisenberg_chain(12))
    cf = qk.continued_fraction_coeffs(H, golden_vecs["heis12_sz0/phi_szpi"], 40)
    E0 = m["lanczos"]["energy"]
    w = np.array(m["spectral"]["omega"])
    S = qk.spectral_function_batch(cf, w, E0, 0.05)
    S1 = np.array([qk.evaluate_spectral_function(cf, x, E0, 0.05) for x in w])
    S_ref = np.array(m["spectral"]["S"])
    assert np.abs(S - S1).max() <= 1e-13 * np.abs(S1).max()
    assert np.abs(S - S_ref).max() <= 1e-10 * np.abs(S_ref).max()


def test_spectral_batch_ragged_fractions():
    rng = np.random.default_rng(4)
    rs = []
    for n in (7, 1, 0, 30):
        rs.append(qk.DynamicsResult(rng.standard_normal(n), np.abs(rng.standard_normal(max(n - 1, 0))) + 0.1,
                                    0.5 + n / 10))
    w = np.linspace(-3.0, 3.0, 513)
    S = qk.spectral_function_batch(rs, w, 0.25, 0.1)
    assert S.shape == (4, 513)
    for c, r in enumerate(rs):
        one = np.array([qk.evaluate_spectral_function(r, x, 0.25, 0.1) for x in w])
        scale = max(np.abs(one).max(), 1e-300)
        assert np.abs(S[c] - one).max() <= 1e-13 * scale, c
    assert np.all(S[2] == 0.0)


def test_apply_operator_szq_and_correlations():
    N = 12
    sec = dict(use_sz=1, sz2=0)
    H = ham("spin", N, sec, O.heisenberg_chain(N))
    gs = qk.lanczos_fp64(H, seed=2, tol=1e-12, eigenvector=True)
    psi = gs.eigenvector
    B = qk.SpinHalfBasis(N, sz=0)
    st = B.states()
    spin = (((st[:, None] >> np.arange(N, dtype=np.uint64)[None, :]) & np.uint64(1)).astype(np.float64) - 0.5)
    # Sz(pi)|psi> = N^-1/2 sum_j (-1)^j Sz_j |psi>
    szq = qk.OpSum(dtype=np.float64)
    for j in range(N):
        szq.add_term((-1.0) ** j / np.sqrt(N), "Sz", j)
    y = qk.apply_operator(B, qk.SpinHalfSite(), szq, psi)
    want = psi * (spin * ((-1.0) ** np.arange(N))[None, :]).sum(axis=1) / np.sqrt(N)
    assert np.abs(y - want).max() <= 1e-14 * np.abs(want).max()
    # <psi|S_0 . S_d|psi> (diagonal and exchange parts) against the oracle
    for d in (1, 3, 6):
        op = qk.OpSum(dtype=np.float64)
        op.add_term(1.0, "Sz", 0, "Sz", d)
        op.add_term(0.5, "Sp", 0, "Sm", d)
        op.add_term(0.5, "Sm", 0, "Sp", d)
        _, e = qk.apply_operator(B, qk.SpinHalfSite(), op, psi, expectation=True)
        terms = [(1.0, [("Sz", 0), ("Sz", d)]), (0.5, [("Sp", 0), ("Sm", d)]), (0.5, [("Sm", 0), ("Sp", d)])]
        yo = O.port().hamiltonian("spin", N, sec, terms).apply(psi.astype(np.complex128))
        e_ref = np.vdot(psi, yo)
        assert abs(e - e_ref) <= 1e-13 and abs(e.imag) <= 1e-15
    # sum over bonds of <S_i . S_i+1> is the energy
    _, e = qk.apply_operator(B, qk.SpinHalfSite(), _heis(N), psi, expectation=True)
    assert abs(e.real - gs.energy) <= 1e-12 * abs(gs.energy)


def _heis(N):
    op = qk.OpSum(dtype=np.float64)
    for i in range(N):
        j = (i + 1) % N
        op.add_term(1.0, "Sz", i, "Sz", j)
        op.add_term(0.5, "Sp", i, "Sm", j)
        op.add_term(0.5, "Sm", i, "Sp", j)
    return op
