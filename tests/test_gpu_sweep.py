"""Batched coupling sweep on the GPU: ground states of H0 + g H1 for many
couplings g as one block of Lanczos recurrences, against the plain FP64
GPU Lanczos run on each H0 + g H1 separately and against the CPU oracle.
Acceptance is the same as for the one-vector solvers: explicit residual
|H psi - E psi| / |E| <= tol and |dE| < 1e-10."""
import numpy as np
import pytest

import oracle as O
import qkrylov_b200 as qk
from test_gpu_hx import ham

pytestmark = pytest.mark.gpu

TOL = 1e-10
SZ0 = dict(use_sz=1, sz2=0)


def nnn_terms(N):
    terms = []
    for i in range(N):
        j = (i + 2) % N
        terms += [(1.0, [("Sz", i), ("Sz", j)]), (0.5, [("Sp", i), ("Sm", j)]), (0.5, [("Sm", i), ("Sp", j)])]
    return terms


def test_j1j2_sweep_matches_one_at_a_time():
    N = 16
    H0 = ham("spin", N, SZ0, O.heisenberg_chain(N))
    H1 = ham("spin", N, SZ0, nnn_terms(N))
    g = np.linspace(0.0, 1.0, 32)
    r = qk.lanczos_sweep(H0, H1, g, tol=TOL)
    assert r.block == 32 and r.converged.all() and (r.residuals <= TOL).all()
    for q in (0, 5, 11, 17, 24, 31):
        ref = qk.lanczos_fp64(ham("spin", N, SZ0, O.j1j2_chain(N, 1.0, g[q])), seed=3, tol=TOL)
        assert abs(r.energies[q] - ref.energy) < 1e-10, (q, r.energies[q], ref.energy)


def test_sweep_against_oracle():
    N = 14
    H0 = ham("spin", N, SZ0, O.heisenberg_chain(N))
    H1 = ham("spin", N, SZ0, nnn_terms(N))
    g = [0.1, 0.45, 0.8]
    r = qk.lanczos_sweep(H0, H1, g, tol=TOL, pass_len=24)
    assert r.converged.all() and r.passes >= 2   # 24-step passes: at least one restart
    for q, gq in enumerate(g):
        E = O.port().hamiltonian("spin", N, SZ0, O.j1j2_chain(N, 1.0, gq)).lanczos(200, 1e-13)["energy"]
        assert abs(r.energies[q] - E) < 1e-10


def test_tj_coupling_sweep_two_part_plan():
    # hopping part and J part of the t-J chain: a sweep over J on the
    # two-part tables (fermion signs, charge-changing crossing groups)
    N, ne = 10, 8
    sec = dict(use_nup=1, nup=ne // 2, use_ndn=1, ndn=ne - ne // 2)
    H0 = ham("tj", N, sec, O.tj_chain(N, 1.0, 0.0))
    H1 = ham("tj", N, sec, O.tj_chain(N, 0.0, 1.0))
    g = [0.2, 0.4, 0.7, 1.0, 1.5]
    r = qk.lanczos_sweep(H0, H1, g, tol=TOL)
    assert r.block == 32 and r.converged.all()
    for q, gq in enumerate(g):
        ref = qk.lanczos_fp64(ham("tj", N, sec, O.tj_chain(N, 1.0, gq)), seed=2, tol=TOL)
        assert abs(r.energies[q] - ref.energy) < 1e-10


def test_sweep_is_reproducible_and_block_sizes():
    N = 12
    H0 = ham("spin", N, SZ0, O.heisenberg_chain(N))
    H1 = ham("spin", N, SZ0, nnn_terms(N))
    g = np.linspace(0, 1, 40)   # 64 columns
    a = qk.lanczos_sweep(H0, H1, g, tol=TOL, seed=4)
    b = qk.lanczos_sweep(H0, H1, g, tol=TOL, seed=4)
    assert a.block == 64 and np.array_equal(a.energies, b.energies) and a.steps == b.steps
    c = qk.lanczos_sweep(H0, H1, g[:33], tol=TOL, seed=4)
    assert c.block == 64 and np.max(np.abs(c.energies - a.energies[:33])) < 1e-10


def test_argument_checks():
    H0 = ham("spin", 10, SZ0, O.heisenberg_chain(10))
    H1 = ham("spin", 10, SZ0, nnn_terms(10))
    H8 = ham("spin", 8, SZ0, O.heisenberg_chain(8))
    with pytest.raises(ValueError):
        qk.lanczos_sweep(H0, H8, [0.1])
    with pytest.raises(ValueError):
        qk.lanczos_sweep(H0, H1, [])
    with pytest.raises(ValueError):
        qk.lanczos_sweep(H0, H1, np.zeros(129))
    with pytest.raises(ValueError):
        qk.lanczos_sweep(H0, H1, [0.1], pass_len=1)
    with pytest.raises(ValueError):
        qk.lanczos_sweep(H0, H1, [0.1], tol=0.0)
    terms = O.heisenberg_chain(10) + [(0.3j, [("Sp", 0), ("Sm", 1)]), (-0.3j, [("Sm", 0), ("Sp", 1)])]
    Hc = ham("spin", 10, SZ0, terms)
    with pytest.raises(ValueError):
        qk.lanczos_sweep(Hc, H1, [0.1])


def test_sweep_from_learned_start_vectors():
    # the warm-start network trained on a few couplings gives each column its
    # start vector; same acceptance, fewer steps than random starts
    N = 16
    B = qk.SpinHalfBasis(N, sz=0)
    net = qk.WarmStartMLP(B, seed=0)
    for j in (0.0, 0.15, 0.3, 0.45):
        r = qk.lanczos_fp64(ham("spin", N, SZ0, O.j1j2_chain(N, 1.0, j)), seed=1, tol=TOL, eigenvector=True)
        net.add_target(j, r.eigenvector)
    net.train(steps=400, batch=4096, lr=2e-3, seed=3)
    H0 = ham("spin", N, SZ0, O.heisenberg_chain(N))
    H1 = ham("spin", N, SZ0, nnn_terms(N))
    g = [0.05, 0.1, 0.2, 0.25, 0.35, 0.4]
    w = qk.lanczos_sweep(H0, H1, g, tol=TOL, net=net)
    c = qk.lanczos_sweep(H0, H1, g, tol=TOL)
    assert w.converged.all() and c.converged.all() and w.seconds_inference > 0 and c.seconds_inference == 0
    assert np.max(np.abs(w.energies - c.energies)) < 1e-10
    assert w.steps < c.steps, (w.steps, c.steps)
    H8 = ham("spin", 8, SZ0, O.heisenberg_chain(8))
    with pytest.raises(ValueError):
        qk.lanczos_sweep(H8, H8, g, net=net)   # network on another basis


def test_transverse_field_ising_sweep():
    # single-spin flips on the full basis (no conserved charge): whichever
    # H.X path the plans take, the sweep matches one-at-a-time Lanczos
    N = 10
    full = dict(use_sz=0)
    zz = [(-1.0, [("Sz", i), ("Sz", (i + 1) % N)]) for i in range(N)]
    x = [(-1.0, [("Sx", i)]) for i in range(N)]
    H0, H1 = ham("spin", N, full, zz), ham("spin", N, full, x)
    g = [0.6, 0.8, 1.0, 1.2, 1.6, 2.0]   # away from the near-degenerate ordered pair at small g
    r = qk.lanczos_sweep(H0, H1, g, tol=TOL)
    assert r.converged.all()
    for q, gq in enumerate(g):
        ref = qk.lanczos_fp64(ham("spin", N, full, zz + [(c * gq, f) for c, f in x]), seed=2, tol=TOL)
        assert abs(r.energies[q] - ref.energy) < 1e-10, (gq, r.energies[q], ref.energy)
