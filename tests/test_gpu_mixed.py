"""Mixed-precision Lanczos on the GPU: FP32 vectors and H.x, FP64 alpha,
beta, reorthogonalisation coefficients and tridiagonal, then FP64 refinement
until the explicit residual ||H psi - E psi|| / |E| <= tol.  Energies are
checked against the reference's FP64 Lanczos (golden fixtures) and the CPU
oracle at |dE| < 1e-10; residuals are recomputed independently through the
FP64 apply."""
import numpy as np
import pytest

import oracle as O
import qkrylov_b200 as qk
from test_gpu_hx import ham

pytestmark = pytest.mark.gpu

TOL = 1e-10


def residual(H, E, psi):
    psi = psi.astype(np.complex128)
    return np.linalg.norm(H.apply(psi) - E * psi) / (abs(E) * np.linalg.norm(psi))


def test_mixed_heisenberg16_matches_reference(golden):
    m = golden["models"]["heis16_sz0"]
    E_ref = m["lanczos"]["energy"]
    H = ham("spin", 16, m["sector"], O.heisenberg_chain(16))
    r = qk.lanczos_mixed(H, seed=5, tol=TOL, eigenvector=True)
    assert r.converged and r.residual <= TOL
    assert abs(r.energy - E_ref) < 1e-10
    assert r.eigenvector.dtype == np.float64          # real operator: real FP64 ground state
    assert abs(np.linalg.norm(r.eigenvector) - 1.0) < 1e-12
    assert residual(H, r.energy, r.eigenvector) < 2 * TOL
    assert r.iterations_low > 0 and r.iterations_high > 0
    # energies and Ritz values decrease (Cauchy interlacing within a pass;
    # across passes up to FP32 rounding of the correction)
    es = [e for (it, e, s) in r.trace]
    assert all(b <= a + 1e-6 * abs(a) for a, b in zip(es, es[1:]))
    assert [it for (it, e, s) in r.trace] == list(range(1, len(r.trace) + 1))


def test_mixed_j1j2_vs_oracle():
    N, J2 = 18, 0.35
    model = ("spin", N, dict(use_sz=1, sz2=0), O.j1j2_chain(N, 1.0, J2))
    E_ref = O.port().hamiltonian(*model).lanczos(200, 1e-13)["energy"]
    H = ham(*model)
    r = qk.lanczos_mixed(H, seed=11, tol=TOL)
    assert r.converged and r.residual <= TOL
    assert abs(r.energy - E_ref) < 1e-10


def test_mixed_converges_at_a_small_relative_gap():
    """J1-J2 chain N=24, J2 = 191/255 (dimerised phase: the two lowest
    singlets nearly degenerate), random start seed 2: with passes of a fixed
    32 steps the restarted recurrence stalled near residual 2e-9 and ran out
    of passes; passes that grow when the residual falls less than twentyfold
    reach tol."""
    N, J2 = 24, 191 / 255
    H = ham("spin", N, dict(use_sz=1, sz2=0), O.j1j2_chain(N, 1.0, J2))
    r = qk.lanczos_mixed(H, seed=2, tol=TOL)
    ref = qk.lanczos_fp64(H, seed=2, tol=TOL)
    assert ref.converged
    assert r.converged and r.residual <= TOL
    assert abs(r.energy - ref.energy) < 1e-10


@pytest.mark.parametrize("N,J2", [(18, 0.35), (20, 0.6)])
def test_partial_and_full_reorthogonalisation_agree(N, J2):
    """The default form (partial reorthogonalisation inside the FP32 passes)
    and the form that orthogonalises every step against all the pass's
    vectors reach the same energy at the same explicit residual; the
    oracle's FP64 Lanczos pins both."""
    model = ("spin", N, dict(use_sz=1, sz2=0), O.j1j2_chain(N, 1.0, J2))
    E_ref = O.port().hamiltonian(*model).lanczos(200, 1e-13)["energy"]
    H = ham(*model)
    rp = qk.lanczos_mixed(H, seed=4, tol=TOL, eigenvector=True)
    rf = qk.lanczos_mixed(H, seed=4, tol=TOL, eigenvector=True, reorth="full")
    for r in (rp, rf):
        assert r.converged and r.residual <= TOL
        assert abs(r.energy - E_ref) < 1e-10
        assert residual(H, r.energy, r.eigenvector) < 2 * TOL
    with pytest.raises(ValueError):
        qk.lanczos_mixed(H, reorth="none")


def test_fp64_baseline_reaches_the_same_energy(golden):
    m = golden["models"]["heis16_sz0"]
    H = ham("spin", 16, m["sector"], O.heisenberg_chain(16))
    r = qk.lanczos_fp64(H, seed=5, tol=TOL, eigenvector=True)
    assert r.converged and r.residual <= TOL and r.iterations_low == 0 and r.iterations_high > 0
    assert abs(r.energy - m["lanczos"]["energy"]) < 1e-10
    assert residual(H, r.energy, r.eigenvector) < 2 * TOL


def test_complex_operator_uses_complex_vectors():
    # Heisenberg + Dzyaloshinskii-Moriya z term: (i D / 2) (S+_i S-_j - S-_i S+_j), Hermitian and complex
    N, D = 12, 0.4
    terms = O.heisenberg_chain(N)
    for i in range(N):
        j = (i + 1) % N
        terms += [(0.5j * D, [("Sp", i), ("Sm", j)]), (-0.5j * D, [("Sm", i), ("Sp", j)])]
    H = ham("spin", N, dict(use_sz=1, sz2=0), terms)
    assert not H.all_real
    ref = qk.lanczos_ground_state(H, 300, 1e-14)
    r = qk.lanczos_mixed(H, seed=3, tol=TOL, eigenvector=True)
    assert r.converged and r.residual <= TOL
    assert r.eigenvector.dtype == np.complex128
    assert abs(r.energy - ref.energy) < 1e-10
    assert residual(H, r.energy, r.eigenvector) < 2 * TOL


def test_host_and_device_start_vectors_agree():
    import torch
    N = 14
    H = ham("spin", N, dict(use_sz=1, sz2=0), O.heisenberg_chain(N))
    s = np.random.default_rng(0).uniform(-1, 1, H.dimension).astype(np.float32)
    a = qk.lanczos_mixed(H, start=s, tol=TOL)
    t = torch.from_numpy(s).cuda()
    torch.cuda.synchronize()
    b = qk.lanczos_mixed(H, start_device=t.data_ptr(), tol=TOL)
    assert a.energy == b.energy and a.iterations_low == b.iterations_low
    assert a.iterations_high == b.iterations_high


def test_argument_checks():
    H = ham("spin", 8, dict(use_sz=1, sz2=0), O.heisenberg_chain(8))
    with pytest.raises(ValueError):
        qk.lanczos_mixed(H, maxiter=0)
    with pytest.raises(ValueError):
        qk.lanczos_mixed(H, maxiter=600)
    with pytest.raises(ValueError):
        qk.lanczos_mixed(H, tol=0.0)
    with pytest.raises(ValueError):
        qk.lanczos_mixed(H, start=np.ones(3, np.float32))
