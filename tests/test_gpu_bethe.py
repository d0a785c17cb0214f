"""Ground-state energies at the headline sizes against an independent FP64
oracle: the Bethe-ansatz energy of the periodic Heisenberg ring
(oracle/bethe.py, itself pinned to the reference's own E0 values in
tests/test_bethe.py).  The plain FP64 GPU Lanczos and the mixed-precision
form (FP32 vectors, FP64 refinement) must both land within |dE| < 1e-10 of
it at an explicit residual <= 1e-10, at N = 24 (dim 2,704,156) and N = 28
(dim 40,116,600), where the reference's CSR build does not fit in memory."""
import numpy as np
import pytest

import oracle as O
import qkrylov_b200 as qk
from oracle import bethe
from test_gpu_hx import ham

pytestmark = pytest.mark.gpu

TOL = 1e-10


@pytest.mark.parametrize("N", [24, 28])
def test_headline_energies_match_bethe_ansatz(N):
    E_exact = bethe.ground_energy(N)
    H = ham("spin", N, dict(use_sz=1, sz2=0), O.heisenberg_chain(N))
    plain = qk.lanczos_fp64(H, seed=3, tol=TOL)
    mixed = qk.lanczos_mixed(H, seed=3, tol=TOL)
    for r in (plain, mixed):
        assert r.converged and r.residual <= TOL
        assert abs(r.energy - E_exact) < 1e-10, (N, r.energy, E_exact)
    assert mixed.iterations_low > 0
