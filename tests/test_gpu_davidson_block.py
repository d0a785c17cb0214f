"""Block Davidson (real vectors, bounded basis, diagonal preconditioner)
against the dense spectrum of small operators and against Lanczos."""
import numpy as np
import pytest

import oracle as O
import qkrylov_b200 as qk
from test_gpu_hx import ham

pytestmark = pytest.mark.gpu


def dense(H):
    dim = H.dimension
    M = np.zeros((dim, dim))
    for j in range(dim):
        e = np.zeros(dim, np.complex128)
        e[j] = 1.0
        M[:, j] = H.apply(e).real
    return M


@pytest.mark.parametrize("model", [
    ("spin", 12, dict(use_sz=1, sz2=0), O.j1j2_chain(12, 1.0, 0.3)),
    ("hubbard", 6, dict(use_nup=1, nup=3, use_ndn=1, ndn=3), O.hubbard_square(3, 2, 1.0, 4.0)),
    ("tj", 8, dict(use_nup=1, nup=3, use_ndn=1, ndn=3), O.tj_chain(8, 1.0, 0.4)),
])
def test_lowest_eigenvalues_match_dense(model):
    H = ham(*model)
    ev = np.linalg.eigvalsh(dense(H))[:4]
    r = qk.davidson_block(H, n_eig=4, block=8, max_subspace=48, tol=1e-8, seed=3, eigenvectors=True)
    assert r.converged
    assert np.allclose(r.eigenvalues, ev, rtol=0, atol=1e-9), (r.eigenvalues, ev)
    for a in range(4):
        v = r.eigenvectors[a]
        assert abs(np.linalg.norm(v) - 1) < 1e-10
        res = np.linalg.norm(H.apply(v.astype(np.complex128)).real - r.eigenvalues[a] * v)
        assert res < 1e-8 * 1.01


def test_restarts_and_fp32():
    # a small subspace forces restarts; FP32 vectors still find the spectrum
    H = ham("spin", 14, dict(use_sz=1, sz2=0), O.heisenberg_chain(14))
    ref = qk.lanczos_fp64(H, seed=1, tol=1e-12)
    r = qk.davidson_block(H, n_eig=2, block=4, max_subspace=12, tol=1e-7, seed=5)
    assert r.converged and r.restarts > 0
    assert abs(r.eigenvalues[0] - ref.energy) < 1e-9
    r32 = qk.davidson_block(H, n_eig=2, block=4, max_subspace=24, tol=1e-4, seed=5, precision=32)
    assert abs(r32.eigenvalues[0] - ref.energy) < 1e-5 * abs(ref.energy)


def test_argument_checks():
    H = ham("spin", 8, dict(use_sz=1, sz2=0), O.heisenberg_chain(8))
    with pytest.raises(RuntimeError):
        qk.davidson_block(H, n_eig=4, block=2)        # block < n_eig
    with pytest.raises(RuntimeError):
        qk.davidson_block(H, n_eig=2, block=4, max_subspace=8)


def test_restarts_keep_the_previous_ritz_vectors():
    """Hubbard 4x2 (4 up, 4 down; dim 4900) with a small basis: many
    restarts, each keeping 2*block Ritz vectors plus the previous
    iteration's; the 4 lowest eigenvalues converge to the sparse
    eigensolver's values."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as sla
    model = ("hubbard", 8, dict(use_nup=1, nup=4, use_ndn=1, ndn=4), O.hubbard_square(4, 2, 1.0, 4.0))
    H = ham(*model)
    r, c, v = O.port().hamiltonian(*model).coo()
    A = sp.csr_matrix((v.real, (r, c)), shape=(H.dimension, H.dimension))
    ev = np.sort(sla.eigsh(A, k=6, which="SA", tol=1e-12)[0])[:4]
    d = qk.davidson_block(H, n_eig=4, block=6, max_subspace=24, tol=1e-8, seed=2, maxiter=300)
    assert d.converged and d.restarts > 2
    assert np.allclose(d.eigenvalues, ev, rtol=0, atol=1e-9), (d.eigenvalues, ev)
