"""Checkpoints of the Krylov state and of results.

* The continued fraction (the reference's three-term recurrence,
  src/solvers/dynamics.cpp:12-59) saved after some steps and resumed runs to
  the same coefficients, bit for bit, as one uninterrupted run; the saved
  files are plain .npy files numpy reads (alphas, betas, norm_phi0, state,
  and the current and previous Lanczos vectors).
* save_result / load_result keep the dataset names of the reference's
  examples/hdf5_storage.py:5-13."""
import os

import numpy as np
import pytest

import oracle as O
import qkrylov_b200 as qk
from test_gpu_hx import ham

pytestmark = pytest.mark.gpu


def test_cf_resume_is_bit_identical(tmp_path):
    N = 14
    H = ham("spin", N, dict(use_sz=1, sz2=0), O.heisenberg_chain(N))
    rng = np.random.default_rng(3)
    phi = rng.standard_normal(H.dimension) + 1j * rng.standard_normal(H.dimension)
    full = qk.continued_fraction_coeffs(H, phi, 60)
    a = str(tmp_path / "a")
    part = qk.continued_fraction_coeffs(H, phi, 25, save=a)
    assert len(part.alphas) == 25
    b = str(tmp_path / "b")
    rest = qk.continued_fraction_coeffs(H, None, 60, resume=a, save=b)
    assert np.array_equal(rest.alphas, full.alphas) and np.array_equal(rest.betas, full.betas)
    assert rest.norm_phi0 == full.norm_phi0
    # the checkpoint as numpy sees it
    st = np.load(os.path.join(b, "state.npy"))
    assert st[0] == 60 and st[1] == 0
    assert np.array_equal(np.load(os.path.join(b, "alphas.npy")), full.alphas)
    v, vp = np.load(os.path.join(b, "v.npy")), np.load(os.path.join(b, "v_prev.npy"))
    assert v.dtype == np.complex128 and v.shape == (H.dimension,)
    assert abs(np.linalg.norm(v) - 1.0) < 1e-12 and abs(np.vdot(vp, v)) < 1e-8
    # the plain entry point and the checkpointed one agree
    assert np.array_equal(qk.continued_fraction_coeffs(H, phi, 60, save=str(tmp_path / "c")).alphas, full.alphas)


def test_cf_checkpoint_of_a_finished_run_resumes_as_stopped(tmp_path):
    # |up up> is an eigenstate of the two-site Heisenberg model: the
    # recurrence stops after one step (beta = 0)
    H = ham("spin", 2, {}, O.heisenberg_chain(2, periodic=False))
    phi = np.zeros(H.dimension, complex)
    phi[3] = 1.0
    full = qk.continued_fraction_coeffs(H, phi, 40)
    assert len(full.alphas) == 1 and len(full.betas) == 0
    d = str(tmp_path / "s")
    qk.continued_fraction_coeffs(H, phi, 40, save=d)
    again = qk.continued_fraction_coeffs(H, None, 40, resume=d)
    assert np.array_equal(again.alphas, full.alphas) and np.array_equal(again.betas, full.betas)
    assert np.load(os.path.join(d, "state.npy"))[1] == 1


def test_checkpoint_of_another_operator_is_rejected(tmp_path):
    H = ham("spin", 10, dict(use_sz=1, sz2=0), O.heisenberg_chain(10))
    d = str(tmp_path / "x")
    qk.continued_fraction_coeffs(H, np.ones(H.dimension, complex), 5, save=d)
    H2 = ham("spin", 12, dict(use_sz=1, sz2=0), O.heisenberg_chain(12))
    with pytest.raises(RuntimeError):
        qk.continued_fraction_coeffs(H2, None, 10, resume=d)


def test_save_result_uses_the_reference_dataset_names(tmp_path):
    H = ham("spin", 10, dict(use_sz=1, sz2=0), O.heisenberg_chain(10))
    r = qk.lanczos_ground_state(H, 200, 1e-12)
    qk.save_result(str(tmp_path / "l"), r)
    got = qk.load_result(str(tmp_path / "l"))
    assert got["energy"] == r.energy and np.array_equal(got["eigenvector"], np.asarray(r.eigenvector))
    d = qk.davidson_lowest(H, 2, 20, 1e-8)
    qk.save_result(str(tmp_path / "d"), d)
    got = qk.load_result(str(tmp_path / "d"))
    assert np.array_equal(got["eigenvalues"], np.asarray(d.eigenvalues)) and "eigenvector_1" in got
