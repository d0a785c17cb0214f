"""GPU solvers against the reference (golden fixtures) and its pinned tests."""
import numpy as np
import pytest

import oracle as O
import qkrylov_b200 as qk
from conftest import terms_from_golden
from test_gpu_hx import ham

pytestmark = pytest.mark.gpu


def test_lanczos_matches_reference(golden, golden_vecs):
    for name, m in golden["models"].items():
        terms = terms_from_golden(m) if "terms" in m else O.heisenberg_chain(m["N"])
        H = ham(m["kind"], m["N"], m["sector"], terms)
        r = qk.lanczos_ground_state(H, 200, 1e-12)
        ref = m["lanczos"]
        assert abs(r.energy - ref["energy"]) <= 1e-12 * max(1.0, abs(ref["energy"])), name
        assert r.iterations == ref["iterations"] and r.converged == ref["converged"], name
        if f"{name}/lanczos_vec" in golden_vecs:
            v = golden_vecs[f"{name}/lanczos_vec"]
            assert np.abs(r.eigenvector - v).max() < 1e-8, name
            assert abs(np.linalg.norm(r.eigenvector) - 1) < 1e-12


def test_lanczos_alphas_betas_vs_oracle():
    m = ("spin", 14, dict(use_sz=1, sz2=0), O.j1j2_chain(14, 1.0, 0.3))
    H = ham(*m)
    r = qk.lanczos_ground_state(H, 200, 1e-12)
    o = O.port().hamiltonian(*m).lanczos(200, 1e-12)
    k = min(len(r.alphas), len(o["alphas"]))
    assert np.allclose(r.alphas[:k], o["alphas"][:k], rtol=1e-12, atol=1e-12)
    assert np.allclose(r.betas[:k - 1], o["betas"][:k - 1], rtol=1e-11, atol=1e-12)
    assert abs(r.energy - o["energy"]) <= 1e-12 * abs(o["energy"])


def test_davidson_matches_reference(golden):
    for name, m in golden["models"].items():
        if "davidson" not in m:
            continue
        H = ham(m["kind"], m["N"], m["sector"], terms_from_golden(m))
        r = qk.davidson_lowest(H, 2, 10, 1e-8)
        ref = m["davidson"]
        if not ref["converged"]:
            continue  # non-Hermitian test operator: no converged reference to match
        assert r.converged
        assert np.allclose(r.eigenvalues, ref["eigenvalues"], rtol=1e-10, atol=1e-10), name
        for k, v in enumerate(r.eigenvectors):   # residuals
            assert np.abs(H.apply(v) - r.eigenvalues[k] * v).max() < 1e-6, name


def test_cf_and_spectral_match_reference(golden, golden_vecs):
    m = golden["models"]["heis12_sz0"]
    H = ham("spin", 12, m["sector"], O.heisenberg_chain(12))
    cf = qk.continued_fraction_coeffs(H, golden_vecs["heis12_sz0/phi_szpi"], 40)
    assert len(cf.alphas) == len(m["cf_szpi"]["alphas"])
    assert np.allclose(cf.alphas[:6], m["cf_szpi"]["alphas"][:6], rtol=0, atol=1e-12)
    E0 = m["lanczos"]["energy"]
    S_ref = np.array(m["spectral"]["S"])
    S = np.array([qk.evaluate_spectral_function(cf, w, E0, 0.05) for w in m["spectral"]["omega"]])
    assert np.abs(S - S_ref).max() <= 1e-10 * np.abs(S_ref).max()
    for name, mm in golden["models"].items():
        if "cf_e0" not in mm:
            continue
        Hm = ham(mm["kind"], mm["N"], mm["sector"], terms_from_golden(mm))
        phi = np.zeros(Hm.dimension, complex)
        phi[0] = 1.0
        c = qk.continued_fraction_coeffs(Hm, phi, 8)
        k = min(4, len(c.alphas))
        assert np.allclose(c.alphas[:k], mm["cf_e0"]["alphas"][:k], atol=1e-12), name
        assert c.norm_phi0 == mm["cf_e0"]["norm_phi0"]


def test_ftlm_matches_reference(golden):
    for name, m in golden["models"].items():
        if "ftlm" not in m:
            continue
        terms = terms_from_golden(m) if "terms" in m else O.heisenberg_chain(m["N"])
        H = ham(m["kind"], m["N"], m["sector"], terms)
        R, M = (4, 30) if name == "heis12_sz0" else (5, 20)
        res = qk.ftlm_sweep(H, [f["beta"] for f in m["ftlm"]], R, M)
        for f, r in zip(m["ftlm"], res):
            assert abs(r.partition_function - f["Z"]) <= 1e-10 * abs(f["Z"]), name
            assert abs(r.internal_energy - f["U"]) <= 1e-10 * max(1, abs(f["U"])), name
            assert abs(r.specific_heat - f["Cv"]) <= 1e-10 * max(1, abs(f["Cv"])), name


def test_reference_c_api_sequence():
    """tests/test_c_api.cpp:11-157 through the single-precision C ABI."""
    H = qk.MatrixFreeHamiltonian(qk.SpinHalfBasis(4, sz=0), qk.SpinHalfSite(), _obc4(), dtype=np.float32)
    assert H.dimension == 6
    y = H.apply(np.ones(6, np.complex64))
    r = qk.lanczos_ground_state(H, 200, 1e-12)
    assert abs(r.energy - (-1.6160254038)) < 1e-5
    assert abs(np.sum(np.abs(r.eigenvector) ** 2) - 1.0) < 1e-4
    d = qk.davidson_lowest(H, 2, 20, 1e-6)
    assert d.converged and abs(d.eigenvalues[0] - r.energy) < 1e-4 and d.eigenvalues[0] <= d.eigenvalues[1]
    for k in range(2):
        v = d.eigenvectors[k]
        assert np.abs(H.apply(v) - d.eigenvalues[k] * v).max() < 1e-3
    cf = qk.continued_fraction_coeffs(H, r.eigenvector, 20)
    assert len(cf.alphas) > 0 and abs(cf.norm_phi0 - 1.0) < 1e-3
    assert qk.evaluate_spectral_function(cf, 0.5, r.energy, 0.1) > 0.0
    f = qk.ftlm(H, 1.0, 10, 20)
    assert f.partition_function > 0.0
    assert y.shape == (6,)


def _obc4():
    os_ = qk.OpSum(dtype=np.float32)
    for i in range(3):
        os_ += 1.0 * qk.Sz(i) * qk.Sz(i + 1) + 0.5 * qk.Sp(i) * qk.Sm(i + 1) + 0.5 * qk.Sm(i) * qk.Sp(i + 1)
    return os_


def test_reference_julia_constants():
    """bindings/julia/test/runtests.jl:102-106, 154-175, 207-212."""
    os3 = qk.OpSum(dtype=np.float64)
    os3.add_term(1.0, "Sz", 0, "Sz", 1)
    os3.add_term(0.5, "Sz", 0, "Sz", 1, "Sz", 2)
    H3 = qk.MatrixFreeHamiltonian(qk.SpinHalfBasis(3), qk.SpinHalfSite(), os3, dtype=np.float64)
    x = np.zeros(8, complex)
    x[7] = 1.0
    assert abs(H3.apply(x)[7] - 0.3125) < 1e-6
    os4 = qk.OpSum(dtype=np.float64)
    for i in range(4):
        j = (i + 1) % 4
        os4 += 1.0 * qk.Sz(i) * qk.Sz(j) + 0.5 * (qk.Sp(i) * qk.Sm(j) + qk.Sm(i) * qk.Sp(j))
    H4 = qk.MatrixFreeHamiltonian(qk.SpinHalfBasis(4), qk.SpinHalfSite(), os4, dtype=np.float64)
    r = qk.lanczos_ground_state(H4, 50, 1e-12)
    assert abs(r.energy + 2.0) < 1e-6 and r.converged and r.iterations > 0
    assert np.abs(H4.apply(r.eigenvector) - r.energy * r.eigenvector).max() < 1e-5
    lim = qk.lanczos_ground_state(H4, 2, 1e-15)
    assert lim.iterations == 2 and not lim.converged
    d = qk.davidson_lowest(H4, 2, 10, 1e-6)
    assert len(d.eigenvalues) == 2 and abs(d.eigenvalues[0] + 2.0) < 1e-5 and len(d.eigenvectors[0]) == 16
