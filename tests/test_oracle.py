"""The CPU oracle (oracle/qk_oracle.cpp) pinned against the reference.

Pins: the golden fixtures written by tests/golden/make_golden.py from the
reference's own sources, and the constants the reference's tests assert
(each cited).  When oracle/_ref is built (the reference checkout is
present) the restatement is also compared with it directly.
"""
import hashlib

import numpy as np
import pytest

import oracle as O
from conftest import dense_from_coo, terms_from_golden


@pytest.fixture(scope="module")
def P():
    return O.port()


def test_bases_match_reference_digests(P, golden):
    for b in golden["bases"]:
        st = P.basis_states(b["kind"], b["N"], b["sector"])
        assert st.size == b["dim"], b
        assert hashlib.sha256(st.astype(np.uint64).tobytes()).hexdigest() == b["sha256"], b


def test_site_actions_match_reference(P, golden):
    for a in golden["sites"]:
        v, ns, me = P.site_apply(a["kind"], a["op"], a["site"], a["state"])
        assert (v, ns, me) == (a["valid"], a["new_state"], complex(*a["me"])), a


def test_reference_site_known_answers(P):
    # tests/test_fermion_site.cpp:13-26
    assert P.site_apply("fermion", "N", 1, 0b1010) == (True, 0b1010, 1.0)
    assert P.site_apply("fermion", "N", 0, 0b1010)[2] == 0.0
    assert P.site_apply("fermion", "C", 1, 0b1010) == (True, 0b1000, 1.0)
    assert P.site_apply("fermion", "C", 3, 0b1010) == (True, 0b0010, -1.0)
    # tests/test_tj_site.cpp:13-18
    assert P.site_apply("tj", "CUp", 0, 0b01) == (True, 0, 1.0)
    assert P.site_apply("tj", "CdagDn", 0, 0b01)[0] is False
    with pytest.raises(O.OracleError, match="Unknown spin operator: Foo"):
        P.site_apply("spin", "Foo", 0, 0)


def test_reference_basis_dims(P):
    assert P.basis_states("spin", 4, dict(use_sz=1, sz2=0)).size == 6    # tests/test_c_api.cpp:23
    assert P.basis_states("fermion", 4).size == 16                        # tests/test_fermion_basis.cpp:10-12
    assert P.basis_states("fermion", 4, dict(use_n=1, n=2)).size == 6     # tests/test_fermion_basis.cpp:18-20
    assert P.basis_states("tj", 2).size == 9                              # tests/test_tj_basis.cpp:12-14
    assert P.basis_states("spin", 16, dict(use_sz=1, sz2=0)).size == 12870


def test_coo_matches_reference_csr(P, golden, golden_vecs):
    for name, m in golden["models"].items():
        if f"{name}/coo_rows" not in golden_vecs:
            continue
        H = P.hamiltonian(m["kind"], m["N"], m["sector"], terms_from_golden(m))
        r, c, v = H.coo()
        assert np.array_equal(r, golden_vecs[f"{name}/coo_rows"]), name
        assert np.array_equal(c, golden_vecs[f"{name}/coo_cols"]), name
        assert np.array_equal(v, golden_vecs[f"{name}/coo_vals"]), name


def test_reference_pinned_energies(P):
    h4 = []
    for i in range(3):
        h4 += [(1.0, [("Sz", i), ("Sz", i + 1)]), (0.5, [("Sp", i), ("Sm", i + 1)]), (0.5, [("Sm", i), ("Sp", i + 1)])]
    e = P.hamiltonian("spin", 4, dict(use_sz=1, sz2=0), h4).lanczos()["energy"]
    assert abs(e - (-1.6160254038)) < 1e-5                                      # tests/test_workflow.cpp:46-48
    assert abs(P.hamiltonian("spin", 2, {}, O.heisenberg_chain(2, periodic=False)).lanczos()["energy"] + 0.75) < 1e-5  # tests/test_lanczos_ritz.cpp:45-46
    assert abs(P.hamiltonian("spin", 4, {}, O.heisenberg_chain(4)).lanczos(50, 1e-12)["energy"] + 2.0) < 1e-6  # bindings/julia/test/runtests.jl:164-166
    H3 = P.hamiltonian("spin", 3, {}, [(1.0, [("Sz", 0), ("Sz", 1)]), (0.5, [("Sz", 0), ("Sz", 1), ("Sz", 2)])])
    x = np.zeros(8, complex)
    x[7] = 1.0
    assert abs(H3.apply(x)[7] - 0.3125) < 1e-6                                  # bindings/julia/test/runtests.jl:102-106
    lim = P.hamiltonian("spin", 4, {}, O.heisenberg_chain(4)).lanczos(2, 1e-15)
    assert lim["iterations"] == 2 and not lim["converged"]                     # bindings/julia/test/runtests.jl:172-175


def test_solvers_match_golden(P, golden, golden_vecs):
    for name, m in golden["models"].items():
        terms = terms_from_golden(m) if "terms" in m else O.heisenberg_chain(m["N"])
        H = P.hamiltonian(m["kind"], m["N"], m["sector"], terms)
        lz = H.lanczos(200, 1e-12)
        ref = m["lanczos"]
        assert abs(lz["energy"] - ref["energy"]) <= 1e-12 * max(1.0, abs(ref["energy"])), name
        assert lz["iterations"] == ref["iterations"] and lz["converged"] == ref["converged"], name
        if f"{name}/lanczos_vec" in golden_vecs:
            assert np.abs(lz["eigenvector"] - golden_vecs[f"{name}/lanczos_vec"]).max() < 1e-8, name
        if "ftlm" in m:
            for f in m["ftlm"]:
                got = H.ftlm(f["beta"], 5 if name != "heis12_sz0" else 4, 20 if name != "heis12_sz0" else 30)
                for k in ("Z", "U", "Cv"):
                    assert abs(got[k] - f[k]) <= 1e-10 * max(1.0, abs(f[k])), (name, k)


def test_ftlm_and_cf_on_heis12(P, golden, golden_vecs):
    """Continued fraction for S(q=pi, w) at N=12.

    The three-term recurrence runs without reorthogonalisation, so its
    coefficients past the first steps depend on rounding order: the
    reference itself, run with 1 and with 8 OpenMP threads, differs by 1e-8
    at step 10 and O(1) at step 39.  Parity is therefore asserted on the
    early coefficients and on the spectral function, which is stable."""
    m = golden["models"]["heis12_sz0"]
    H = P.hamiltonian("spin", 12, m["sector"], O.heisenberg_chain(12))
    cf = H.cf(golden_vecs["heis12_sz0/phi_szpi"], 40)
    n = len(m["cf_szpi"]["alphas"])
    assert len(cf["alphas"]) == n
    assert np.allclose(cf["alphas"][:6], m["cf_szpi"]["alphas"][:6], rtol=0, atol=1e-12)
    assert np.allclose(cf["betas"][:6], m["cf_szpi"]["betas"][:6], rtol=0, atol=1e-12)
    E0 = m["lanczos"]["energy"]
    S_ref = np.array(m["spectral"]["S"])
    S = np.array([P.spectral(cf["alphas"], cf["betas"], cf["norm_phi0"], w, E0, 0.05) for w in m["spectral"]["omega"]])
    assert np.abs(S - S_ref).max() <= 1e-10 * np.abs(S_ref).max()
    S_same = [P.spectral(m["cf_szpi"]["alphas"], m["cf_szpi"]["betas"], m["cf_szpi"]["norm_phi0"], w, E0, 0.05)
              for w in m["spectral"]["omega"]]
    assert np.allclose(S_same, S_ref, rtol=1e-13, atol=1e-13)


@pytest.mark.skipif(not O.have_ref(), reason="reference build (oracle/_ref) not available")
def test_restatement_equals_reference_build():
    P, R = O.port(), O.ref()
    rng = np.random.default_rng(7)
    for kind, N, sec, terms in [("spin", 12, dict(use_sz=1, sz2=0), O.j1j2_chain(12, 1.0, 0.37)),
                                ("hubbard", 6, dict(use_nup=1, nup=3, use_ndn=1, ndn=3), O.hubbard_square(3, 2)),
                                ("tj", 8, dict(use_nup=1, nup=3, use_ndn=1, ndn=3), O.tj_chain(8))]:
        hp, hr = P.hamiltonian(kind, N, sec, terms), R.hamiltonian(kind, N, sec, terms)
        x = rng.standard_normal(hp.dim) + 1j * rng.standard_normal(hp.dim)
        assert np.array_equal(hp.apply(x), hr.apply(x))
        assert abs(hp.lanczos()["energy"] - hr.lanczos()["energy"]) < 1e-12 * hp.dim


def test_tj_model_is_the_physical_operator(P):
    """The t-J OpSum (annihilator-first hops, J expanded) gives the physical
    H = -t sum c+c + J sum (S.S - n n / 4): checked against a direct
    construction on the same basis at N=6, 2 holes."""
    N, t, J = 6, 1.0, 0.4
    sec = dict(use_nup=1, nup=2, use_ndn=1, ndn=2)
    H = P.hamiltonian("tj", N, sec, O.tj_chain(N, t, J))
    st = H.states()
    idx = {int(s): i for i, s in enumerate(st)}
    D = np.zeros((len(st), len(st)))
    for a, s in enumerate(st):
        s = int(s)
        for i in range(N):
            j = (i + 1) % N
            for (p, q) in ((i, j), (j, i)):       # c+_p c_q, both spins
                for off in (0, 1):
                    bp, bq = 2 * p + off, 2 * q + off
                    if not (s >> bq) & 1 or (s >> (2 * p)) & 1 or (s >> (2 * p + 1)) & 1:
                        continue
                    sg = (-1) ** bin(s & ((1 << bq) - 1)).count("1")
                    s1 = s & ~(1 << bq)
                    sg *= (-1) ** bin(s1 & ((1 << bp) - 1)).count("1")
                    s2 = s1 | (1 << bp)
                    D[idx[s2], a] += -t * sg
            nu = lambda x, k: (x >> (2 * k)) & 1
            nd = lambda x, k: (x >> (2 * k + 1)) & 1
            szi, szj = 0.5 * (nu(s, i) - nd(s, i)), 0.5 * (nu(s, j) - nd(s, j))
            ni, nj = nu(s, i) + nd(s, i), nu(s, j) + nd(s, j)
            D[a, a] += J * (szi * szj - ni * nj / 4)
            for (p, q) in ((i, j), (j, i)):       # 1/2 S+_p S-_q
                if nd(s, p) and nu(s, q):
                    s2 = s & ~(1 << (2 * p + 1)) | (1 << (2 * p))
                    s2 = s2 & ~(1 << (2 * q)) | (1 << (2 * q + 1))
                    # fermion sign of c+_pu c_pd c+_qd c_qu on the JW ordering
                    ops = [("a", 2 * q), ("c", 2 * q + 1), ("a", 2 * p + 1), ("c", 2 * p)]
                    x, sg = s, 1
                    for kind_, b in ops:
                        sg *= (-1) ** bin(x & ((1 << b) - 1)).count("1")
                        x = x & ~(1 << b) if kind_ == "a" else x | (1 << b)
                    assert x == s2
                    D[idx[s2], a] += 0.5 * J * sg
    r, c, v = H.coo()
    M = dense_from_coo(r, c, v, len(st))
    assert np.allclose(M, D, atol=1e-14)
