"""The OpSum compiler (host C++) checked without a GPU.

The compiled tables (condition / flip / sign masks and one coefficient per
term, grouped by flip) are evaluated here in numpy on every basis state and
must give the reference's matrix bit for bit: the same entries, summed in
the reference's order, for every site family, complex coefficients,
n-body terms and sector-leaving terms.
"""
import numpy as np
import pytest

import oracle as O
import qkrylov_b200 as qk
from conftest import dense_from_coo, terms_from_golden
from test_sector_tables import make_basis

SITES = {"spin": qk.SpinHalfSite, "fermion": qk.FermionSite, "hubbard": qk.HubbardSite, "tj": qk.TJSite}


def opsum(terms):
    os_ = qk.OpSum(dtype=np.float64)
    for c, f in terms:
        os_.add_term(c, *[x for pair in f for x in pair])
    return os_


def popc(a):
    return np.array([bin(int(v)).count("1") for v in a])


def matrix_from_tables(B, info):
    """Column-by-column H from the compiled tables, evaluated per row."""
    st = B.states()
    dim = st.size
    M = np.zeros((dim, dim), dtype=np.complex128)
    mask, coef = info["mask"], info["coef"]
    for g in range(len(info["flip"])):
        f0, cnt = int(info["first"][g]), int(info["count"][g])
        acc = np.zeros(dim, np.complex128)
        any_ = np.zeros(dim, bool)
        for t in range(f0, f0 + cnt):
            ok = (st & mask[t, 0]) == mask[t, 1]
            sgn = np.where(popc(st & mask[t, 2]) % 2 == 1, -1.0, 1.0)
            acc = np.where(ok, acc + np.where(sgn < 0, -coef[t], coef[t]), acc)
            any_ |= ok
        tgt = st ^ info["flip"][g]
        col = B.index_many(tgt)
        rows = np.nonzero(any_ & (col >= 0))[0]
        if not info["check"][g]:
            assert np.all(col[any_] >= 0), "group marked always-in-sector left the sector"
        for r in rows:
            M[r, col[r]] += acc[r]
    return M


def test_golden_models_bit_exact(golden, golden_vecs):
    for name, m in golden["models"].items():
        if f"{name}/coo_rows" not in golden_vecs:
            continue
        B = make_basis(m["kind"], m["N"], m["sector"])
        info = qk.compile_info(B, SITES[m["kind"]](), opsum(terms_from_golden(m)))
        M = matrix_from_tables(B, info)
        R = dense_from_coo(golden_vecs[f"{name}/coo_rows"], golden_vecs[f"{name}/coo_cols"],
                           golden_vecs[f"{name}/coo_vals"], m["dim"])
        assert np.array_equal(M, R), name


OPS = {"spin": ["Sz", "Sp", "Sm", "Sx", "Sy"], "fermion": ["N", "Id", "C", "Cdag"],
       "hubbard": ["Nup", "Ndn", "Nupdn", "CUp", "CdagUp", "CDn", "CdagDn"],
       "tj": ["Nup", "Ndn", "CUp", "CdagUp", "CDn", "CdagDn"]}
SECS = {"spin": [(7, dict(use_sz=1, sz2=1)), (6, {})], "fermion": [(7, dict(use_n=1, n=3)), (5, {})],
        "hubbard": [(4, dict(use_nup=1, nup=2, use_ndn=1, ndn=1)), (3, {}), (4, dict(use_nup=1, nup=2))],
        "tj": [(5, dict(use_nup=1, nup=2, use_ndn=1, ndn=1)), (4, {}), (5, dict(use_ndn=1, ndn=2))]}


@pytest.mark.parametrize("kind", list(OPS))
@pytest.mark.parametrize("seed", range(6))
def test_random_opsums_match_oracle(kind, seed):
    rng = np.random.default_rng(100 * seed + len(kind))
    P = O.port()
    for N, sec in SECS[kind]:
        terms = []
        for _ in range(25):
            nf = int(rng.integers(1, 5))
            f = [(OPS[kind][int(rng.integers(len(OPS[kind])))], int(rng.integers(0, N + (1 if seed == 5 else 0))))
                 for _ in range(nf)]
            c = complex(rng.choice([1.0, -0.5, 0.25, 0.7]), rng.choice([0.0, 0.0, 0.3, -1.25]))
            terms.append((c, f))
        B = make_basis(kind, N, sec)
        info = qk.compile_info(B, SITES[kind](), opsum(terms))
        M = matrix_from_tables(B, info)
        H = P.hamiltonian(kind, N, sec, terms)
        r, c_, v = H.coo()
        assert np.array_equal(M, dense_from_coo(r, c_, v, H.dim)), (kind, N, sec)


def test_site_apply_matches_reference(golden):
    L = qk.lib()
    for a in golden["sites"]:
        sh = SITES[a["kind"]]()._handle()
        try:
            import ctypes
            v, ns, me = ctypes.c_int(), ctypes.c_uint64(), (ctypes.c_double * 2)()
            assert L.qkrylov_b200_site_apply(sh, a["op"].encode(), a["site"], a["state"], ctypes.byref(v),
                                             ctypes.byref(ns), me) == 0
            assert (bool(v.value), int(ns.value), complex(me[0], me[1])) == (a["valid"], a["new_state"],
                                                                             complex(*a["me"])), a
        finally:
            L.qkrylov_site_destroy(sh)


def test_unknown_operator_is_reported():
    B = qk.SpinHalfBasis(4)
    with pytest.raises(RuntimeError, match="Unknown spin operator: Foo"):
        qk.compile_info(B, qk.SpinHalfSite(), opsum([(1.0, [("Foo", 0)])]))
    with pytest.raises(RuntimeError, match="Unknown TJ operator: Nupdn"):
        qk.compile_info(qk.TJBasis(3), qk.TJSite(), opsum([(1.0, [("Nupdn", 0)])]))


def test_grouping_and_real_flags():
    B = qk.SpinHalfBasis(28, sz=0)
    info = qk.compile_info(B, qk.SpinHalfSite(), opsum(O.heisenberg_chain(28)))
    assert info["all_real"] and info["has_diag"]
    assert len(info["flip"]) == 1 + 28                  # diagonal + one target per bond
    assert int(info["count"][0]) == 28 and not info["check"].any()
