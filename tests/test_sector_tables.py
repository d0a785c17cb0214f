"""Product sector tables (two-level ranking) against the reference's bases.

Runs without a GPU: the tables are host data built by libqkrylov_b200.so.
States must come out in the reference's ascending order, bit for bit, and
index/contains must agree with it for members and non-members.
"""
import hashlib

import numpy as np
import pytest

import oracle as O
import qkrylov_b200 as qk


def make_basis(kind, N, sec):
    if kind == "spin":
        return qk.SpinHalfBasis(N, sz=sec["sz2"] / 2) if sec.get("use_sz") else qk.SpinHalfBasis(N)
    if kind == "fermion":
        return qk.FermionBasis(N, conserve_n=bool(sec.get("use_n")), n=sec.get("n", 0))
    cls = qk.HubbardBasis if kind == "hubbard" else qk.TJBasis
    return cls(N, conserve_nup=bool(sec.get("use_nup")), nup=sec.get("nup", 0),
               conserve_ndn=bool(sec.get("use_ndn")), ndn=sec.get("ndn", 0))


def test_golden_bases(golden):
    for b in golden["bases"]:
        B = make_basis(b["kind"], b["N"], b["sector"])
        st = B.states()
        assert B.size == b["dim"]
        assert hashlib.sha256(st.astype(np.uint64).tobytes()).hexdigest() == b["sha256"], b
        assert np.array_equal(B.index_many(st), np.arange(B.size))


CASES = [("spin", N, dict(use_sz=1, sz2=s)) for N in (1, 2, 5, 8, 13) for s in (-N, -1, 0, 1, 2, N)]
CASES += [("spin", N, {}) for N in (1, 7, 11)]
CASES += [("fermion", N, dict(use_n=1, n=n)) for N in (3, 9) for n in (0, 2, N)] + [("fermion", 6, {})]
CASES += [("hubbard", N, dict(use_nup=1, nup=u, use_ndn=1, ndn=d)) for N in (3, 5) for u in (0, 2) for d in (1, 3)]
CASES += [("hubbard", 5, dict(use_nup=1, nup=2)), ("hubbard", 4, dict(use_ndn=1, ndn=1)), ("hubbard", 3, {})]
CASES += [("tj", N, dict(use_nup=1, nup=u, use_ndn=1, ndn=d)) for N in (4, 7) for u in (0, 2) for d in (1, 3)]
CASES += [("tj", 6, dict(use_nup=1, nup=2)), ("tj", 6, dict(use_ndn=1, ndn=3)), ("tj", 5, {})]


@pytest.mark.parametrize("kind,N,sec", CASES)
def test_tables_match_oracle(kind, N, sec):
    ref = O.port().basis_states(kind, N, sec)
    B = make_basis(kind, N, sec)
    assert B.size == ref.size
    assert np.array_equal(B.states(), ref)
    nbits = 2 * N if kind in ("hubbard", "tj") else N
    cand = np.arange(min(1 << nbits, 1 << 16), dtype=np.uint64)
    got = B.index_many(cand)
    pos = np.searchsorted(ref, cand)
    if ref.size == 0:
        inside = np.zeros(cand.size, bool)
    else:
        inside = (pos < ref.size) & (ref[np.minimum(pos, ref.size - 1)] == cand)
    assert np.array_equal(got, np.where(inside, pos, -1))
    # states above the basis width are never members
    assert B.index_many(np.array([1 << nbits, (1 << 63) | 1], dtype=np.uint64)).tolist() == [-1, -1]


def test_large_sector_without_enumeration():
    # Heisenberg N=28, Sz=0 and t-J N=20 with 2 holes: the reference loops
    # over 2^28 / 2^40 integers; the tables give the same order directly.
    B = qk.SpinHalfBasis(28, sz=0)
    assert B.size == 40116600
    assert B.state(0) == (1 << 14) - 1 and B.state(B.size - 1) == ((1 << 14) - 1) << 14
    rng = np.random.default_rng(3)
    idx = rng.integers(0, B.size, 2000)
    st = np.array([B.state(int(i)) for i in idx], dtype=np.uint64)
    assert all(bin(int(s)).count("1") == 14 for s in st)
    assert np.array_equal(B.index_many(st), idx)
    srt = np.sort(idx)
    assert np.all(np.diff(np.array([B.state(int(i)) for i in srt], dtype=np.int64)) > 0)
    T = qk.TJBasis(20, nup=9, ndn=9)
    assert T.size == 9237800
    assert qk.HubbardBasis(16, nup=8, ndn=8).size == 165636900


def test_reference_errors():
    with pytest.raises(RuntimeError, match="1 <= N <= 63"):
        qk.SpinHalfBasis(0)
    with pytest.raises(RuntimeError, match="1 <= N <= 31"):
        qk.HubbardBasis(32)
    B = qk.SpinHalfBasis(4, sz=0)
    with pytest.raises(KeyError):
        B.index(0b1110)
    with pytest.raises(IndexError):
        B.state(6)
    assert qk.SpinHalfBasis(5, sz=0).size == 0  # 2*Sz parity mismatch: empty, as the reference
