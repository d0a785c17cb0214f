"""CPU oracles for the qkrylov H.x / Krylov path.  TEST INFRASTRUCTURE ONLY.

Two interchangeable back-ends expose the same small Python API:

* ``port()``  -- this project's C++ restatement (oracle/qk_oracle.cpp,
  built into oracle/liboracle.so by ``make -C oracle``).  Always available.
* ``ref()``   -- the qkrylov reference's own unchanged sources compiled
  against a minimal OpenMP Kokkos-API shim (oracle/_ref/liboracle_ref.so,
  built by ``make -C oracle ref`` where the reference checkout exists).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs use
this package, and only as the checker.

Problem descriptions are plain Python: ``kind`` in {"spin", "fermion",
"hubbard", "tj"}, a sector dict (keys of qkrylov's Sector struct:
use_sz, sz2, use_nup, nup, use_ndn, ndn, use_n, n, use_nb, nb) and a term
list ``[(coeff, [(op, site), ...]), ...]``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
KINDS = {"spin": 0, "fermion": 1, "hubbard": 2, "tj": 3}
SECTOR_KEYS = ("use_sz", "sz2", "use_nup", "nup", "use_ndn", "ndn", "use_n", "n", "use_nb", "nb")

_vp, _i, _d, _u64, _i64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_uint64, ctypes.c_int64


def build_port():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def build_ref(ref_dir=None):
    """Build oracle/_ref from a qkrylov reference checkout: ``ref_dir`` or
    the QKRYLOV_REFERENCE environment variable (no default path)."""
    ref_dir = ref_dir or os.environ.get("QKRYLOV_REFERENCE")
    if not ref_dir or not os.path.isdir(ref_dir):
        return False
    subprocess.run(["make", "-s", "-C", HERE, "ref", "-j8", f"REF={ref_dir}"], check=True)
    return True


def sector_array(sector=None):
    sector = sector or {}
    unknown = set(sector) - set(SECTOR_KEYS)
    if unknown:
        raise ValueError(f"unknown sector keys {unknown}")
    return (ctypes.c_int * 10)(*[int(sector.get(k, 0)) for k in SECTOR_KEYS])


def _flatten_terms(terms):
    coef = np.array([[complex(c).real, complex(c).imag] for c, _ in terms], dtype=np.float64).ravel()
    nfac = np.array([len(f) for _, f in terms], dtype=np.int32)
    names = [op.encode() for _, f in terms for op, _ in f]
    sites = np.array([s for _, f in terms for _, s in f], dtype=np.int32)
    return coef, nfac, (ctypes.c_char_p * max(len(names), 1))(*names), sites


class OracleError(RuntimeError):
    pass


class _Port:
    """Restatement back-end (oracle/qk_oracle.cpp)."""

    name = "port"

    def __init__(self):
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build_port()
        L = ctypes.CDLL(path)
        L.qko_last_error.restype = ctypes.c_char_p
        L.qko_site_apply.argtypes = [_i, ctypes.c_char_p, _i, _u64, _vp, _vp, _vp]
        L.qko_basis_count.restype = _i64
        L.qko_basis_count.argtypes = [_i, _i, _vp]
        L.qko_basis_states.argtypes = [_i, _i, _vp, _vp]
        L.qko_ham_create.restype = _vp
        L.qko_ham_create.argtypes = [_i, _i, _vp, _i, _vp, _vp, _vp, _vp]
        L.qko_ham_destroy.argtypes = [_vp]
        L.qko_ham_dim.restype = _u64
        L.qko_ham_dim.argtypes = [_vp]
        L.qko_ham_states.argtypes = [_vp, _vp]
        L.qko_ham_apply.argtypes = [_vp, _vp, _vp]
        L.qko_ham_coo_count.restype = _i64
        L.qko_ham_coo_count.argtypes = [_vp]
        L.qko_ham_coo.argtypes = [_vp, _vp, _vp, _vp]
        L.qko_ham_diagonal.argtypes = [_vp, _vp]
        L.qko_lanczos_start.argtypes = [_u64, _vp]
        L.qko_ftlm_vectors.argtypes = [_u64, _i, _vp]
        L.qko_lanczos.argtypes = [_vp, _i, _d, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]
        L.qko_davidson.argtypes = [_vp, _i, _i, _d, _vp, _vp, _vp, _vp, _vp]
        L.qko_cf.argtypes = [_vp, _vp, _i, _vp, _vp, _vp, _vp, _vp]
        L.qko_spectral.restype = _d
        L.qko_spectral.argtypes = [_vp, _vp, ctypes.c_size_t, _d, _d, _d, _d]
        L.qko_ftlm.argtypes = [_vp, _d, _i, _i, _vp, _vp, _vp]
        L.qko_ftlm_tridiag.argtypes = [_vp, _vp, _i, _vp, _vp, _vp, _vp]
        L.qko_tridiag_eig.argtypes = [_vp, _vp, _i, _vp, _vp]
        L.qko_jacobi_eig.argtypes = [_vp, _i, _vp, _vp]
        self.L = L

    def _err(self):
        raise OracleError(self.L.qko_last_error().decode())

    def site_apply(self, kind, op, site, state):
        v, ns, me = ctypes.c_int(), ctypes.c_uint64(), np.zeros(2)
        if self.L.qko_site_apply(KINDS[kind], op.encode(), site, state, ctypes.byref(v), ctypes.byref(ns), me.ctypes.data):
            self._err()
        return bool(v.value), int(ns.value), complex(me[0], me[1])

    def basis_states(self, kind, nsites, sector=None):
        sec = sector_array(sector)
        n = self.L.qko_basis_count(KINDS[kind], nsites, sec)
        if n < 0:
            self._err()
        out = np.zeros(n, dtype=np.uint64)
        self.L.qko_basis_states(KINDS[kind], nsites, sec, out.ctypes.data)
        return out

    def hamiltonian(self, kind, nsites, sector, terms):
        return _PortHam(self, kind, nsites, sector, terms)

    def lanczos_start(self, dim):
        v = np.zeros(dim, dtype=np.complex128)
        self.L.qko_lanczos_start(dim, v.ctypes.data)
        return v

    def ftlm_vectors(self, dim, n_random):
        v = np.zeros((n_random, dim), dtype=np.complex128)
        self.L.qko_ftlm_vectors(dim, n_random, v.ctypes.data)
        return v

    def spectral(self, alphas, betas, norm_phi0, omega, E0, eta=0.1):
        a = np.ascontiguousarray(alphas, dtype=np.float64)
        b = np.ascontiguousarray(np.concatenate([betas, [0.0]]), dtype=np.float64)
        return self.L.qko_spectral(a.ctypes.data, b.ctypes.data, len(a), norm_phi0, omega, E0, eta)

    def tridiag_eig(self, alphas, betas):
        a = np.ascontiguousarray(alphas, dtype=np.float64)
        b = np.ascontiguousarray(np.concatenate([betas, [0.0]]), dtype=np.float64)
        n = len(a)
        ev, fc = np.zeros(n), np.zeros(n)
        if self.L.qko_tridiag_eig(a.ctypes.data, b.ctypes.data, n, ev.ctypes.data, fc.ctypes.data):
            self._err()
        return ev, fc

    def jacobi_eig(self, H):
        H = np.ascontiguousarray(H, dtype=np.complex128)
        n = H.shape[0]
        ev, V = np.zeros(n), np.zeros((n, n), dtype=np.complex128)
        if self.L.qko_jacobi_eig(H.ctypes.data, n, ev.ctypes.data, V.ctypes.data):
            self._err()
        return ev, V


class _PortHam:
    def __init__(self, back, kind, nsites, sector, terms):
        self.back, self.L = back, back.L
        coef, nfac, names, sites = _flatten_terms(terms)
        self._keep = (coef, nfac, names, sites)
        self.h = self.L.qko_ham_create(KINDS[kind], nsites, sector_array(sector), len(terms),
                                       coef.ctypes.data, nfac.ctypes.data, names, sites.ctypes.data)
        if not self.h:
            back._err()
        self.dim = int(self.L.qko_ham_dim(self.h))

    def __del__(self):
        if getattr(self, "h", None):
            self.L.qko_ham_destroy(self.h)
            self.h = None

    def states(self):
        out = np.zeros(self.dim, dtype=np.uint64)
        self.L.qko_ham_states(self.h, out.ctypes.data)
        return out

    def apply(self, x):
        x = np.ascontiguousarray(x, dtype=np.complex128)
        y = np.zeros(self.dim, dtype=np.complex128)
        if self.L.qko_ham_apply(self.h, x.ctypes.data, y.ctypes.data):
            self.back._err()
        return y

    def apply_into(self, x, y):
        """y = H x into caller-owned complex128 arrays (no allocation here)."""
        assert x.dtype == y.dtype == np.complex128 and x.flags.c_contiguous and y.flags.c_contiguous
        if self.L.qko_ham_apply(self.h, x.ctypes.data, y.ctypes.data):
            self.back._err()
        return y

    def coo(self):
        n = self.L.qko_ham_coo_count(self.h)
        if n < 0:
            self.back._err()
        r, c, v = np.zeros(n, np.int64), np.zeros(n, np.int64), np.zeros(n, np.complex128)
        if self.L.qko_ham_coo(self.h, r.ctypes.data, c.ctypes.data, v.ctypes.data):
            self.back._err()
        return r, c, v

    def diagonal(self):
        d = np.zeros(self.dim, dtype=np.complex128)
        if self.L.qko_ham_diagonal(self.h, d.ctypes.data):
            self.back._err()
        return d

    def lanczos(self, maxiter=200, tol=1e-12, want_vector=True):
        e, it, cv, na, nb = _d(), _i(), _i(), _i(), _i()
        ev = np.zeros(self.dim, np.complex128) if want_vector else None
        a, b = np.zeros(max(maxiter, 1) + 1), np.zeros(max(maxiter, 1) + 1)
        if self.L.qko_lanczos(self.h, maxiter, tol, ctypes.byref(e), ctypes.byref(it), ctypes.byref(cv),
                              ev.ctypes.data if ev is not None else None, a.ctypes.data, b.ctypes.data,
                              ctypes.byref(na), ctypes.byref(nb)):
            self.back._err()
        return dict(energy=e.value, iterations=it.value, converged=bool(cv.value), eigenvector=ev,
                    alphas=a[:na.value].copy(), betas=b[:nb.value].copy())

    def davidson(self, n_eig=1, max_subspace=20, tol=1e-8):
        evals, evecs = np.zeros(n_eig), np.zeros((n_eig, self.dim), np.complex128)
        n, it, cv = _i(), _i(), _i()
        if self.L.qko_davidson(self.h, n_eig, max_subspace, tol, evals.ctypes.data, evecs.ctypes.data,
                               ctypes.byref(n), ctypes.byref(it), ctypes.byref(cv)):
            self.back._err()
        return dict(eigenvalues=evals[:n.value].copy(), eigenvectors=evecs[:n.value].copy(),
                    iterations=it.value, converged=bool(cv.value))

    def cf(self, phi0, n_iter=100):
        phi0 = np.ascontiguousarray(phi0, dtype=np.complex128)
        a, b = np.zeros(n_iter + 1), np.zeros(n_iter + 1)
        nrm, na, nb = _d(), _i(), _i()
        if self.L.qko_cf(self.h, phi0.ctypes.data, n_iter, a.ctypes.data, b.ctypes.data, ctypes.byref(nrm),
                         ctypes.byref(na), ctypes.byref(nb)):
            self.back._err()
        return dict(alphas=a[:na.value].copy(), betas=b[:nb.value].copy(), norm_phi0=nrm.value)

    def ftlm(self, beta, n_random=50, n_steps=100):
        Z, U, C = _d(), _d(), _d()
        if self.L.qko_ftlm(self.h, beta, n_random, n_steps, ctypes.byref(Z), ctypes.byref(U), ctypes.byref(C)):
            self.back._err()
        return dict(beta=beta, Z=Z.value, U=U.value, Cv=C.value)

    def ftlm_tridiag(self, v_start, n_steps):
        v = np.ascontiguousarray(v_start, dtype=np.complex128)
        a, b = np.zeros(n_steps + 1), np.zeros(n_steps + 1)
        na, nb = _i(), _i()
        if self.L.qko_ftlm_tridiag(self.h, v.ctypes.data, n_steps, a.ctypes.data, b.ctypes.data,
                                   ctypes.byref(na), ctypes.byref(nb)):
            self.back._err()
        return a[:na.value].copy(), b[:nb.value].copy()


class _Ref:
    """The reference's own sources (oracle/_ref/liboracle_ref.so)."""

    name = "ref"

    def __init__(self):
        path = os.path.join(HERE, "_ref", "liboracle_ref.so")
        if not os.path.exists(path) and not build_ref():
            raise FileNotFoundError("oracle/_ref/liboracle_ref.so is not built and the reference is absent")
        L = ctypes.CDLL(path)
        L.refb_last_error.restype = ctypes.c_char_p
        L.refb_basis_create.restype = _vp
        L.refb_basis_create.argtypes = [_i, _i, _vp]
        L.refb_basis_destroy.argtypes = [_vp]
        L.refb_basis_dim.restype = _u64
        L.refb_basis_dim.argtypes = [_vp]
        L.refb_basis_states.argtypes = [_vp, _vp]
        L.refb_basis_index.restype = _i64
        L.refb_basis_index.argtypes = [_vp, _u64]
        L.refb_site_apply.argtypes = [_i, ctypes.c_char_p, _i, _u64, _vp, _vp, _vp]
        L.refb_ham_create.restype = _vp
        L.refb_ham_create.argtypes = [_vp, _i, _i, _vp, _vp, _vp, _vp]
        L.refb_ham_destroy.argtypes = [_vp]
        L.refb_ham_dim.restype = _u64
        L.refb_ham_dim.argtypes = [_vp]
        L.refb_ham_nnz.restype = _u64
        L.refb_ham_nnz.argtypes = [_vp]
        L.refb_ham_csr.argtypes = [_vp, _vp, _vp, _vp]
        L.refb_ham_apply.argtypes = [_vp, _vp, _vp]
        L.refb_ham_diagonal.argtypes = [_vp, _vp]
        L.refb_lanczos.argtypes = [_vp, _i, _d, _vp, _vp, _vp, _vp]
        L.refb_davidson.argtypes = [_vp, _i, _i, _d, _vp, _vp, _vp, _vp, _vp]
        L.refb_cf.argtypes = [_vp, _vp, _i, _vp, _vp, _vp, _vp, _vp]
        L.refb_spectral.restype = _d
        L.refb_spectral.argtypes = [_vp, _vp, ctypes.c_size_t, _d, _d, _d, _d]
        L.refb_ftlm.argtypes = [_vp, _d, _i, _i, _vp, _vp, _vp]
        self.L = L

    def _err(self):
        raise OracleError(self.L.refb_last_error().decode())

    def site_apply(self, kind, op, site, state):
        v, ns, me = ctypes.c_int(), ctypes.c_uint64(), np.zeros(2)
        if self.L.refb_site_apply(KINDS[kind], op.encode(), site, state, ctypes.byref(v), ctypes.byref(ns), me.ctypes.data):
            self._err()
        return bool(v.value), int(ns.value), complex(me[0], me[1])

    def basis_states(self, kind, nsites, sector=None):
        b = self.L.refb_basis_create(KINDS[kind], nsites, sector_array(sector))
        if not b:
            self._err()
        try:
            out = np.zeros(self.L.refb_basis_dim(b), dtype=np.uint64)
            self.L.refb_basis_states(b, out.ctypes.data)
            return out
        finally:
            self.L.refb_basis_destroy(b)

    def hamiltonian(self, kind, nsites, sector, terms):
        return _RefHam(self, kind, nsites, sector, terms)

    def spectral(self, alphas, betas, norm_phi0, omega, E0, eta=0.1):
        a = np.ascontiguousarray(alphas, dtype=np.float64)
        b = np.ascontiguousarray(np.concatenate([betas, [0.0]]), dtype=np.float64)
        return self.L.refb_spectral(a.ctypes.data, b.ctypes.data, len(a), norm_phi0, omega, E0, eta)


class _RefHam:
    def __init__(self, back, kind, nsites, sector, terms):
        self.back, self.L = back, back.L
        self.b = self.L.refb_basis_create(KINDS[kind], nsites, sector_array(sector))
        if not self.b:
            back._err()
        coef, nfac, names, sites = _flatten_terms(terms)
        self._keep = (coef, nfac, names, sites)
        self.h = self.L.refb_ham_create(self.b, KINDS[kind], len(terms), coef.ctypes.data, nfac.ctypes.data,
                                        names, sites.ctypes.data)
        if not self.h:
            self.L.refb_basis_destroy(self.b)
            self.b = None
            back._err()
        self.dim = int(self.L.refb_ham_dim(self.h))

    def __del__(self):
        if getattr(self, "h", None):
            self.L.refb_ham_destroy(self.h)
        if getattr(self, "b", None):
            self.L.refb_basis_destroy(self.b)

    def states(self):
        out = np.zeros(self.dim, dtype=np.uint64)
        self.L.refb_basis_states(self.b, out.ctypes.data)
        return out

    def csr(self):
        nnz = self.L.refb_ham_nnz(self.h)
        rp, c, v = np.zeros(self.dim + 1, np.int32), np.zeros(nnz, np.int32), np.zeros(nnz, np.complex128)
        self.L.refb_ham_csr(self.h, rp.ctypes.data, c.ctypes.data, v.ctypes.data)
        return rp, c, v

    def coo(self):
        rp, c, v = self.csr()
        rows = np.repeat(np.arange(self.dim, dtype=np.int64), np.diff(rp))
        return rows, c.astype(np.int64), v

    def apply(self, x):
        x = np.ascontiguousarray(x, dtype=np.complex128)
        y = np.zeros(self.dim, dtype=np.complex128)
        if self.L.refb_ham_apply(self.h, x.ctypes.data, y.ctypes.data):
            self.back._err()
        return y

    def apply_into(self, x, y):
        """y = H x into caller-owned complex128 arrays (no allocation here)."""
        assert x.dtype == y.dtype == np.complex128 and x.flags.c_contiguous and y.flags.c_contiguous
        if self.L.refb_ham_apply(self.h, x.ctypes.data, y.ctypes.data):
            self.back._err()
        return y

    def diagonal(self):
        d = np.zeros(self.dim, dtype=np.complex128)
        self.L.refb_ham_diagonal(self.h, d.ctypes.data)
        return d

    def lanczos(self, maxiter=200, tol=1e-12, want_vector=True):
        e, it, cv = _d(), _i(), _i()
        ev = np.zeros(self.dim, np.complex128)
        if self.L.refb_lanczos(self.h, maxiter, tol, ctypes.byref(e), ctypes.byref(it), ctypes.byref(cv), ev.ctypes.data):
            self.back._err()
        return dict(energy=e.value, iterations=it.value, converged=bool(cv.value), eigenvector=ev)

    def davidson(self, n_eig=1, max_subspace=20, tol=1e-8):
        evals, evecs = np.zeros(n_eig), np.zeros((n_eig, self.dim), np.complex128)
        n, it, cv = _i(), _i(), _i()
        if self.L.refb_davidson(self.h, n_eig, max_subspace, tol, evals.ctypes.data, evecs.ctypes.data,
                                ctypes.byref(n), ctypes.byref(it), ctypes.byref(cv)):
            self.back._err()
        return dict(eigenvalues=evals[:n.value].copy(), eigenvectors=evecs[:n.value].copy(),
                    iterations=it.value, converged=bool(cv.value))

    def cf(self, phi0, n_iter=100):
        phi0 = np.ascontiguousarray(phi0, dtype=np.complex128)
        a, b = np.zeros(n_iter + 1), np.zeros(n_iter + 1)
        nrm, na, nb = _d(), _i(), _i()
        if self.L.refb_cf(self.h, phi0.ctypes.data, n_iter, a.ctypes.data, b.ctypes.data, ctypes.byref(nrm),
                          ctypes.byref(na), ctypes.byref(nb)):
            self.back._err()
        return dict(alphas=a[:na.value].copy(), betas=b[:nb.value].copy(), norm_phi0=nrm.value)

    def ftlm(self, beta, n_random=50, n_steps=100):
        Z, U, C = _d(), _d(), _d()
        if self.L.refb_ftlm(self.h, beta, n_random, n_steps, ctypes.byref(Z), ctypes.byref(U), ctypes.byref(C)):
            self.back._err()
        return dict(beta=beta, Z=Z.value, U=U.value, Cv=C.value)


_port = None
_ref = None


def port():
    global _port
    if _port is None:
        _port = _Port()
    return _port


def ref():
    global _ref
    if _ref is None:
        _ref = _Ref()
    return _ref


def have_ref():
    try:
        ref()
        return True
    except (FileNotFoundError, OSError):
        return False


# ------------------------------------------------------------ model builders
def heisenberg_chain(N, J=1.0, periodic=True):
    """Terms of the spin-1/2 Heisenberg chain in the order the reference's
    tests write them (tests/test_workflow.cpp:34-36): per bond Sz Sz, then
    0.5 Sp Sm, then 0.5 Sm Sp."""
    terms = []
    nb = N if periodic else N - 1
    for i in range(nb):
        j = (i + 1) % N
        terms += [(J, [("Sz", i), ("Sz", j)]), (0.5 * J, [("Sp", i), ("Sm", j)]), (0.5 * J, [("Sm", i), ("Sp", j)])]
    return terms


def j1j2_chain(N, J1=1.0, J2=0.0):
    terms = heisenberg_chain(N, J1)
    for i in range(N):
        j = (i + 2) % N
        terms += [(J2, [("Sz", i), ("Sz", j)]), (0.5 * J2, [("Sp", i), ("Sm", j)]), (0.5 * J2, [("Sm", i), ("Sp", j)])]
    return terms


def hubbard_square(Lx, Ly, t=1.0, U=4.0):
    """Periodic Lx x Ly Hubbard model, site = x + Lx*y.  Directed hops
    -t c+_i c_j written annihilator first ([C(j), Cdag(i)]: factors act in
    list order on the ket), both spins, both directions, then U Nupdn."""
    terms = []
    N = Lx * Ly
    bonds = set()
    for y in range(Ly):
        for x in range(Lx):
            i = x + Lx * y
            for j in ((x + 1) % Lx + Lx * y, x + Lx * ((y + 1) % Ly)):
                if i != j:
                    bonds.add((min(i, j), max(i, j)) if False else (i, j))
    for (i, j) in sorted(bonds):
        for (a, b) in ((i, j), (j, i)):
            terms.append((-t, [("CUp", b), ("CdagUp", a)]))
            terms.append((-t, [("CDn", b), ("CdagDn", a)]))
    for i in range(N):
        terms.append((U, [("Nupdn", i)]))
    return terms


def tj_chain(N, t=1.0, J=0.4):
    """Periodic t-J chain.  Hops as in hubbard_square (annihilator first);
    J (S_i.S_j - n_i n_j / 4) expanded into Nup/Ndn products and the two
    spin-flip four-fermion terms, with the factor order chosen so that the
    operator the reference computes (T^dagger per term, factors applied in
    list order) is the physical one."""
    terms = []
    for i in range(N):
        j = (i + 1) % N
        for (a, b) in ((i, j), (j, i)):
            terms.append((-t, [("CUp", b), ("CdagUp", a)]))
            terms.append((-t, [("CDn", b), ("CdagDn", a)]))
    for i in range(N):
        j = (i + 1) % N
        # Sz Sz - n n / 4 = -1/2 (nu_i nd_j + nd_i nu_j)
        terms.append((-0.5 * J, [("Nup", i), ("Ndn", j)]))
        terms.append((-0.5 * J, [("Ndn", i), ("Nup", j)]))
        # 1/2 (S+_i S-_j + S-_i S+_j), S+_i S-_j = c+_iu c_id c+_jd c_ju
        terms.append((0.5 * J, [("CUp", j), ("CdagDn", j), ("CDn", i), ("CdagUp", i)]))
        terms.append((0.5 * J, [("CUp", i), ("CdagDn", i), ("CDn", j), ("CdagUp", j)]))
    return terms
