"""qkrylov_b200: qkrylov's matrix-free H.x and Krylov solvers on NVIDIA B200.

Python mirror of qkrylov's Python API (bindings/python/qkrylov/*.py: same
class and function names, argument meaning and errors) over this project's
C ABI, libqkrylov_b200.so (include/qkrylov_c_api.h, include/qkrylov_b200.h).
All numerical work runs in the CUDA library; this module only marshals
arguments.  ``dtype=np.float64`` selects the double-precision path (the
reference's fp64 C++ namespace), ``np.float32`` the single-precision one
(the reference's C ABI and default Python dtype).
"""
from __future__ import annotations

import ctypes
import enum
import os
from typing import List, Optional, Sequence, Tuple, Union

import numpy as np

from ._lib import lib, LibraryError  # noqa: F401

__all__ = [
    "Op", "OpSum", "Sz", "Sp", "Sm", "Sx", "Sy", "CdagUp", "CUp", "CdagDn", "CDn", "Nup", "Ndn", "Nupdn",
    "Bdag", "B", "N", "Site", "SpinHalfSite", "FermionSite", "HubbardSite", "TJSite", "Basis", "SpinHalfBasis",
    "FermionBasis", "HubbardBasis", "TJBasis", "MatrixFreeHamiltonian", "LanczosResult", "lanczos_ground_state",
    "DavidsonResult", "davidson_lowest", "DynamicsResult", "continued_fraction_coeffs",
    "evaluate_spectral_function", "FTLMResult", "ftlm", "ftlm_sweep", "find_gpu", "gpu_count",
]

DTYPE_C128, DTYPE_C64, DTYPE_F64, DTYPE_F32 = 0, 1, 2, 3


def _check(rc, what):
    if rc == -1:
        raise ValueError(f"{what}: invalid argument ({lib().qkrylov_b200_last_error().decode()})")
    if rc != 0:
        raise RuntimeError(f"{what}: {lib().qkrylov_b200_last_error().decode()}")


# ----------------------------------------------------------------- operators
class Op(str, enum.Enum):
    Sz = "Sz"; Sp = "Sp"; Sm = "Sm"; Sx = "Sx"; Sy = "Sy"
    CdagUp = "CdagUp"; CUp = "CUp"; CdagDn = "CdagDn"; CDn = "CDn"
    Nup = "Nup"; Ndn = "Ndn"; Nupdn = "Nupdn"; Bdag = "Bdag"; B = "B"; N = "N"


class LocalOpExpr:
    def __init__(self, name: str, site: int):
        self.name, self.site = name, site

    def __mul__(self, other):
        if isinstance(other, LocalOpExpr):
            return TermExpr(1.0, [self, other])
        if isinstance(other, (int, float, complex)):
            return TermExpr(complex(other), [self])
        return NotImplemented

    def __rmul__(self, other):
        if isinstance(other, (int, float, complex)):
            return TermExpr(complex(other), [self])
        return NotImplemented


class TermExpr:
    def __init__(self, coeff, ops):
        self.coeff, self.ops = coeff, ops

    def __mul__(self, other):
        if isinstance(other, LocalOpExpr):
            return TermExpr(self.coeff, self.ops + [other])
        if isinstance(other, TermExpr):
            return TermExpr(self.coeff * other.coeff, self.ops + other.ops)
        if isinstance(other, (int, float, complex)):
            return TermExpr(self.coeff * complex(other), self.ops)
        return NotImplemented

    def __rmul__(self, other):
        if isinstance(other, (int, float, complex)):
            return TermExpr(self.coeff * complex(other), self.ops)
        return NotImplemented

    def __add__(self, other):
        if isinstance(other, TermExpr):
            return OpSumExpr([self, other])
        if isinstance(other, OpSumExpr):
            return OpSumExpr([self] + other.terms)
        return NotImplemented

    def __sub__(self, other):
        if isinstance(other, TermExpr):
            return OpSumExpr([self, TermExpr(-other.coeff, other.ops)])
        return NotImplemented


class OpSumExpr:
    def __init__(self, terms):
        self.terms = terms

    def __add__(self, other):
        if isinstance(other, TermExpr):
            return OpSumExpr(self.terms + [other])
        if isinstance(other, OpSumExpr):
            return OpSumExpr(self.terms + other.terms)
        return NotImplemented

    def __mul__(self, other):
        if isinstance(other, (int, float, complex)):
            return OpSumExpr([t * other for t in self.terms])
        return NotImplemented

    __rmul__ = __mul__

    def __sub__(self, other):
        if isinstance(other, TermExpr):
            return OpSumExpr(self.terms + [TermExpr(-other.coeff, other.ops)])
        if isinstance(other, OpSumExpr):
            return OpSumExpr(self.terms + [TermExpr(-t.coeff, t.ops) for t in other.terms])
        return NotImplemented


def Sz(i): return LocalOpExpr("Sz", i)
def Sp(i): return LocalOpExpr("Sp", i)
def Sm(i): return LocalOpExpr("Sm", i)
def Sx(i): return LocalOpExpr("Sx", i)
def Sy(i): return LocalOpExpr("Sy", i)
def CdagUp(i): return LocalOpExpr("CdagUp", i)
def CUp(i): return LocalOpExpr("CUp", i)
def CdagDn(i): return LocalOpExpr("CdagDn", i)
def CDn(i): return LocalOpExpr("CDn", i)
def Nup(i): return LocalOpExpr("Nup", i)
def Ndn(i): return LocalOpExpr("Ndn", i)
def Nupdn(i): return LocalOpExpr("Nupdn", i)
def Bdag(i): return LocalOpExpr("Bdag", i)
def B(i): return LocalOpExpr("B", i)
def N(i): return LocalOpExpr("N", i)


class OpSum:
    """Ordered list of terms (coeff, [(op, site), ...]); factors act in list order."""

    def __init__(self, dtype=np.float32):
        self.dtype = dtype
        self.terms: List[Tuple[complex, List[Tuple[str, int]]]] = []

    def add_term(self, coeff: complex, *ops: Union[str, Op, int]):
        if len(ops) % 2 != 0:
            raise ValueError("Operators must be provided in (name, site) pairs.")
        factors = []
        for i in range(0, len(ops), 2):
            name = ops[i].value if isinstance(ops[i], Op) else str(ops[i])
            factors.append((name, int(ops[i + 1])))
        if not factors:
            raise ValueError("Term must be a tuple of (coeff, op1, site1, ...)")
        self.terms.append((complex(coeff), factors))

    def __iadd__(self, term):
        if isinstance(term, tuple):
            if len(term) < 3 or len(term) % 2 == 0:
                raise ValueError("Term must be a tuple of (coeff, op1, site1, ...)")
            self.add_term(term[0], *term[1:])
        elif isinstance(term, TermExpr):
            self.terms.append((complex(term.coeff), [(o.name, o.site) for o in term.ops]))
        elif isinstance(term, OpSumExpr):
            for t in term.terms:
                self.__iadd__(t)
        else:
            raise ValueError("Unsupported type for += on OpSum")
        return self

    def clear(self):
        self.terms.clear()

    @property
    def size(self) -> int:
        return len(self.terms)

    def _handle(self):
        L = lib()
        h = L.qkrylov_opsum_create()
        for c, f in self.terms:
            names = (ctypes.c_char_p * len(f))(*[n.encode() for n, _ in f])
            sites = (ctypes.c_int * len(f))(*[s for _, s in f])
            if self.dtype == np.float32:
                c = complex(np.float32(c.real), np.float32(c.imag))  # the reference's float coefficients
            _check(L.qkrylov_opsum_add_term_nbody_f64(h, c.real, c.imag, len(f), names, sites), "OpSum")
        return h

    def __repr__(self):
        return f"OpSum(terms={self.size})"


# --------------------------------------------------------------------- sites
class Site:
    family = -1

    def __init__(self, dtype=np.float32):
        self.dtype = dtype

    def _handle(self):
        L = lib()
        return {0: L.qkrylov_spinhalf_site_create, 1: L.qkrylov_fermion_site_create,
                2: L.qkrylov_hubbard_site_create, 3: L.qkrylov_tj_site_create}[self.family]()


class SpinHalfSite(Site):
    """Spin-1/2 site: Sz, Sp, Sm, Sx, Sy."""
    family = 0


class FermionSite(Site):
    """Spinless fermion mode: N, Id, C, Cdag."""
    family = 1


class HubbardSite(Site):
    """Hubbard site: Nup, Ndn, Nupdn, CUp, CdagUp, CDn, CdagDn."""
    family = 2


class TJSite(Site):
    """t-J site: as Hubbard without double occupancy (no Nupdn)."""
    family = 3


# --------------------------------------------------------------------- bases
class Basis:
    family = -1

    def __init__(self, N: int, sector: Optional[dict] = None, dtype=np.float32):
        self._N, self._sector, self.dtype = N, dict(sector or {}), dtype
        L = lib()
        sec = L.qkrylov_sector_create()
        try:
            s = self._sector
            if s.get("use_sz"):
                _check(L.qkrylov_sector_set_sz(sec, int(s.get("sz2", 0))), "sector")
            if s.get("use_n"):
                _check(L.qkrylov_sector_set_n(sec, int(s.get("n", 0))), "sector")
            self._h = self._create(L, N, sec)
        finally:
            L.qkrylov_sector_destroy(sec)
        if not self._h:
            raise RuntimeError(L.qkrylov_b200_last_error().decode())

    def _create(self, L, N, sec):
        raise NotImplementedError

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                lib().qkrylov_basis_destroy(h)
            except Exception:  # interpreter shutdown: the library is already gone
                pass
            self._h = None

    @property
    def size(self) -> int:
        return int(lib().qkrylov_basis_dimension(self._h))

    @property
    def nsites(self) -> int:
        return self._N

    def states(self, first: int = 0, count: Optional[int] = None) -> np.ndarray:
        count = self.size - first if count is None else count
        out = np.zeros(count, dtype=np.uint64)
        _check(lib().qkrylov_basis_states(self._h, first, count, out.ctypes.data), "basis states")
        return out

    def state(self, i: int) -> int:
        if i < 0 or i >= self.size:
            raise IndexError("basis index out of range")
        return int(lib().qkrylov_basis_state(self._h, i))

    def index(self, s: int) -> int:
        r = int(lib().qkrylov_basis_index(self._h, s))
        if r < 0:
            raise KeyError("State not present in basis")
        return r

    def contains(self, s: int) -> bool:
        return bool(lib().qkrylov_basis_contains(self._h, s))

    def index_many(self, states) -> np.ndarray:
        s = np.ascontiguousarray(states, dtype=np.uint64)
        out = np.zeros(s.size, dtype=np.int64)
        _check(lib().qkrylov_basis_index_many(self._h, s.ctypes.data, s.size, out.ctypes.data), "index")
        return out


class SpinHalfBasis(Basis):
    """Spin-1/2 chain; ``sz`` (total Sz) selects a sector as in qkrylov."""
    family = 0

    def __init__(self, N: int, conserve_sz: bool = False, sz: Optional[float] = None, dtype=np.float32):
        if sz is not None:
            conserve_sz = True
        else:
            sz = 0
        sec = {"use_sz": True, "sz2": int(2 * sz)} if conserve_sz else {}
        self._conserve_sz, self._sz = conserve_sz, sz
        super().__init__(N, sec, dtype)

    def _create(self, L, N, sec):
        return L.qkrylov_spinhalf_basis_create(N, sec)

    def __repr__(self):
        return f"SpinHalfBasis(N={self.nsites}, dim={self.size}" + (f", sz={self._sz})" if self._conserve_sz else ")")


class FermionBasis(Basis):
    family = 1

    def __init__(self, N: int, conserve_n: bool = False, n: int = 0, dtype=np.float32):
        if n != 0:
            conserve_n = True
        super().__init__(N, {"use_n": True, "n": n} if conserve_n else {}, dtype)

    def _create(self, L, N, sec):
        return L.qkrylov_fermion_basis_create(N, sec)


class _PairBasis(Basis):
    def __init__(self, N, conserve_nup=False, nup=0, conserve_ndn=False, ndn=0, dtype=np.float32):
        if nup != 0:
            conserve_nup = True
        if ndn != 0:
            conserve_ndn = True
        self._pairs = (conserve_nup, nup, conserve_ndn, ndn)
        super().__init__(N, {}, dtype)

    def _create(self, L, N, sec):
        cu, nu, cd, nd = self._pairs
        # The C ABI sets both counts together (c_api.cpp:80-91); a single
        # conserved species goes through the extended sector setters.
        if cu or cd:
            _check(L.qkrylov_sector_set_hubbard_particles(sec, nu, nd), "sector")
            if not (cu and cd):
                _check(L.qkrylov_b200_sector_set_species(sec, int(cu), int(cd)), "sector")
        return self._ctor(L)(N, sec)


class HubbardBasis(_PairBasis):
    family = 2

    def _ctor(self, L):
        return L.qkrylov_hubbard_basis_create


class TJBasis(_PairBasis):
    family = 3

    def _ctor(self, L):
        return L.qkrylov_tj_basis_create


# --------------------------------------------------------------- Hamiltonian
class MatrixFreeHamiltonian:
    """y = H x generated on the fly on the GPU from (basis, site, ops)."""

    def __init__(self, basis: Basis, site: Site, ops: OpSum, device: str = "cuda", dtype=np.float32):
        self.basis, self.site, self.ops, self.device, self.dtype = basis, site, ops, device, dtype
        dev = device.lower()
        if dev == "cpu":
            raise ValueError("qkrylov_b200 has no CPU back-end; use device='cuda'")
        dev_id = int(dev.split(":")[1]) if ":" in dev else 0
        L = lib()
        sh, oh = site._handle(), ops._handle()
        try:
            self._h = L.qkrylov_hamiltonian_create_ex(basis._h, sh, oh, 64 if dtype == np.float64 else 32, dev_id)
        finally:
            L.qkrylov_site_destroy(sh)
            L.qkrylov_opsum_destroy(oh)
        if not self._h:
            raise RuntimeError(L.qkrylov_b200_last_error().decode())

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                lib().qkrylov_hamiltonian_destroy(h)
            except Exception:  # interpreter shutdown: the library is already gone
                pass
            self._h = None

    @property
    def dimension(self) -> int:
        return int(lib().qkrylov_hamiltonian_dimension(self._h))

    @property
    def cdtype(self):
        return np.complex128 if self.dtype == np.float64 else np.complex64

    @property
    def all_real(self) -> bool:
        return bool(lib().qkrylov_hamiltonian_all_real(self._h))

    def apply(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=self.cdtype)
        if x.shape != (self.dimension,):
            raise ValueError("Input array size does not match Hamiltonian dimension")
        y = np.zeros_like(x)
        if self.dtype == np.float64:
            _check(lib().qkrylov_hamiltonian_apply_complex_f64(self._h, x.ctypes.data, y.ctypes.data), "apply")
        else:
            _check(lib().qkrylov_hamiltonian_apply_complex(self._h, x.ctypes.data, y.ctypes.data), "apply")
        return y

    __matmul__ = apply

    def diagonal(self) -> np.ndarray:
        d = np.zeros(self.dimension, dtype=np.complex128)
        _check(lib().qkrylov_hamiltonian_diagonal_complex_f64(self._h, d.ctypes.data), "diagonal")
        return d.astype(self.cdtype)

    def apply_device(self, x_ptr: int, y_ptr: int, dtype: int, stream: int = 0):
        """y = H x on device pointers (e.g. torch ``tensor.data_ptr()``), no sync."""
        _check(lib().qkrylov_hamiltonian_apply_device(self._h, dtype, ctypes.c_void_p(x_ptr),
                                                      ctypes.c_void_p(y_ptr), ctypes.c_void_p(stream or None)),
               "apply_device")

    def apply_block_device(self, X_ptr: int, Y_ptr: int, dtype: int, R: int, lanes_per_row: int = 0,
                           dots: bool = False, stream: int = 0):
        """Y = H X for R row-interleaved vectors (element (i, r) at X[i*R + r])
        on device pointers; returns the 2R column dots <X_r, Y_r> (re, im
        interleaved) when dots, else None (no sync)."""
        out = np.zeros(2 * R) if dots else None
        _check(lib().qkrylov_b200_apply_block_device(self._h, dtype, int(R), int(lanes_per_row), ctypes.c_void_p(X_ptr),
                                                     ctypes.c_void_p(Y_ptr), out.ctypes.data if dots else None,
                                                     ctypes.c_void_p(stream or None)), "apply_block_device")
        return out

    def block_shape_timings(self, precision: int = 64, R: int = 64) -> np.ndarray:
        """The block apply's autotuner table for this operator: fastest timed
        launch in ms, rows = lanes per row 32, 16, 8, columns = CTA tiles of
        256, 128, 512 rows; 0 where not timed (the tuner runs on the first
        batched FTLM or sweep with this precision and block size)."""
        dt = {64: DTYPE_F64, 32: DTYPE_F32}[precision]
        out = np.zeros(9)
        _check(lib().qkrylov_b200_block_shape_timings(self._h, dt, int(R), out.ctypes.data), "block_shape_timings")
        return out.reshape(3, 3)

    @property
    def kernel(self) -> str:
        """The H.x kernel this operator uses: 'spin-exchange' (two-site
        exchange in a single-charge sector), 'spin-product' (Hubbard-type
        operators with N_up and N_dn conserved: hops of one species applied
        as T_up x 1 + 1 x T_dn in the (up, down) order), 'two-part' (any
        operator whose terms factorise over the sector split: Hubbard, t-J,
        fermions) or 'generic' (term-table walk)."""
        return {1: "spin-exchange", 2: "two-part", 3: "spin-product"}.get(
            int(lib().qkrylov_hamiltonian_kernel(self._h)), "generic")

    @property
    def stream(self) -> int:
        return int(lib().qkrylov_hamiltonian_stream(self._h) or 0)

    def __repr__(self):
        return f"MatrixFreeHamiltonian(dim={self.dimension})"


# ------------------------------------------------------------------- solvers
class LanczosResult:
    def __init__(self, energy, eigenvector, iterations=0, converged=False, alphas=None, betas=None):
        self.energy, self.eigenvector = energy, eigenvector
        self.iterations, self.converged = iterations, converged
        self.alphas = np.zeros(0) if alphas is None else alphas
        self.betas = np.zeros(0) if betas is None else betas

    def __repr__(self):
        return f"LanczosResult(energy={self.energy:.10f})"


def lanczos_ground_state(H: MatrixFreeHamiltonian, maxiter: int = 200, tol: float = 1e-12,
                         start: Optional[np.ndarray] = None) -> LanczosResult:
    L = lib()
    dim = H.dimension
    if H.dtype == np.float64:
        res = _LanczosF64()
        ev = np.zeros(dim, dtype=np.complex128)
        a, b = np.zeros(max(maxiter, 1)), np.zeros(max(maxiter, 1))
        st = None if start is None else np.ascontiguousarray(start, dtype=np.complex128)
        _check(L.qkrylov_lanczos_ground_state_f64(H._h, maxiter, tol, st.ctypes.data if st is not None else None,
                                                  ctypes.byref(res), ev.ctypes.data, a.ctypes.data, b.ctypes.data),
               "lanczos_ground_state")
        return LanczosResult(res.energy, ev, res.iterations, bool(res.converged), a[:res.n_alpha].copy(),
                             b[:res.n_beta].copy())
    if start is not None:
        raise ValueError("a start vector needs dtype=np.float64")
    res = _LanczosC()
    ev = np.zeros(dim, dtype=np.complex64)
    _check(L.qkrylov_lanczos_ground_state_complex(H._h, maxiter, ctypes.c_float(tol), ctypes.byref(res),
                                                  ev.ctypes.data), "lanczos_ground_state")
    return LanczosResult(float(res.energy), ev, res.iterations, bool(res.converged))


class MixedLanczosResult:
    """Result of lanczos_mixed / lanczos_fp64: energy, explicit FP64 residual
    ||H psi - E psi|| / |E|, iterations per phase, wall seconds per phase and
    the per-step trace (iteration, Ritz value, seconds since the start)."""

    def __init__(self, r, trace, eigenvector):
        self.energy, self.residual = r.energy, r.residual
        self.iterations_low, self.iterations_high = r.iterations_low, r.iterations_high
        self.seconds_low, self.seconds_high = r.seconds_low, r.seconds_high
        self.seconds = r.seconds_low + r.seconds_high
        self.restarts, self.converged = r.restarts, bool(r.converged)
        self.trace, self.eigenvector = trace, eigenvector

    def __repr__(self):
        return (f"MixedLanczosResult(energy={self.energy:.15g}, residual={self.residual:.2e}, "
                f"iterations={self.iterations_low}+{self.iterations_high}, seconds={self.seconds:.4f})")


def _two_phase(fn, H, seed, start, start_device, maxiter, tol, want_vector, low):
    L = lib()
    dim = H.dimension
    real = bool(L.qkrylov_hamiltonian_all_real(H._h))
    sdt = (np.float32 if real else np.complex64) if low else (np.float64 if real else np.complex128)
    odt = np.float64 if real else np.complex128
    sp, on_dev = None, 0
    if start_device is not None:
        sp, on_dev = int(start_device), 1
    elif start is not None:
        st = np.ascontiguousarray(start, dtype=sdt)
        if st.size != dim:
            raise ValueError("start vector has the wrong length")
        sp = st.ctypes.data
    psi = np.empty(dim, dtype=odt) if want_vector else None
    cap = 8 * max(maxiter, 1) + 8
    ti, te, ts = np.zeros(cap, np.int32), np.zeros(cap), np.zeros(cap)
    r = _MixedC()
    _check(fn(H._h, ctypes.c_uint64(seed), sp, on_dev, maxiter, tol, ctypes.byref(r),
              psi.ctypes.data if psi is not None else None, cap, ti.ctypes.data, te.ctypes.data, ts.ctypes.data),
           "lanczos_mixed" if low else "lanczos_fp64")
    n = r.trace_len
    trace = list(zip(ti[:n].tolist(), te[:n].tolist(), ts[:n].tolist()))
    return MixedLanczosResult(r, trace, psi)


def lanczos_mixed(H: MatrixFreeHamiltonian, seed: int = 0, start: Optional[np.ndarray] = None,
                  maxiter: int = 200, tol: float = 1e-10, start_device: Optional[int] = None,
                  eigenvector: bool = False, reorth: str = "partial") -> MixedLanczosResult:
    """FP32-vector Lanczos (FP64 scalars) followed by FP64 refinement until the
    explicit residual ||H psi - E psi|| / |E| <= tol.  `start`: host FP32
    vector (float32 for real operators, complex64 otherwise), or
    `start_device`: a device pointer to one; neither: GPU random start.
    `reorth`: "partial" (Simon's partial reorthogonalisation inside the FP32
    passes) or "full" (every step against all the pass's vectors)."""
    fns = {"partial": "qkrylov_b200_lanczos_mixed", "full": "qkrylov_b200_lanczos_mixed_full"}
    if reorth not in fns:
        raise ValueError('reorth must be "partial" or "full"')
    return _two_phase(getattr(lib(), fns[reorth]), H, seed, start, start_device, maxiter, tol, eigenvector, True)


def lanczos_fp64(H: MatrixFreeHamiltonian, seed: int = 0, start: Optional[np.ndarray] = None,
                 maxiter: int = 200, tol: float = 1e-10, start_device: Optional[int] = None,
                 eigenvector: bool = False) -> MixedLanczosResult:
    """Plain FP64 Lanczos with lanczos_mixed's stopping rule (the baseline of
    time-to-E0 comparisons); `start` is float64 / complex128."""
    return _two_phase(lib().qkrylov_b200_lanczos_fp64, H, seed, start, start_device, maxiter, tol, eigenvector,
                      False)


class FTLMBlockResult:
    """Thermodynamics at each temperature (log Z, U, Cv arrays) plus timing:
    seconds (whole call), seconds_device (the Lanczos steps), the autotuned
    block H.X shape (lanes_per_row) and whether a CUDA graph ran."""

    def __init__(self, temps, logZ, U, Cv, info):
        self.temperatures, self.logZ, self.U, self.Cv = temps, logZ, U, Cv
        self.seconds, self.seconds_device = info.seconds, info.seconds_device
        self.e_min, self.lanes_per_row, self.graph = info.e_min, info.lanes_per_row, bool(info.graph)
        self.vectors, self.steps = info.vectors, info.steps

    def __repr__(self):
        return (f"FTLMBlockResult(vectors={self.vectors}, steps={self.steps}, seconds={self.seconds:.3f}, "
                f"lanes_per_row={self.lanes_per_row}, graph={self.graph})")


def _ftlm_call(fn, H, temps, extra):
    T = np.ascontiguousarray(temps, dtype=np.float64)
    lz, u, cv = np.zeros(T.size), np.zeros(T.size), np.zeros(T.size)
    info = _FTLMInfo()
    _check(fn(H._h, *extra[0], T.size, T.ctypes.data, lz.ctypes.data, u.ctypes.data, cv.ctypes.data, *extra[1],
              ctypes.byref(info)), "ftlm")
    return FTLMBlockResult(T, lz, u, cv, info)


def ftlm_block(H: MatrixFreeHamiltonian, temperatures: Sequence[float], n_random: int = 64, n_steps: int = 100,
               seed: int = 0, precision: int = 32, graph: bool = True) -> FTLMBlockResult:
    """Batched FTLM: n_random (32/64/128) Rademacher vectors as one block,
    n_steps Lanczos steps (one block H.X each, CUDA graph), Z/U/Cv at every
    temperature.  precision 32: FP32 vectors with FP64 dots; 64: FP64."""
    return _ftlm_call(lib().qkrylov_b200_ftlm_block, H, temperatures,
                      ((precision, n_random, n_steps, ctypes.c_uint64(seed)), (int(graph),)))


def ftlm_loop(H: MatrixFreeHamiltonian, temperatures: Sequence[float], n_random: int = 64, n_steps: int = 100,
              seed: int = 0, precision: int = 64, n_vectors: Optional[int] = None) -> FTLMBlockResult:
    """The same random vectors as ftlm_block run one at a time (the first
    n_vectors of them; all by default)."""
    nv = n_random if n_vectors is None else n_vectors
    return _ftlm_call(lib().qkrylov_b200_ftlm_loop, H, temperatures,
                      ((precision, n_random, n_steps, ctypes.c_uint64(seed), nv), ()))


class WarmStartMLP:
    """Learned warm start for spin-1/2 ground states: an MLP (spins as +-1
    and the coupling J2 -> 128 -> 128 -> log-amplitude, sign logit; GELU;
    BF16 weights, FP32 accumulation) trained on the GPU by the library's own
    kernels on ground states added with add_target, whose start vector
    M(s) exp(o0) tanh(o1) (M: Marshall's sign rule) seeds Lanczos at new
    couplings (lanczos_warm)."""

    def __init__(self, basis: "SpinHalfBasis", seed: int = 0, device: int = 0):
        self._basis = basis
        self._h = lib().qkrylov_b200_mlp_create(basis._h, device, ctypes.c_uint64(seed))
        if not self._h:
            raise RuntimeError(lib().qkrylov_b200_last_error().decode())

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                lib().qkrylov_b200_mlp_destroy(h)
            except Exception:
                pass
            self._h = None

    @property
    def n_params(self) -> int:
        return int(lib().qkrylov_b200_mlp_num_params(self._h))

    @property
    def params(self) -> np.ndarray:
        p = np.zeros(self.n_params, np.float32)
        _check(lib().qkrylov_b200_mlp_get_params(self._h, p.ctypes.data), "mlp params")
        return p

    @params.setter
    def params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.n_params:
            raise ValueError("parameter vector has the wrong size")
        _check(lib().qkrylov_b200_mlp_set_params(self._h, p.ctypes.data), "mlp params")

    def add_target(self, j2: float, psi: np.ndarray):
        psi = np.ascontiguousarray(np.real(psi), dtype=np.float64)
        if psi.size != self._basis.size:
            raise ValueError("target state has the wrong length")
        _check(lib().qkrylov_b200_mlp_add_target(self._h, float(j2), psi.ctypes.data), "mlp target")

    def train(self, steps: int = 1000, batch: int = 8192, lr: float = 1e-3, seed: int = 0,
              c_sign: float = 1.0) -> np.ndarray:
        loss = np.zeros(max(steps, 1))
        _check(lib().qkrylov_b200_mlp_train(self._h, steps, batch, lr, ctypes.c_uint64(seed), c_sign,
                                            loss.ctypes.data), "mlp train")
        return loss[:steps]

    def set_tensor_cores(self, on: bool = True):
        """Inference on the tensor cores (tcgen05, BF16 activations; default)
        or on the CUDA cores (FP32 activations, as in training)."""
        _check(lib().qkrylov_b200_mlp_set_tensor_cores(self._h, int(bool(on))), "mlp tensor cores")

    def start_vector(self, j2: float) -> np.ndarray:
        out = np.zeros(self._basis.size, np.float32)
        _check(lib().qkrylov_b200_mlp_start_vector(self._h, float(j2), out.ctypes.data, 0), "mlp start vector")
        return out

    def loss_grad(self, states, j2, targets, c_sign: float = 1.0):
        st = np.ascontiguousarray(states, dtype=np.uint64)
        j = np.ascontiguousarray(np.broadcast_to(np.asarray(j2, np.float64), st.shape), dtype=np.float64)
        tg = np.ascontiguousarray(targets, dtype=np.float32)
        if tg.shape != (st.size, 3):
            raise ValueError("targets must be (n, 3): log-amplitude, sign, weight")
        g = np.zeros(self.n_params, np.float32)
        loss = ctypes.c_double()
        _check(lib().qkrylov_b200_mlp_loss_grad(self._h, st.size, st.ctypes.data, j.ctypes.data, tg.ctypes.data,
                                                c_sign, g.ctypes.data, ctypes.byref(loss)), "mlp loss")
        return loss.value, g


def lanczos_warm(H: MatrixFreeHamiltonian, net: WarmStartMLP, j2: float, maxiter: int = 200,
                 tol: float = 1e-10) -> MixedLanczosResult:
    """lanczos_mixed started from the network's start vector at j2 (built on
    the GPU; its time is part of the result's seconds and is also given as
    seconds_inference)."""
    r = _MixedC()
    tinf = ctypes.c_double()
    _check(lib().qkrylov_b200_lanczos_warm(H._h, net._h, float(j2), maxiter, tol, ctypes.byref(r),
                                           ctypes.byref(tinf)), "lanczos_warm")
    out = MixedLanczosResult(r, [], None)
    out.seconds_inference = tinf.value
    return out


class DavidsonBlockResult:
    def __init__(self, evals, resid, evecs, info):
        self.eigenvalues, self.residuals, self.eigenvectors = evals, resid, evecs
        self.iterations, self.applies, self.restarts = info.iterations, info.applies, info.restarts
        self.converged, self.seconds = bool(info.converged), info.seconds

    def __repr__(self):
        return (f"DavidsonBlockResult(eigenvalues={self.eigenvalues}, iterations={self.iterations}, "
                f"applies={self.applies}, seconds={self.seconds:.3f})")


def davidson_block(H: MatrixFreeHamiltonian, n_eig: int = 4, block: int = 8, max_subspace: int = 64,
                   tol: float = 1e-8, seed: int = 0, maxiter: int = 200, precision: int = 64,
                   eigenvectors: bool = False) -> DavidsonBlockResult:
    """Block Davidson on real vectors for real operators: n_eig lowest
    eigenpairs with `block` corrections per iteration, diagonal
    preconditioner, basis of at most max_subspace vectors, seeded random
    start block; converged at residual norms < tol."""
    ev, rs = np.zeros(n_eig), np.zeros(n_eig)
    vec = np.zeros((n_eig, H.dimension)) if eigenvectors else None
    info = _DavidsonBlockInfo()
    _check(lib().qkrylov_b200_davidson_block(H._h, precision, n_eig, block, max_subspace, tol, ctypes.c_uint64(seed),
                                             maxiter, ev.ctypes.data, rs.ctypes.data,
                                             vec.ctypes.data if vec is not None else None, ctypes.byref(info)),
           "davidson_block")
    return DavidsonBlockResult(ev, rs, vec, info)


class SweepResult:
    def __init__(self, energies, residuals, converged, info):
        self.energies, self.residuals, self.converged = energies, residuals, converged
        self.block, self.steps, self.passes = info.block, info.steps, info.passes
        self.applies, self.lanes_per_row, self.seconds = info.applies, info.lanes_per_row, info.seconds
        self.seconds_inference = info.seconds_inference

    def __repr__(self):
        return (f"SweepResult({len(self.energies)} couplings, steps={self.steps}, passes={self.passes}, "
                f"seconds={self.seconds:.3f})")


def lanczos_sweep(H0: MatrixFreeHamiltonian, H1: MatrixFreeHamiltonian, couplings: Sequence[float],
                  tol: float = 1e-10, pass_len: int = 64, max_passes: int = 16, seed: int = 1,
                  net: Optional["WarmStartMLP"] = None) -> SweepResult:
    """Ground states of H0 + g H1 for every g in `couplings` (at most 128)
    at once: one FP64 block of Lanczos recurrences (one column per
    coupling, partial reorthogonalisation, restarts from the Ritz vector
    after pass_len steps) until every explicit residual |H psi - E psi| / |E|
    is <= tol.  H0 and H1: real operators on the same basis.  net: a
    WarmStartMLP on that basis whose coupling input is g; each column then
    starts from the network's start vector (random starts without one)."""
    g = np.ascontiguousarray(couplings, dtype=np.float64)
    n = len(g)
    e, r, cv = np.zeros(n), np.zeros(n), np.zeros(n, dtype=np.int32)
    info = _SweepInfo()
    _check(lib().qkrylov_b200_lanczos_sweep(H0._h, H1._h, n, g.ctypes.data, pass_len, max_passes, tol,
                                            ctypes.c_uint64(seed), net._h if net is not None else None,
                                            e.ctypes.data, r.ctypes.data, cv.ctypes.data, ctypes.byref(info)),
           "lanczos_sweep")
    return SweepResult(e, r, cv.astype(bool), info)


class DavidsonResult:
    def __init__(self, eigenvalues, eigenvectors, iterations=0, converged=False):
        self.eigenvalues, self.eigenvectors = eigenvalues, eigenvectors
        self.iterations, self.converged = iterations, converged

    def __repr__(self):
        return f"DavidsonResult(energies={self.eigenvalues})"


def davidson_lowest(H: MatrixFreeHamiltonian, n_eig: int = 1, max_subspace: int = 20,
                    tol: float = 1e-8) -> DavidsonResult:
    L = lib()
    dim = H.dimension
    k = max(1, min(n_eig, dim))
    info = _DavidsonInfo()
    if H.dtype == np.float64:
        ev, vec = np.zeros(k), np.zeros((k, dim), dtype=np.complex128)
        _check(L.qkrylov_davidson_lowest_f64(H._h, n_eig, max_subspace, tol, ev.ctypes.data, vec.ctypes.data,
                                             ctypes.byref(info)), "davidson_lowest")
    else:
        ev, vec = np.zeros(k, dtype=np.float32), np.zeros((k, dim), dtype=np.complex64)
        _check(L.qkrylov_davidson_lowest_complex(H._h, n_eig, max_subspace, ctypes.c_float(tol), ev.ctypes.data,
                                                 vec.ctypes.data, ctypes.byref(info)), "davidson_lowest")
    return DavidsonResult(ev.astype(float), list(vec), info.iterations, bool(info.converged))


class DynamicsResult:
    def __init__(self, alphas, betas, norm_phi0):
        self.alphas, self.betas, self.norm_phi0 = np.asarray(alphas), np.asarray(betas), norm_phi0


def continued_fraction_coeffs(H: MatrixFreeHamiltonian, phi0: Optional[np.ndarray], n_iter: int = 100,
                              save: Optional[str] = None, resume: Optional[str] = None) -> DynamicsResult:
    """The reference's continued_fraction_coeffs.  With `save` and/or
    `resume` (directories; FP64 operators only) the run writes / continues
    a checkpoint of its state (.npy files: alphas, betas, norm_phi0, state,
    v, v_prev); `n_iter` counts all steps, a resumed run matches an
    uninterrupted one bit for bit."""
    L = lib()
    if save is not None or resume is not None:
        if H.dtype != np.float64:
            raise ValueError("checkpointed continued fractions run on FP64 operators")
        p = None if resume is not None else np.ascontiguousarray(phi0, dtype=np.complex128)
        if p is not None and p.shape != (H.dimension,):
            raise ValueError("phi0 vector size does not match Hamiltonian dimension")
        a, b = np.zeros(n_iter), np.zeros(n_iter)
        nrm, na, nb = ctypes.c_double(), ctypes.c_int(), ctypes.c_int()
        if save is not None:
            os.makedirs(save, exist_ok=True)
        _check(L.qkrylov_b200_cf_checkpointed(H._h, p.ctypes.data if p is not None else None,
                                              resume.encode() if resume is not None else None, n_iter,
                                              save.encode() if save is not None else None, a.ctypes.data,
                                              b.ctypes.data, ctypes.byref(nrm), ctypes.byref(na), ctypes.byref(nb)),
               "continued_fraction_coeffs")
        return DynamicsResult(a[:na.value].copy(), b[:nb.value].copy(), nrm.value)
    phi0 = np.ascontiguousarray(phi0, dtype=H.cdtype)
    if phi0.shape != (H.dimension,):
        raise ValueError("phi0 vector size does not match Hamiltonian dimension")
    if H.dtype == np.float64:
        a, b = np.zeros(n_iter), np.zeros(n_iter)
        nrm, na, nb = ctypes.c_double(), ctypes.c_int(), ctypes.c_int()
        _check(L.qkrylov_continued_fraction_coeffs_f64(H._h, phi0.ctypes.data, n_iter, a.ctypes.data, b.ctypes.data,
                                                       ctypes.byref(nrm), ctypes.byref(na), ctypes.byref(nb)),
               "continued_fraction_coeffs")
        return DynamicsResult(a[:na.value].copy(), b[:nb.value].copy(), nrm.value)
    a, b = np.zeros(n_iter, np.float32), np.zeros(n_iter, np.float32)
    nrm, nc = ctypes.c_float(), ctypes.c_int()
    _check(L.qkrylov_continued_fraction_coeffs_complex(H._h, phi0.ctypes.data, n_iter, a.ctypes.data, b.ctypes.data,
                                                       ctypes.byref(nrm), ctypes.byref(nc)),
           "continued_fraction_coeffs")
    n = nc.value
    return DynamicsResult(a[:n].copy(), b[:max(n - 1, 0)].copy(), nrm.value)


def cf_block(H: MatrixFreeHamiltonian, start, n_steps: int = 100, precision: int = 64, graph: bool = True,
             n_vectors: Optional[int] = None, complex_vectors: bool = False) -> List[DynamicsResult]:
    """continued_fraction_coeffs for many start vectors at once (one block
    of three-term recurrences on the GPU).  start: a host array of shape
    (dimension, k) (k <= 128 columns; padded with zero columns to a block of
    32, 64 or 128; a complex array selects complex vectors), or a device
    pointer (int) to a row-interleaved block of n_vectors columns (complex
    when complex_vectors or the operator is complex).  Returns one
    DynamicsResult per column."""
    L = lib()
    if not isinstance(start, int) and np.iscomplexobj(start):
        complex_vectors = True
    real = H.all_real and not complex_vectors
    if isinstance(start, int):
        if n_vectors not in (32, 64, 128):
            raise ValueError("n_vectors must be 32, 64 or 128 for a device start block")
        R, k, ptr, keep = n_vectors, n_vectors, start, None
        on_dev = 1
    else:
        a = np.asarray(start)
        if a.ndim != 2 or a.shape[0] != H.dimension or not 1 <= a.shape[1] <= 128:
            raise ValueError("start must have shape (dimension, k) with 1 <= k <= 128")
        k = a.shape[1]
        R = 32 if k <= 32 else 64 if k <= 64 else 128
        dt = (np.float32 if precision == 32 else np.float64) if real else \
            (np.complex64 if precision == 32 else np.complex128)
        keep = np.zeros((H.dimension, R), dtype=dt)
        keep[:, :k] = a
        ptr, on_dev = keep.ctypes.data, 0
    al, be = np.zeros((R, n_steps)), np.zeros((R, n_steps))
    nr, ln = np.zeros(R), np.zeros(R, dtype=np.int32)
    info = _FTLMInfo()
    _check(L.qkrylov_b200_cf_block(H._h, precision, int(complex_vectors), R, n_steps, ptr, on_dev, int(graph), al.ctypes.data,
                                   be.ctypes.data, nr.ctypes.data, ln.ctypes.data, ctypes.byref(info)), "cf_block")
    out = []
    for r in range(k):
        if nr[r] < 1e-15:  # the reference returns an empty fraction for a zero start vector
            out.append(DynamicsResult(np.zeros(0), np.zeros(0), 0.0))
            continue
        n = int(ln[r])
        nb = n if (n == n_steps and be[r, n - 1] >= 1e-15) else n - 1
        out.append(DynamicsResult(al[r, :n].copy(), be[r, :max(nb, 0)].copy(), float(nr[r])))
    return out


def evaluate_spectral_function(res: DynamicsResult, omega: float, E0: float, eta: float = 0.1) -> float:
    a = np.ascontiguousarray(res.alphas, dtype=np.float64)
    b = np.ascontiguousarray(res.betas, dtype=np.float64)
    if len(a) == 0:
        return 0.0
    return lib().qkrylov_evaluate_spectral_function_f64(a.ctypes.data, b.ctypes.data if len(b) else None, len(a),
                                                        res.norm_phi0, omega, E0, eta)


def spectral_function_batch(results, omegas, E0: float, eta: float = 0.1, device: int = 0) -> np.ndarray:
    """evaluate_spectral_function for many continued fractions at many
    frequencies in one GPU call.  `results`: a DynamicsResult or a sequence
    of them (fractions of different lengths allowed).  Returns S with shape
    (len(omegas),) for one result, (len(results), len(omegas)) otherwise."""
    single = isinstance(results, DynamicsResult)
    rs = [results] if single else list(results)
    w = np.ascontiguousarray(omegas, dtype=np.float64)
    ld = max([len(r.alphas) for r in rs] + [1])
    A = np.zeros((len(rs), ld))
    Bt = np.zeros((len(rs), ld))
    lens = np.zeros(len(rs), dtype=np.int32)
    nrm = np.zeros(len(rs))
    for c, r in enumerate(rs):
        n = len(r.alphas)
        A[c, :n] = r.alphas
        nb = min(len(r.betas), max(n - 1, 0))
        Bt[c, :nb] = np.asarray(r.betas, dtype=np.float64)[:nb]
        lens[c] = n
        nrm[c] = r.norm_phi0
    out = np.zeros((len(rs), len(w)))
    _check(lib().qkrylov_b200_spectral_function_batch(device, len(rs), ld, A.ctypes.data, Bt.ctypes.data,
                                                      lens.ctypes.data, nrm.ctypes.data, len(w), w.ctypes.data,
                                                      E0, eta, out.ctypes.data), "spectral_function_batch")
    return out[0] if single else out


def apply_operator(basis: "Basis", site: "Site", ops: "OpSum", x, expectation: bool = False, device: int = 0):
    """y = O x for the operator an OpSum defines on `basis` (the reference's
    H.x convention), without keeping a Hamiltonian.  `x`: a numpy vector
    (copied to the GPU and back; complex128, or float64 for a real
    operator) or a torch CUDA tensor (used in place; the result is a tensor
    of the same dtype).  With expectation=True also returns <x|O x>."""
    codes = {"complex128": DTYPE_C128, "complex64": DTYPE_C64, "float64": DTYPE_F64, "float32": DTYPE_F32}
    is_torch = hasattr(x, "data_ptr")
    if is_torch:
        import torch
        xt = x.contiguous()
        code = codes[str(xt.dtype).replace("torch.", "")]
    else:
        import torch
        xa = np.ascontiguousarray(x)
        if xa.dtype not in (np.complex128, np.float64):
            xa = xa.astype(np.complex128)
        xt = torch.from_numpy(xa).to(f"cuda:{device}")
        code = codes[str(xa.dtype)]
    yt = torch.empty_like(xt)
    e = np.zeros(2)
    _check(lib().qkrylov_b200_apply_operator(basis._h, site._handle(), ops._handle(), device, code,
                                             ctypes.c_void_p(xt.data_ptr()), ctypes.c_void_p(yt.data_ptr()),
                                             e.ctypes.data if expectation else None), "apply_operator")
    y = yt if is_torch else yt.cpu().numpy()
    return (y, complex(e[0], e[1])) if expectation else y


def save_result(path: str, result) -> None:
    """Store a ground-state or Davidson result under `path` (a directory)
    with the dataset names of the reference's examples/hdf5_storage.py:5-13
    (energy and eigenvector; eigenvalues and eigenvector_<i>), one .npy file
    per dataset (h5py is not a dependency of this package)."""
    os.makedirs(path, exist_ok=True)
    if hasattr(result, "eigenvalues"):
        np.save(os.path.join(path, "eigenvalues.npy"), np.asarray(result.eigenvalues, dtype=np.float64))
        for i, v in enumerate(getattr(result, "eigenvectors", None) or []):
            np.save(os.path.join(path, f"eigenvector_{i}.npy"), np.asarray(v))
    else:
        np.save(os.path.join(path, "energy.npy"), np.float64(result.energy))
        if getattr(result, "eigenvector", None) is not None:
            np.save(os.path.join(path, "eigenvector.npy"), np.asarray(result.eigenvector))


def load_result(path: str) -> dict:
    """The datasets save_result wrote, as a dict of numpy values."""
    out = {}
    for f in sorted(os.listdir(path)):
        if f.endswith(".npy"):
            v = np.load(os.path.join(path, f))
            out[f[:-4]] = v.item() if v.shape == () else v
    return out


class FTLMResult:
    def __init__(self, beta, Z, U, Cv):
        self.beta, self.partition_function, self.internal_energy, self.specific_heat = beta, Z, U, Cv


def ftlm_sweep(H: MatrixFreeHamiltonian, betas: Sequence[float], n_random: int = 50, n_steps: int = 100):
    b = np.ascontiguousarray(betas, dtype=np.float64)
    Z, U, C = np.zeros(len(b)), np.zeros(len(b)), np.zeros(len(b))
    _check(lib().qkrylov_ftlm_sweep_f64(H._h, len(b), b.ctypes.data, n_random, n_steps, Z.ctypes.data,
                                        U.ctypes.data, C.ctypes.data), "ftlm")
    return [FTLMResult(float(b[q]), Z[q], U[q], C[q]) for q in range(len(b))]


def ftlm(H: MatrixFreeHamiltonian, beta: float, n_random: int = 50, n_steps: int = 100) -> FTLMResult:
    if H.dtype == np.float64:
        return ftlm_sweep(H, [beta], n_random, n_steps)[0]
    r = _FTLMC()
    _check(lib().qkrylov_ftlm(H._h, ctypes.c_float(beta), n_random, n_steps, ctypes.byref(r)), "ftlm")
    return FTLMResult(r.beta, r.partition_function, r.internal_energy, r.specific_heat)


def die_count():
    """(dies, SMs on die 0, SMs on die 1) of the current device as the row
    kernels' topology probe measured them; (1, 0, 0) where it saw one die."""
    a, b = ctypes.c_int(0), ctypes.c_int(0)
    n = lib().qkrylov_b200_die_count(ctypes.byref(a), ctypes.byref(b))
    return int(n), a.value, b.value


def set_kernel_policy(policy: str):
    """'auto' (the specialised row kernels where the operator has their
    tables, per-die work queues on a two-die GPU), 'generic' (the term-walk
    kernel only), 'no-die-queues' (auto with one grid-stride order) or
    'no-spin-product' (auto with Hubbard-type operators on the two-part row
    kernel), for comparisons."""
    codes = {"auto": 0, "generic": 1, "no-die-queues": 2, "no-spin-product": 3}
    _check(lib().qkrylov_b200_set_kernel_policy(codes[policy]), "set_kernel_policy")


def find_gpu():
    return "cuda" if gpu_count() > 0 else None


def gpu_count() -> int:
    return int(lib().qkrylov_b200_device_count())


def compile_info(basis: Basis, site: Site, ops: OpSum) -> dict:
    """The OpSum compiler's bit-mask tables for (basis, site, ops), no GPU needed."""
    L = lib()
    sh, oh = site._handle(), ops._handle()
    try:
        nt, ng, hd, ar = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(L.qkrylov_opsum_compile(basis._h, sh, oh, ctypes.byref(nt), ctypes.byref(ng), ctypes.byref(hd),
                                       ctypes.byref(ar), None, None, None, None, None, None), "compile")
        mask = np.zeros((nt.value, 3), np.uint64)
        coef = np.zeros(nt.value, np.complex128)
        flip = np.zeros(ng.value, np.uint64)
        first, count, check = (np.zeros(ng.value, np.uint32) for _ in range(3))
        _check(L.qkrylov_opsum_compile(basis._h, sh, oh, None, None, None, None, mask.ctypes.data, coef.ctypes.data,
                                       flip.ctypes.data, first.ctypes.data, count.ctypes.data, check.ctypes.data),
               "compile")
        return dict(mask=mask, coef=coef, flip=flip, first=first, count=count, check=check,
                    has_diag=bool(hd.value), all_real=bool(ar.value))
    finally:
        L.qkrylov_site_destroy(sh)
        L.qkrylov_opsum_destroy(oh)


class _LanczosF64(ctypes.Structure):
    _fields_ = [("energy", ctypes.c_double), ("iterations", ctypes.c_int), ("converged", ctypes.c_int),
                ("n_alpha", ctypes.c_int), ("n_beta", ctypes.c_int)]


class _LanczosC(ctypes.Structure):
    _fields_ = [("energy", ctypes.c_float), ("iterations", ctypes.c_int), ("converged", ctypes.c_int)]


class _DavidsonBlockInfo(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("applies", ctypes.c_int), ("restarts", ctypes.c_int),
                ("converged", ctypes.c_int), ("seconds", ctypes.c_double)]


class _SweepInfo(ctypes.Structure):
    _fields_ = [("block", ctypes.c_int), ("steps", ctypes.c_int), ("passes", ctypes.c_int), ("applies", ctypes.c_int),
                ("lanes_per_row", ctypes.c_int), ("seconds", ctypes.c_double), ("seconds_inference", ctypes.c_double)]


class _FTLMInfo(ctypes.Structure):
    _fields_ = [("seconds", ctypes.c_double), ("seconds_device", ctypes.c_double), ("e_min", ctypes.c_double),
                ("lanes_per_row", ctypes.c_int), ("graph", ctypes.c_int), ("vectors", ctypes.c_int),
                ("steps", ctypes.c_int)]


class _MixedC(ctypes.Structure):
    _fields_ = [("energy", ctypes.c_double), ("residual", ctypes.c_double), ("seconds_low", ctypes.c_double),
                ("seconds_high", ctypes.c_double), ("iterations_low", ctypes.c_int),
                ("iterations_high", ctypes.c_int), ("restarts", ctypes.c_int), ("converged", ctypes.c_int),
                ("trace_len", ctypes.c_int)]


class _DavidsonInfo(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("converged", ctypes.c_int)]


class _FTLMC(ctypes.Structure):
    _fields_ = [("beta", ctypes.c_float), ("partition_function", ctypes.c_float),
                ("internal_energy", ctypes.c_float), ("specific_heat", ctypes.c_float)]
