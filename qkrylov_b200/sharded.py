"""Row-sharded H.x and Lanczos over several GPUs (one process per GPU).

The reference runs one Hamiltonian on one device; a sector too large for
one B200 (e.g. Hubbard 4x4 at half filling with a stored Krylov basis:
165,636,900 rows, 1.3 GB per FP64 vector) is split here into contiguous row
ranges at sector-block boundaries (qkrylov_b200_basis_shard_bounds).  Each
rank keeps only its rows of every Krylov vector; one step of Lanczos is

* an all-gather of the current vector's slices into a complete x on every
  rank (the step's one exchange: each GPU receives the others' rows, NCCL
  over NVLink; nothing else crosses GPUs),
* the rank's rows of H x from that x (qkrylov_hamiltonian_apply_range_device:
  the same row kernels, restricted to the rank's sector blocks),
* all-reduces of the scalars: alpha, the reorthogonalisation coefficients
  (one all-reduce of k values) and beta.

The tridiagonal is replicated (every rank solves the same small problem
with the same numbers).  The algorithm is the library's FP64 Lanczos
(three-term recurrence, classical Gram-Schmidt against the stored slices
twice, the reference's stopping rule |E_k - E_{k-1}| < tol) on slices.

`apply_rows(x_full, lo, hi) -> y_rows` is the one operator hook: on GPUs it
is the library's range apply (`gpu_apply_rows`); the CPU tests pass a
host implementation with gloo ranks.
"""
from __future__ import annotations

import ctypes
from typing import Callable, Optional

import numpy as np

from ._lib import lib


def shard_bounds(basis, nshards: int) -> np.ndarray:
    """nshards + 1 row bounds at sector-block boundaries (host only)."""
    b = np.zeros(nshards + 1, dtype=np.uint64)
    rc = lib().qkrylov_b200_basis_shard_bounds(basis._h, int(nshards), b.ctypes.data)
    if rc != 0:
        raise RuntimeError(lib().qkrylov_b200_last_error().decode())
    return b.astype(np.int64)


def gpu_apply_rows(H, dtype_code: int):
    """The range apply of a MatrixFreeHamiltonian as an apply_rows hook:
    x_full is a CUDA tensor of the whole vector, the result the rows
    [lo, hi) of H x (a view of a per-hook buffer)."""
    import torch
    state = {}

    def apply_rows(x_full, lo, hi):
        y = state.get("y")
        if y is None or y.shape != x_full.shape or y.dtype != x_full.dtype:
            y = state["y"] = torch.empty_like(x_full)
        rc = lib().qkrylov_hamiltonian_apply_range_device(H._h, dtype_code, ctypes.c_void_p(x_full.data_ptr()),
                                                          ctypes.c_void_p(y.data_ptr()), int(lo), int(hi), None)
        if rc != 0:
            raise RuntimeError(lib().qkrylov_b200_last_error().decode())
        torch.cuda.current_stream().wait_stream(torch.cuda.ExternalStream(H.stream))
        return y[lo:hi]
    return apply_rows


class ShardedLanczosResult:
    def __init__(self, energy, iterations, converged, alphas, betas, eigenvector_rows):
        self.energy, self.iterations, self.converged = energy, iterations, converged
        self.alphas, self.betas = alphas, betas
        self.eigenvector_rows = eigenvector_rows  # this rank's rows of the Ritz vector


def _tridiag_lowest(alphas, betas):
    T = np.diag(np.asarray(alphas, dtype=np.float64))
    if len(betas):
        T += np.diag(np.asarray(betas, dtype=np.float64), 1) + np.diag(np.asarray(betas, dtype=np.float64), -1)
    w, v = np.linalg.eigh(T)
    return w[0], v[:, 0]


def lanczos_sharded(apply_rows: Callable, dim: int, bounds, start_rows, maxiter: int = 200, tol: float = 1e-12,
                    group=None, want_vector: bool = False) -> ShardedLanczosResult:
    """Lanczos ground state with every vector split by rows over the ranks
    of `group` (torch.distributed; None: the default group, or one process
    when torch.distributed is not initialised).  `bounds`: shard_bounds of
    the basis for the world size; `start_rows`: this rank's rows of the
    start vector (a torch tensor on the rank's device; float64 or
    complex128).  Every rank returns the same energy and tridiagonal."""
    import torch
    import torch.distributed as dist
    distributed = dist.is_available() and dist.is_initialized()
    world = dist.get_world_size(group) if distributed else 1
    rank = dist.get_rank(group) if distributed else 0
    bounds = [int(b) for b in bounds]
    if len(bounds) != world + 1 or bounds[0] != 0 or bounds[-1] != dim:
        raise ValueError("bounds must be the shard bounds of this basis for the group's size")
    lo, hi = bounds[rank], bounds[rank + 1]
    v = start_rows.clone()
    if v.shape != (hi - lo,):
        raise ValueError("start_rows must hold this rank's rows")
    sizes = [bounds[k + 1] - bounds[k] for k in range(world)]
    pad = max(sizes)

    def allreduce(t):
        if distributed:
            dist.all_reduce(t, group=group)
        return t

    def gather(vr):
        # slices padded to the largest shard, gathered, unpadded in rank order
        if not distributed:
            return vr
        buf = torch.zeros(pad, dtype=vr.dtype, device=vr.device)
        buf[:vr.shape[0]] = vr
        parts = [torch.empty(pad, dtype=vr.dtype, device=vr.device) for _ in range(world)]
        dist.all_gather(parts, buf, group=group)
        return torch.cat([parts[k][:sizes[k]] for k in range(world)])

    def dot(a, b):  # sum over all ranks of conj(a) . b, FP64
        d = torch.sum(torch.conj(a) * b) if a.is_complex() else torch.sum(a * b)
        r = torch.tensor([d.real.item(), d.imag.item() if a.is_complex() else 0.0], dtype=torch.float64,
                         device=a.device)
        return allreduce(r)

    n0 = float(dot(v, v)[0]) ** 0.5
    if n0 == 0.0:
        raise ValueError("zero start vector")
    v = v / n0
    V = [v]
    alphas, betas = [], []
    e_prev, energy, converged, it = None, None, False, 0
    for it in range(1, maxiter + 1):
        w = apply_rows(gather(v), lo, hi).clone()
        a = float(dot(v, w)[0])
        alphas.append(a)
        w = w - a * v
        if len(V) > 1:
            w = w - betas[-1] * V[-2]
        for _ in range(2):  # classical Gram-Schmidt against every stored slice, twice
            Vm = torch.stack(V)
            c = (torch.conj(Vm) @ w) if w.is_complex() else (Vm @ w)
            cr = torch.view_as_real(c).reshape(-1).to(torch.float64) if c.is_complex() else c.to(torch.float64)
            cr = allreduce(cr.clone())
            c = torch.view_as_complex(cr.reshape(-1, 2)) if w.is_complex() else cr
            w = w - c.to(w.dtype) @ Vm
        energy, _ = _tridiag_lowest(alphas, betas)
        if e_prev is not None and abs(energy - e_prev) < tol:
            converged = True
            break
        e_prev = energy
        b = float(dot(w, w)[0]) ** 0.5
        if b < 1e-15:
            converged = True
            break
        betas.append(b)
        v = w / b
        V.append(v)
    vec = None
    if want_vector:
        _, y = _tridiag_lowest(alphas, betas[:len(alphas) - 1])
        vec = sum(float(y[j]) * V[j] for j in range(len(y)))
        nv = float(dot(vec, vec)[0]) ** 0.5
        vec = vec / nv
    return ShardedLanczosResult(float(energy), it, converged, alphas, betas, vec)
