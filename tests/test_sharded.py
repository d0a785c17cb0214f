"""Row-sharded H.x and Lanczos (qkrylov_b200.sharded): the shard bounds
(host code of the library: sector-block boundaries, balanced rows) and the
sharded Lanczos with two gloo ranks on the CPU.  The operator hook here is a
host CSR built from the CPU oracle (test infrastructure); on GPUs the same
solver calls the library's range apply and NCCL.  The two-rank run must
give the single-process energy and the reference's Lanczos energy."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle as O
import qkrylov_b200 as qk
from qkrylov_b200 import sharded


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _csr_apply(kind, N, sec, terms):
    import scipy.sparse as sp
    H = O.port().hamiltonian(kind, N, sec, terms)
    r, c, v = H.coo()
    A = sp.csr_matrix((v, (r, c)), shape=(H.dim, H.dim))
    if np.all(A.data.imag == 0):
        A = A.real

    def apply_rows(x_full, lo, hi):
        y = A[lo:hi] @ x_full.numpy()
        return torch.from_numpy(np.ascontiguousarray(y).astype(x_full.numpy().dtype))
    return apply_rows, H.dim


def test_shard_bounds_are_block_boundaries_and_balanced():
    for N, n in ((16, 2), (16, 3), (20, 8)):
        B = qk.SpinHalfBasis(N, sz=0)
        b = sharded.shard_bounds(B, n)
        assert b[0] == 0 and b[-1] == B.size and np.all(np.diff(b) >= 0)
        st = B.states()
        L = N // 2
        for k in b[1:-1]:  # a bound starts a new high part
            assert (int(st[k]) >> L) != (int(st[k - 1]) >> L)
        assert np.max(np.diff(b)) - np.min(np.diff(b)) <= 2 * 3432
    hb = qk.HubbardBasis(6, nup=3, ndn=3)
    b = sharded.shard_bounds(hb, 4)
    assert b[-1] == hb.size


def _rank(rank, world, port, q):
    import datetime
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        out = {}
        for label, (kind, N, sec, terms, cplx) in {
                "heis16": ("spin", 16, dict(use_sz=1, sz2=0), O.heisenberg_chain(16), False),
                "hub3x2": ("hubbard", 6, dict(use_nup=1, nup=3, use_ndn=1, ndn=3), O.hubbard_square(3, 2, 1.0, 4.0),
                           True)}.items():
            apply_rows, dim = _csr_apply(kind, N, sec, terms)
            basis = {"spin": lambda: qk.SpinHalfBasis(N, sz=0),
                     "hubbard": lambda: qk.HubbardBasis(N, nup=3, ndn=3)}[kind]()
            bounds = sharded.shard_bounds(basis, world)
            lo, hi = int(bounds[rank]), int(bounds[rank + 1])
            x0 = np.random.default_rng(9).uniform(-1, 1, dim)
            if cplx:
                x0 = x0 + 1j * np.random.default_rng(10).uniform(-1, 1, dim)
            r = sharded.lanczos_sharded(apply_rows, dim, bounds, torch.from_numpy(x0[lo:hi].copy()), 200, 1e-12,
                                        want_vector=True)
            y = apply_rows(torch.from_numpy(np.zeros(dim, dtype=x0.dtype)), lo, hi)  # hook shape check
            assert y.shape == (hi - lo,)
            out[label] = (r.energy, r.iterations, r.converged, r.eigenvector_rows.numpy())
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_match_one_process_and_the_reference():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    # drain the queue before joining: a child holding a large item in the
    # queue's pipe does not exit until it is read
    res = dict(q.get(timeout=300) for _ in range(world))
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    for label, (kind, N, sec, terms) in {
            "heis16": ("spin", 16, dict(use_sz=1, sz2=0), O.heisenberg_chain(16)),
            "hub3x2": ("hubbard", 6, dict(use_nup=1, nup=3, use_ndn=1, ndn=3), O.hubbard_square(3, 2, 1.0, 4.0))}.items():
        e0, it0, c0, v0 = res[0][label]
        e1, it1, c1, v1 = res[1][label]
        assert e0 == e1 and it0 == it1 and c0 and c1      # replicated tridiagonal
        E_ref = O.port().hamiltonian(kind, N, sec, terms).lanczos(200, 1e-13)["energy"]
        assert abs(e0 - E_ref) < 1e-10 * abs(E_ref)
        # one process with the same hook
        apply_rows, dim = _csr_apply(kind, N, sec, terms)
        x0 = np.random.default_rng(9).uniform(-1, 1, dim)
        if label == "hub3x2":
            x0 = x0 + 1j * np.random.default_rng(10).uniform(-1, 1, dim)
        one = sharded.lanczos_sharded(apply_rows, dim, [0, dim], torch.from_numpy(x0), 200, 1e-12, want_vector=True)
        assert abs(one.energy - e0) < 1e-12 * abs(E_ref)
        v = np.concatenate([v0, v1])
        Hv = apply_rows(torch.from_numpy(v), 0, dim).numpy()
        assert np.linalg.norm(Hv - e0 * v) < 1e-5
