"""Bethe-ansatz ground-state energy of the periodic spin-1/2 Heisenberg chain.

TEST INFRASTRUCTURE ONLY: an independent FP64 check of the ground-state
energies that the GPU solvers compute at sizes the reference's own CSR build
cannot reach (N = 24 needs ~6 GB of host CSR, N = 28 ~100 GB).

Model: H = J sum_i S_i . S_{i+1} on a ring of N sites (even N), which is
the reference's test OpSum ``Sz Sz + 0.5 (Sp Sm + Sm Sp)`` per bond
(tests/test_workflow.cpp:34-36 of the reference, periodic form as in
bindings/julia/test/runtests.jl:164-166).  For J > 0 the ground state lies in
the Sz = 0 sector with M = N/2 flipped spins.

Method (Bethe 1931; logarithmic form, e.g. Karbach & Mueller, "Introduction
to the Bethe ansatz I/II", Computers in Physics 11 (1997) / 12 (1998)):
rapidities lambda_1..lambda_M solve

    N * 2 atan(2 lambda_j) = 2 pi I_j + sum_{l != j} 2 atan(lambda_j - lambda_l)

with the ground-state quantum numbers I_j = -(M-1)/2, ..., (M-1)/2, and

    E = J N / 4 - (J / 2) sum_j 1 / (lambda_j^2 + 1/4).

The equations are solved by Newton's method from the free-magnon guess
lambda_j = tan(pi I_j / N) / 2 (the scattering phases dropped); the Jacobian
is dense M x M.  Newton converges quadratically; the iteration stops when
the update is at rounding level, which gives E to a few ulps (checked in
tests/test_bethe.py against the reference's own E0 = -2 at N = 4 and its
Lanczos energies at N = 12 and 16).
"""
from __future__ import annotations

import numpy as np


def rapidities(N: int, max_iter: int = 100) -> np.ndarray:
    if N < 2 or N % 2:
        raise ValueError("the Bethe-ansatz ground state here needs an even N >= 2")
    M = N // 2
    I = np.arange(M, dtype=np.float64) - (M - 1) / 2.0
    lam = 0.5 * np.tan(np.pi * I / N)
    polish = 0
    for _ in range(max_iter):
        d = lam[:, None] - lam[None, :]
        F = N * 2.0 * np.arctan(2.0 * lam) - 2.0 * np.pi * I - (2.0 * np.arctan(d)).sum(axis=1)
        K = 2.0 / (1.0 + d * d)              # d/d lambda of 2 atan(lambda_j - lambda_l)
        np.fill_diagonal(K, 0.0)
        Jm = K.copy()                        # dF_j / dlambda_l, l != j
        np.fill_diagonal(Jm, 4.0 * N / (1.0 + 4.0 * lam * lam) - K.sum(axis=1))
        step = np.linalg.solve(Jm, F)
        lam = lam - step
        # quadratic convergence reaches rounding level in a few steps; two
        # more steps past 1e-12 leave only rounding-level updates
        if np.max(np.abs(step)) <= 1e-12 * max(1.0, np.max(np.abs(lam))):
            polish += 1
            if polish > 2:
                break
    else:
        raise RuntimeError(f"Bethe equations did not converge for N={N}")
    return lam


def ground_energy(N: int, J: float = 1.0) -> float:
    """E0 of the periodic Heisenberg ring of N sites (even N), coupling J > 0."""
    lam = rapidities(N)
    # sum in ascending magnitude of the terms for a few ulps less rounding
    t = np.sort(1.0 / (lam * lam + 0.25))
    return float(J * N / 4.0 - (J / 2.0) * t.sum())
