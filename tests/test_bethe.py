"""The Bethe-ansatz energy oracle (oracle/bethe.py) against the reference's
own numbers: E0 = -2 of the periodic 4-site chain (the reference's Julia
test, bindings/julia/test/runtests.jl:164-166) and the reference's FP64
Lanczos energies of the periodic Heisenberg chains N = 12 and N = 16
(golden fixtures from oracle/_ref), plus the CPU restatement's Lanczos at
N = 18.  CPU only."""
import numpy as np

import oracle as O
from oracle import bethe


def test_four_site_ring_is_minus_two():
    assert abs(bethe.ground_energy(4) + 2.0) < 1e-13


def test_matches_reference_lanczos(golden):
    for key, N in (("heis12_sz0", 12), ("heis16_sz0", 16)):
        E_ref = golden["models"][key]["lanczos"]["energy"]
        assert abs(bethe.ground_energy(N) - E_ref) < 1e-12 * abs(E_ref), (N, E_ref)


def test_matches_restatement_lanczos_n18():
    E = O.port().hamiltonian("spin", 18, dict(use_sz=1, sz2=0), O.heisenberg_chain(18)).lanczos(200, 1e-14)["energy"]
    assert abs(bethe.ground_energy(18) - E) < 1e-12 * abs(E)


def test_coupling_scales_energy():
    assert abs(bethe.ground_energy(10, J=2.5) - 2.5 * bethe.ground_energy(10)) < 1e-12


def test_energy_per_site_approaches_hulthen_limit():
    # Hulthen (1938): E0 / N -> 1/4 - ln 2 as N -> infinity, from below in |E|
    e = [bethe.ground_energy(N) / N for N in (8, 16, 28)]
    lim = 0.25 - np.log(2.0)
    assert e[0] < e[1] < e[2] < lim + 1e-3 and abs(e[2] - lim) < 2e-3
