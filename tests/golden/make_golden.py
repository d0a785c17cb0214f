"""Generate the golden fixtures from the qkrylov reference's own code.

Runs the reference's unchanged sources (oracle/_ref/liboracle_ref.so, built
by ``make -C oracle ref REF=<reference checkout>``) on small
problems and writes:

  golden.json        scalar results, basis digests, small COO matrices
  golden_vectors.npz eigenvectors and tridiagonals of a few mid-size runs

Only this script needs the reference; the tests read the committed files.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle as O  # noqa: E402


def digest(states):
    return hashlib.sha256(np.ascontiguousarray(states, dtype=np.uint64).tobytes()).hexdigest()


SECTORS = [
    ("spin", 4, dict(use_sz=1, sz2=0)), ("spin", 3, {}), ("spin", 10, dict(use_sz=1, sz2=2)),
    ("spin", 12, dict(use_sz=1, sz2=0)), ("spin", 16, dict(use_sz=1, sz2=0)), ("spin", 9, dict(use_sz=1, sz2=0)),
    ("spin", 14, dict(use_sz=1, sz2=-6)), ("spin", 20, dict(use_sz=1, sz2=0)),
    ("fermion", 4, {}), ("fermion", 4, dict(use_n=1, n=2)), ("fermion", 12, dict(use_n=1, n=5)),
    ("hubbard", 2, {}), ("hubbard", 4, dict(use_nup=1, nup=2, use_ndn=1, ndn=2)),
    ("hubbard", 6, dict(use_nup=1, nup=3, use_ndn=1, ndn=2)), ("hubbard", 5, dict(use_nup=1, nup=2)),
    ("hubbard", 5, dict(use_ndn=1, ndn=3)), ("hubbard", 8, dict(use_nup=1, nup=4, use_ndn=1, ndn=4)),
    ("tj", 2, {}), ("tj", 6, dict(use_nup=1, nup=2, use_ndn=1, ndn=2)), ("tj", 7, dict(use_nup=1, nup=3)),
    ("tj", 10, dict(use_nup=1, nup=4, use_ndn=1, ndn=4)), ("tj", 5, {}),
]


def small_models():
    """(name, kind, N, sector, terms) of the COO / solver fixtures."""
    h4 = []
    for i in range(3):  # tests/test_workflow.cpp:34-36 (open chain)
        h4 += [(1.0, [("Sz", i), ("Sz", i + 1)]), (0.5, [("Sp", i), ("Sm", i + 1)]), (0.5, [("Sm", i), ("Sp", i + 1)])]
    ferm = ([(-1.0, [("C", (i + 1) % 8), ("Cdag", i)]) for i in range(8)] +
            [(-1.0, [("C", i), ("Cdag", (i + 1) % 8)]) for i in range(8)] +
            [(0.5, [("N", i), ("N", (i + 1) % 8)]) for i in range(8)])
    spin_cplx = O.heisenberg_chain(6) + [(0.3, [("Sx", 2)]), (0.2, [("Sy", 3), ("Sz", 1)]),
                                         (0.7, [("Sy", 0), ("Sy", 1)]), (0.25j, [("Sp", 4), ("Sm", 5)]),
                                         (-0.25j, [("Sm", 4), ("Sp", 5)])]
    return [
        ("heis4_obc_sz0", "spin", 4, dict(use_sz=1, sz2=0), h4),
        ("heis4_pbc_full", "spin", 4, {}, O.heisenberg_chain(4)),
        ("heis2_full", "spin", 2, {}, O.heisenberg_chain(2, periodic=False)),
        ("sz3body_3site", "spin", 3, {}, [(1.0, [("Sz", 0), ("Sz", 1)]), (0.5, [("Sz", 0), ("Sz", 1), ("Sz", 2)])]),
        ("heis10_sz0", "spin", 10, dict(use_sz=1, sz2=0), O.heisenberg_chain(10)),
        ("spin6_complex_full", "spin", 6, {}, spin_cplx),
        ("fermion8_n4", "fermion", 8, dict(use_n=1, n=4), ferm),
        ("hubbard_3x2", "hubbard", 6, dict(use_nup=1, nup=3, use_ndn=1, ndn=3), O.hubbard_square(3, 2)),
        ("hubbard_2x2_full", "hubbard", 4, {}, O.hubbard_square(2, 2)),
        ("tj6_2h", "tj", 6, dict(use_nup=1, nup=2, use_ndn=1, ndn=2), O.tj_chain(6)),
        ("tj5_full", "tj", 5, {}, O.tj_chain(5)),
    ]


def main():
    R = O.ref()
    out = {"source": "qkrylov reference sources compiled by oracle/Makefile (target ref)", "bases": [],
           "sites": [], "models": {}}
    # basis digests (src/basis/*.cpp)
    for kind, N, sec in SECTORS:
        st = R.basis_states(kind, N, sec)
        out["bases"].append(dict(kind=kind, N=N, sector=sec, dim=int(st.size), sha256=digest(st),
                                 head=[int(s) for s in st[:8]], tail=[int(s) for s in st[-8:]]))
    # single-site actions on a few states (src/sites/*.cpp)
    ops = {"spin": ["Sz", "Sp", "Sm", "Sx", "Sy"], "fermion": ["N", "Id", "C", "Cdag"],
           "hubbard": ["Nup", "Ndn", "Nupdn", "CUp", "CdagUp", "CDn", "CdagDn"],
           "tj": ["Nup", "Ndn", "CUp", "CdagUp", "CDn", "CdagDn"]}
    for kind, names in ops.items():
        for op in names:
            for site in (0, 1, 3):
                for state in (0b0000, 0b1010, 0b0110, 0b1111, 0b10011001, 0b01100110):
                    v, ns, me = R.site_apply(kind, op, site, state)
                    out["sites"].append(dict(kind=kind, op=op, site=site, state=state, valid=v, new_state=ns,
                                             me=[me.real, me.imag]))
    vecs = {}
    for name, kind, N, sec, terms in small_models():
        H = R.hamiltonian(kind, N, sec, terms)
        r, c, v = H.coo()
        m = dict(kind=kind, N=N, sector=sec, terms=[[[t[0].real, t[0].imag] if isinstance(t[0], complex)
                                                      else [float(t[0]), 0.0], t[1]] for t in terms],
                 dim=H.dim)
        if H.dim <= 400:  # the reference's CSR entries, in its order (zeros kept)
            vecs[f"{name}/coo_rows"] = r.astype(np.int32)
            vecs[f"{name}/coo_cols"] = c.astype(np.int32)
            vecs[f"{name}/coo_vals"] = v
        m["diagonal"] = [[d.real, d.imag] for d in H.diagonal()[:64]]
        lz = H.lanczos(200, 1e-12)
        m["lanczos"] = dict(energy=lz["energy"], iterations=lz["iterations"], converged=lz["converged"])
        vecs[f"{name}/lanczos_vec"] = lz["eigenvector"]
        dv = H.davidson(2, 10, 1e-8)
        m["davidson"] = dict(eigenvalues=dv["eigenvalues"].tolist(), iterations=dv["iterations"],
                             converged=dv["converged"])
        phi = np.zeros(H.dim, complex)
        phi[0] = 1.0
        cf = H.cf(phi, 8)
        m["cf_e0"] = dict(alphas=cf["alphas"].tolist(), betas=cf["betas"].tolist(), norm_phi0=cf["norm_phi0"])
        m["ftlm"] = [dict(beta=b, **{k: v for k, v in H.ftlm(b, 5, 20).items() if k != "beta"}) for b in (0.1, 1.0, 3.0)]
        out["models"][name] = m
    # mid-size runs: Heisenberg N=12 and N=16 (the N=16 Lanczos configuration)
    for N in (12, 16):
        H = R.hamiltonian("spin", N, dict(use_sz=1, sz2=0), O.heisenberg_chain(N))
        lz = H.lanczos(200, 1e-12)
        out["models"][f"heis{N}_sz0"] = dict(kind="spin", N=N, sector=dict(use_sz=1, sz2=0), dim=H.dim,
                                             lanczos=dict(energy=lz["energy"], iterations=lz["iterations"],
                                                          converged=lz["converged"]))
        if N == 12:
            vecs["heis12_sz0/lanczos_vec"] = lz["eigenvector"]
            # S(q=pi, w) start: Sz(pi)|E0> = N^-1/2 sum_j (-1)^j Sz_j |E0>
            st = H.states()
            sz = np.array([[0.5 if (s >> j) & 1 else -0.5 for j in range(N)] for s in st])
            phi = (sz * ((-1.0) ** np.arange(N))).sum(1) / np.sqrt(N) * lz["eigenvector"]
            cf = H.cf(phi, 40)
            out["models"]["heis12_sz0"]["cf_szpi"] = dict(alphas=cf["alphas"].tolist(), betas=cf["betas"].tolist(),
                                                          norm_phi0=cf["norm_phi0"])
            vecs["heis12_sz0/phi_szpi"] = phi
            w = np.linspace(0, 4, 41)
            out["models"]["heis12_sz0"]["spectral"] = dict(
                omega=w.tolist(), eta=0.05,
                S=[R.spectral(cf["alphas"], cf["betas"], cf["norm_phi0"], x, lz["energy"], 0.05) for x in w])
            out["models"]["heis12_sz0"]["ftlm"] = [dict(beta=b, **{k: v for k, v in H.ftlm(b, 4, 30).items()
                                                                  if k != "beta"}) for b in (0.2, 1.0, 5.0)]
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"))
    np.savez_compressed(os.path.join(HERE, "golden_vectors.npz"), **vecs)
    print("wrote", len(out["bases"]), "bases,", len(out["sites"]), "site actions,", len(out["models"]), "models")


if __name__ == "__main__":
    main()
