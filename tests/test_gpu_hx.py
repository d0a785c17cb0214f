"""H.x on the GPU (libqkrylov_b200.so) against the reference and the oracle.

* unit-vector columns: the dense matrix the kernel produces equals the
  reference's CSR (summed in its order) bit for bit;
* random vectors: within 1e-13 (complex128) / 2e-6 (complex64, float32)
  relative to max|y| of the oracle's FP64 result;
* all four vector dtypes through the device-pointer entry point;
* the headline size (Heisenberg N=28, Sz=0) through size-independent
  properties: hermiticity, linearity, sampled rows against the oracle.
"""
import ctypes

import numpy as np
import pytest

import oracle as O
import qkrylov_b200 as qk
from conftest import dense_from_coo, terms_from_golden
from test_compiler import SITES, opsum
from test_sector_tables import make_basis

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def ham(kind, N, sec, terms, dtype=np.float64):
    return qk.MatrixFreeHamiltonian(make_basis(kind, N, sec), SITES[kind](), opsum(terms), dtype=dtype)


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_unit_vector_columns_bit_exact(golden, golden_vecs):
    for name, m in golden["models"].items():
        if f"{name}/coo_rows" not in golden_vecs:
            continue
        H = ham(m["kind"], m["N"], m["sector"], terms_from_golden(m))
        R = dense_from_coo(golden_vecs[f"{name}/coo_rows"], golden_vecs[f"{name}/coo_cols"],
                           golden_vecs[f"{name}/coo_vals"], m["dim"])
        M = np.zeros_like(R)
        for j in range(m["dim"]):
            e = np.zeros(m["dim"], np.complex128)
            e[j] = 1.0
            M[:, j] = H.apply(e)
        assert np.array_equal(M, R), name
        d = H.diagonal()
        assert np.array_equal(d, np.diag(R)), name


@pytest.mark.parametrize("kind,N,sec,terms", [
    ("spin", 20, dict(use_sz=1, sz2=0), O.heisenberg_chain(20)),
    ("spin", 18, dict(use_sz=1, sz2=0), O.j1j2_chain(18, 1.0, 0.41)),
    ("spin", 12, {}, O.heisenberg_chain(12) + [(0.3 + 0.1j, [("Sx", 3)]), (0.2, [("Sy", 5), ("Sz", 1)])]),
    ("fermion", 14, dict(use_n=1, n=6), [(-1.0, [("C", (i + 1) % 14), ("Cdag", i)]) for i in range(14)]
     + [(-1.0, [("C", i), ("Cdag", (i + 1) % 14)]) for i in range(14)] + [(0.4, [("N", i), ("N", (i + 2) % 14)]) for i in range(14)]),
    ("hubbard", 9, dict(use_nup=1, nup=4, use_ndn=1, ndn=4), O.hubbard_square(3, 3)),
    ("hubbard", 8, dict(use_nup=1, nup=4, use_ndn=1, ndn=4), O.hubbard_square(4, 2)),
    ("tj", 12, dict(use_nup=1, nup=5, use_ndn=1, ndn=5), O.tj_chain(12)),
    ("tj", 8, {}, O.tj_chain(8)),
])
def test_random_vectors_vs_oracle(kind, N, sec, terms):
    H = ham(kind, N, sec, terms)
    Po = O.port().hamiltonian(kind, N, sec, terms)
    assert H.dimension == Po.dim
    rng = np.random.default_rng(N)
    x = rng.standard_normal(H.dimension) + 1j * rng.standard_normal(H.dimension)
    yo = Po.apply(x)
    assert rel(H.apply(x), yo) < 1e-13
    H32 = ham(kind, N, sec, terms, dtype=np.float32)
    assert rel(H32.apply(x.astype(np.complex64)).astype(np.complex128), yo) < 2e-6


def test_device_dtypes():
    terms = O.heisenberg_chain(16)
    H = ham("spin", 16, dict(use_sz=1, sz2=0), terms)
    Po = O.port().hamiltonian("spin", 16, dict(use_sz=1, sz2=0), terms)
    rng = np.random.default_rng(1)
    xr = rng.standard_normal(H.dimension)
    xc = xr + 1j * rng.standard_normal(H.dimension)
    for dt, x, tdt, tol in [(qk.DTYPE_C128, xc, torch.complex128, 1e-13), (qk.DTYPE_C64, xc, torch.complex64, 2e-6),
                            (qk.DTYPE_F64, xr, torch.float64, 1e-13), (qk.DTYPE_F32, xr, torch.float32, 2e-6)]:
        xt = torch.tensor(x, dtype=tdt, device="cuda")
        yt = torch.empty_like(xt)
        H.apply_device(xt.data_ptr(), yt.data_ptr(), dt)
        torch.cuda.synchronize()
        assert rel(yt.cpu().numpy().astype(np.complex128), Po.apply(x.astype(np.complex128))) < tol, dt
    # real dtypes are refused for complex operators, aliasing is refused
    Hc = ham("spin", 6, {}, [(0.5j, [("Sp", 0), ("Sm", 1)]), (-0.5j, [("Sm", 0), ("Sp", 1)])])
    t = torch.zeros(Hc.dimension, dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError):
        Hc.apply_device(t.data_ptr(), torch.zeros_like(t).data_ptr(), qk.DTYPE_F64)
    with pytest.raises(ValueError):
        H.apply_device(yt.data_ptr(), yt.data_ptr(), qk.DTYPE_F32)


def sample_rows(kind, N, sec, terms, B, rows, x):
    """y[rows] by the oracle's per-state factor chain (pull mode, one row at a time)."""
    P = O.port()
    out = []
    for a in rows:
        s0, acc = B.state(int(a)), 0j
        for c, f in terms:
            s, amp, ok = s0, complex(c), True
            for op, site in f:
                v, s, me = P.site_apply(kind, op, site, s)
                if not v:
                    ok = False
                    break
                amp *= me
            if ok and B.contains(s):
                acc += amp.conjugate() * x[B.index(s)]
        out.append(acc)
    return np.array(out)


def test_headline_size_properties():
    N = 28
    terms = O.heisenberg_chain(N)
    H = ham("spin", N, dict(use_sz=1, sz2=0), terms)
    D = H.dimension
    assert D == 40116600
    g = torch.Generator(device="cuda").manual_seed(5)
    x = torch.randn(D, dtype=torch.complex128, device="cuda", generator=g)
    z = torch.randn(D, dtype=torch.complex128, device="cuda", generator=g)
    hx, hz, hs = torch.empty_like(x), torch.empty_like(z), torch.empty_like(x)
    H.apply_device(x.data_ptr(), hx.data_ptr(), qk.DTYPE_C128)
    H.apply_device(z.data_ptr(), hz.data_ptr(), qk.DTYPE_C128)
    s = 0.7 * x - 1.3j * z
    H.apply_device(s.data_ptr(), hs.data_ptr(), qk.DTYPE_C128)
    torch.cuda.synchronize()
    # hermiticity <z, Hx> = <Hz, x>
    a, b = torch.vdot(z, hx).item(), torch.vdot(hz, x).item()
    assert abs(a - b) <= 1e-11 * abs(a)
    # linearity
    assert (hs - (0.7 * hx - 1.3j * hz)).abs().max().item() <= 1e-12 * hs.abs().max().item()
    # sampled rows against the oracle's factor-chain evaluation
    B = make_basis("spin", N, dict(use_sz=1, sz2=0))
    rows = np.random.default_rng(2).integers(0, D, 48)
    xh = x.cpu().numpy()
    yo = sample_rows("spin", N, dict(use_sz=1, sz2=0), terms, B, rows, xh)
    assert rel(hx.cpu().numpy()[rows], yo) < 1e-13


@pytest.mark.parametrize("N,terms", [(16, O.heisenberg_chain(16)), (18, O.j1j2_chain(18, 1.0, 0.37)),
                                     (14, [(c * 0.5 if "Sz" in f[0][0] else c, f) for c, f in O.heisenberg_chain(14)]),
                                     (12, O.heisenberg_chain(12, periodic=False))])
def test_spin_exchange_kernel_equals_generic(N, terms):
    """The specialised kernel is selected for exchange models and agrees
    with the generic kernel and the oracle."""
    sec = dict(use_sz=1, sz2=0)
    H = ham("spin", N, sec, terms)
    assert H.kernel == "spin-exchange"
    x = np.random.default_rng(N).standard_normal(H.dimension) + 1j * np.random.default_rng(N + 1).standard_normal(H.dimension)
    y_fast = H.apply(x)
    ys = {}
    try:
        qk.set_kernel_policy("generic")
        ys["generic"] = H.apply(x)
        assert H.kernel == "generic"
    finally:
        qk.set_kernel_policy("auto")
    for pol, y in ys.items():
        assert rel(y_fast, y) < 1e-14, pol
    assert rel(y_fast, O.port().hamiltonian("spin", N, sec, terms).apply(x)) < 1e-13
    Hf = ham("spin", 10, {}, O.heisenberg_chain(10))      # full basis also qualifies
    assert Hf.kernel == "spin-exchange"
    xf = np.random.default_rng(0).standard_normal(Hf.dimension) + 0j
    assert rel(Hf.apply(xf), O.port().hamiltonian("spin", 10, {}, O.heisenberg_chain(10)).apply(xf)) < 1e-13


def test_multi_dot_device():
    """qkrylov_b200_multi_dot against torch on all dtypes (FP64 accumulation)."""
    L = qk.lib()
    rng = np.random.default_rng(9)
    for code, tdt, tol in [(qk.DTYPE_C128, torch.complex128, 1e-13), (qk.DTYPE_C64, torch.complex64, 1e-6),
                           (qk.DTYPE_F64, torch.float64, 1e-13), (qk.DTYPE_F32, torch.float32, 1e-6)]:
        n, k = 300001, 7
        V = [torch.tensor(rng.standard_normal(n), device="cuda").to(tdt) for _ in range(k)]
        x = torch.tensor(rng.standard_normal(n), device="cuda").to(tdt)
        ptrs = (ctypes.c_void_p * k)(*[v.data_ptr() for v in V])
        out = np.zeros(2 * k)
        assert L.qkrylov_b200_multi_dot(torch.cuda.current_device(), code, n, k, ptrs, ctypes.c_void_p(x.data_ptr()),
                                        out.ctypes.data) == 0
        got = out[0::2] + 1j * out[1::2]
        want = np.array([torch.vdot(v.to(torch.complex128), x.to(torch.complex128)).item() for v in V])
        assert np.abs(got - want).max() <= tol * np.abs(want).max() * 10 + 1e-9


@pytest.mark.parametrize("kind,N,sec,terms", [
    ("hubbard", 9, dict(use_nup=1, nup=4, use_ndn=1, ndn=5), O.hubbard_square(3, 3, 1.0, 4.0)),
    ("tj", 12, dict(use_nup=1, nup=5, use_ndn=1, ndn=5), O.tj_chain(12, 1.0, 0.4)),
    ("fermion", 14, dict(use_n=1, n=7), [(-1.0, [("C", (i + 1) % 14), ("Cdag", i)]) for i in range(14)] +
     [(-1.0, [("C", i), ("Cdag", (i + 1) % 14)]) for i in range(14)] + [(0.3, [("N", i), ("N", (i + 1) % 14)]) for i in range(14)]),
])
def test_two_part_kernel_matches_generic(kind, N, sec, terms):
    H = ham(kind, N, sec, terms)
    rng = np.random.default_rng(3)
    x = rng.standard_normal(H.dimension) + 1j * rng.standard_normal(H.dimension)
    qk.set_kernel_policy("no-spin-product")  # Hubbard operators would take the spin-product path
    try:
        assert H.kernel == "two-part"
        y = H.apply(x)
    finally:
        qk.set_kernel_policy("auto")
    qk.set_kernel_policy("generic")
    try:
        yg = H.apply(x)
    finally:
        qk.set_kernel_policy("auto")
    assert rel(y, yg) < 1e-13
    ref = O.port().hamiltonian(kind, N, sec, terms)
    assert rel(y, ref.apply(x)) < 1e-13


def test_per_die_work_queues_give_identical_results():
    """The row kernel hands sector blocks to each die of the GPU from its own
    queue; which CTA computes a row does not change the row's sums, so the
    result is bit-identical to the grid-stride order, for every vector type,
    and across repeated launches (the queues reset themselves)."""
    dies, n0, n1 = qk.die_count()
    assert dies in (1, 2) and (dies == 1 or (n0 > 0 and n1 > 0))
    for kind, N, sec, terms in [("spin", 20, dict(use_sz=1, sz2=0), O.heisenberg_chain(20)),
                                ("tj", 12, dict(use_nup=1, nup=5, use_ndn=1, ndn=5), O.tj_chain(12, 1.0, 0.4))]:
        H = ham(kind, N, sec, terms)
        for code, tdt in [(qk.DTYPE_C128, torch.complex128), (qk.DTYPE_F32, torch.float32)]:
            if kind == "tj" and code == qk.DTYPE_C128:
                continue
            x = torch.randn(H.dimension, dtype=tdt, device="cuda", generator=torch.Generator("cuda").manual_seed(N))
            ys = []
            try:
                for pol in ("auto", "auto", "no-die-queues"):
                    qk.set_kernel_policy(pol)
                    y = torch.empty_like(x)
                    H.apply_device(x.data_ptr(), y.data_ptr(), code)
                    torch.cuda.synchronize()
                    ys.append(y)
            finally:
                qk.set_kernel_policy("auto")
            assert torch.equal(ys[0], ys[1]) and torch.equal(ys[0], ys[2]), (kind, code)
    # the block kernel (batched FTLM): with queues its column dots are summed
    # per tile in tile order, so repeated runs agree bit for bit; the
    # grid-stride form sums per CTA (another order, rounding-level apart)
    H = ham("tj", 12, dict(use_nup=1, nup=5, use_ndn=1, ndn=5), O.tj_chain(12, 1.0, 0.4))
    rs = []
    try:
        for pol in ("auto", "auto", "no-die-queues"):
            qk.set_kernel_policy(pol)
            rs.append(qk.ftlm_block(H, [0.5, 2.0], n_random=32, n_steps=20, seed=3, precision=64, graph=False))
    finally:
        qk.set_kernel_policy("auto")
    assert np.array_equal(rs[0].U, rs[1].U)
    assert np.allclose(rs[0].U, rs[2].U, rtol=1e-12, atol=0)


@pytest.mark.parametrize("N,nup,ndn,lat", [(9, 4, 5, (3, 3)), (16, 2, 3, (4, 4)), (8, 3, 2, (4, 2))])
def test_spin_product_path_matches_two_part_and_oracle(N, nup, ndn, lat):
    """Hubbard operators with N_up and N_dn conserved apply as
    T_up x 1 + 1 x T_dn + D in the (up, down) order (signs S(u, d) at the
    boundary): against the two-part row kernel and the CPU oracle for every
    vector type, and through the fused dot of the solvers (Lanczos energy)."""
    sec = dict(use_nup=1, nup=nup, use_ndn=1, ndn=ndn)
    terms = O.hubbard_square(*lat, 1.0, 4.0)
    H = ham("hubbard", N, sec, terms)
    if H.kernel != "spin-product":
        pytest.skip(f"operator runs on {H.kernel}")
    ref = O.port().hamiltonian("hubbard", N, sec, terms)
    rng = np.random.default_rng(N + nup)
    xh = rng.standard_normal(H.dimension) + 1j * rng.standard_normal(H.dimension)
    yo = ref.apply(xh)
    assert rel(H.apply(xh), yo) < 1e-13
    H32 = ham("hubbard", N, sec, terms, dtype=np.float32)
    assert rel(H32.apply(xh.astype(np.complex64)).astype(np.complex128), yo) < 2e-6
    for code, tdt, tol in [(qk.DTYPE_F64, torch.float64, 1e-13), (qk.DTYPE_C128, torch.complex128, 1e-13),
                           (qk.DTYPE_F32, torch.float32, 1e-5), (qk.DTYPE_C64, torch.complex64, 1e-5)]:
        x = torch.randn(H.dimension, dtype=tdt, device="cuda", generator=torch.Generator("cuda").manual_seed(N))
        ys = []
        try:
            for pol in ("auto", "no-spin-product"):
                qk.set_kernel_policy(pol)
                y = torch.full_like(x, float("nan"))
                torch.cuda.synchronize()
                H.apply_device(x.data_ptr(), y.data_ptr(), code)
                torch.cuda.synchronize()
                ys.append(y.to(torch.complex128).cpu().numpy())
        finally:
            qk.set_kernel_policy("auto")
        assert rel(ys[0], ys[1]) < tol, (code, rel(ys[0], ys[1]))
    es = []
    try:
        for pol in ("auto", "no-spin-product"):
            qk.set_kernel_policy(pol)
            es.append(qk.lanczos_fp64(H, seed=4, tol=1e-12).energy)
    finally:
        qk.set_kernel_policy("auto")
    assert abs(es[0] - es[1]) < 1e-11 * abs(es[1])


@pytest.mark.parametrize("nup,ndn", [(0, 3), (4, 0), (1, 1), (6, 5)])
def test_spin_product_edge_sectors(nup, ndn):
    """Edge sectors of the spin-product path: one species empty (a factor
    with no hops), a single electron of each species, a nearly full
    lattice; against the CPU oracle."""
    N = 6
    sec = dict(use_nup=1, nup=nup, use_ndn=1, ndn=ndn)
    terms = O.hubbard_square(3, 2, 1.0, 4.0)
    H = ham("hubbard", N, sec, terms)
    ref = O.port().hamiltonian("hubbard", N, sec, terms)
    assert H.dimension == ref.dim
    rng = np.random.default_rng(nup * 7 + ndn)
    x = rng.standard_normal(H.dimension) + 1j * rng.standard_normal(H.dimension)
    assert rel(H.apply(x), ref.apply(x)) < 1e-13, H.kernel
