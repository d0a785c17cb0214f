#!/usr/bin/env python
"""Benchmark: matrix-free H.x effective HBM bandwidth on B200.

Workload: periodic spin-1/2 Heisenberg chain, N=28, J=1, Sz=0 sector
(dim 40,116,600), OpSum Sz_i Sz_i+1 + 0.5 (Sp_i Sm_i+1 + Sm_i Sp_i+1).
One step = one y = H x over the whole sector.  Effective bytes per step
= dim * (bytes(x) + bytes(y)), the metric's algorithmic traffic (sector
tables, term tables and repeated gathers are not counted).

  value  device H.x on complex128 vectors resident in HBM (the drop-in
         fp64 path); x (642 MB) is larger than L2, so no flush is needed
  e2e    the same apply through the C ABI entry point with host buffers
         (qkrylov_hamiltonian_apply_complex_f64): H2D of x, kernel, D2H of y
  variants  the same kernel on complex64 / float64 / float32 vectors
  time_to_e0  plain FP64 GPU Lanczos vs FP32-vector Lanczos + FP64
         refinement, both to the explicit residual 1e-10 (wall seconds)
  batched_ftlm  t-J N=20 FTLM, 64 vectors x 100 steps x 200 temperatures:
         one block (FP32 / FP64 vectors, CUDA graph) vs the one-vector loop
  dynamics  S(q=pi, omega) of the same chain: ground state, phi0 =
         Sz(pi)|psi0>, 300 continued-fraction steps, 2001 omega points;
         and at N=24 every momentum at once (block continued fraction)
  warm_start  J1-J2 N=24: network trained on 32 couplings, time-to-E0 at
         untrained couplings for plain FP64 / mixed / mixed + warm start
  coupling_sweep  J1-J2 N=24 at 32 untrained couplings: one batched block
         of 32 FP64 Lanczos recurrences vs one coupling at a time

cpu_baseline  the reference's own CPU H.x (oracle/_ref) at N=24; with the
         solver legs also its Lanczos (Heisenberg N=22) and FTLM (t-J N=14,
         one temperature) beside the library's GPU solvers on the same models

--impl reference times the reference's own CPU implementation (its
unchanged sources, oracle/_ref, OpenMP on all host cores) on a bounded
sample of the workload, on the same metric.

Multi-GPU (--gpus N under torchrun): the operator does not shard in this
build, so every rank runs an independent replica; value = N * bytes / max
rank time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

HBM_FALLBACK_GBS = 6650.0


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


class ClockSampler:
    """nvidia-smi samples (200 ms) during the timed region."""

    def __init__(self, gpu):
        self.gpu, self.samples, self.proc = gpu, [], None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 7:
                self.samples.append(parts)

    def __exit__(self, *a):
        time.sleep(0.25)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=2)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# ncu summary of the default kernel on this workload (complex128, N=28);
# its dram_bytes_per_launch line is the roofline's measured traffic.
PROFILE = os.path.join(ROOT, "profiles", "hx_spin_rows_heisenberg_n28.md")


def profiled_traffic():
    import re
    try:
        with open(PROFILE) as f:
            m = re.search(r"^dram_bytes_per_launch:\s*(\d+)", f.read(), re.M)
        return int(m.group(1)) if m else None
    except OSError:
        return None


def replica_throughput(ms, bytes_step, world, dist=None, device="cpu"):
    """Replicas: every rank applies H to its own vector; the step time is
    the maximum over ranks and the throughput is world * bytes / that time.
    Returns (max ms, GB/s)."""
    if dist is not None and world > 1:
        import torch
        t = torch.tensor([ms], device=device, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return ms, world * bytes_step / (ms * 1e-3) / 1e9


def tj_opsum(qk, N, t, J):
    """Periodic t-J chain: hops -t (annihilator listed first, both spins,
    both directions) and J (S_i.S_j - n_i n_j / 4) as -J/2 (Nup_i Ndn_j +
    Ndn_i Nup_j) plus the two spin-flip four-fermion terms, factors ordered
    so that the operator qkrylov computes (T^dagger per term, factors applied
    in list order) is the physical one."""
    os_ = qk.OpSum(dtype=np.float64)
    for i in range(N):
        j = (i + 1) % N
        for (a, b) in ((i, j), (j, i)):
            os_.add_term(-t, "CUp", b, "CdagUp", a)
            os_.add_term(-t, "CDn", b, "CdagDn", a)
    for i in range(N):
        j = (i + 1) % N
        os_.add_term(-0.5 * J, "Nup", i, "Ndn", j)
        os_.add_term(-0.5 * J, "Ndn", i, "Nup", j)
        os_.add_term(0.5 * J, "CUp", j, "CdagDn", j, "CDn", i, "CdagUp", i)
        os_.add_term(0.5 * J, "CUp", i, "CdagDn", i, "CDn", j, "CdagUp", j)
    return os_


def hubbard_opsum(qk, Lx, Ly, t, U):
    """Periodic Lx x Ly Hubbard model, site = x + Lx*y: directed hops -t
    c+_i c_j written annihilator first (both spins, both directions of each
    bond, x and y bonds), then U Nupdn on every site."""
    os_ = qk.OpSum(dtype=np.float64)
    for y in range(Ly):
        for x in range(Lx):
            i = x + Lx * y
            for j in sorted({(x + 1) % Lx + Lx * y, x + Lx * ((y + 1) % Ly)} - {i}):
                for (a, b) in ((i, j), (j, i)):
                    os_.add_term(-t, "CUp", b, "CdagUp", a)
                    os_.add_term(-t, "CDn", b, "CdagDn", a)
    for i in range(Lx * Ly):
        os_.add_term(U, "Nupdn", i)
    return os_


def hubbard_c3(qk, tol_lanczos=1e-10, tol_davidson=1e-6, davidson_iters=100):
    """Fermi-Hubbard 4x4 torus, t=1, U=4, 8 up + 8 down (dim 165,636,900):
    H.x (float64) timing, the mixed-precision and the plain FP64 Lanczos
    ground state to the explicit residual tol_lanczos, and block Davidson for
    the 4 lowest
    eigenpairs (block 8, diagonal preconditioner, subspace 64, FP64 vectors,
    seeded random start)."""
    import torch
    B = qk.HubbardBasis(16, nup=8, ndn=8)
    t0 = time.perf_counter()
    H = qk.MatrixFreeHamiltonian(B, qk.HubbardSite(), hubbard_opsum(qk, 4, 4, 1.0, 4.0), dtype=np.float64)
    setup = time.perf_counter() - t0
    D = H.dimension
    x = torch.randn(D, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    for _ in range(3):
        H.apply_device(x.data_ptr(), y.data_ptr(), qk.DTYPE_F64)
    stream = torch.cuda.ExternalStream(H.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(10):
        H.apply_device(x.data_ptr(), y.data_ptr(), qk.DTYPE_F64)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / 10
    del x, y
    torch.cuda.empty_cache()
    out = {"workload": "hubbard_4x4_U4_8up8dn", "dim": D, "setup_seconds": setup, "kernel": H.kernel,
           "hx_f64_ms": ms, "hx_f64_GBs_effective": D * 16 / (ms * 1e-3) / 1e9}
    qk.lanczos_mixed(H, seed=1, tol=tol_lanczos)  # first use of the FP32 path (scratch, modules); the second run is timed
    t0 = time.perf_counter()
    r = qk.lanczos_mixed(H, seed=1, tol=tol_lanczos)
    out["lanczos_mixed"] = {"seconds": time.perf_counter() - t0, "energy": r.energy, "residual": r.residual,
                            "converged": r.converged, "iterations_fp32": r.iterations_low,
                            "iterations_fp64": r.iterations_high}
    # plain FP64 Lanczos (full reorthogonalisation) in runs of at most 64
    # steps, so its Krylov vectors (64 x 1.33 GB) fit beside the operator
    t0 = time.perf_counter()
    r = qk.lanczos_fp64(H, seed=1, tol=tol_lanczos, maxiter=64)
    out["lanczos_fp64"] = {"seconds": time.perf_counter() - t0, "energy": r.energy, "residual": r.residual,
                           "converged": r.converged, "iterations": r.iterations_high, "runs": r.restarts,
                           "steps_per_run": 64}
    out["speedup_mixed_vs_fp64"] = out["lanczos_fp64"]["seconds"] / out["lanczos_mixed"]["seconds"]
    out["dE_mixed_vs_fp64"] = abs(out["lanczos_fp64"]["energy"] - out["lanczos_mixed"]["energy"])
    t0 = time.perf_counter()
    d = qk.davidson_block(H, n_eig=4, block=8, max_subspace=64, tol=tol_davidson, seed=1, maxiter=davidson_iters,
                          precision=64)
    out["davidson_block"] = {"seconds": time.perf_counter() - t0, "eigenvalues": [float(v) for v in d.eigenvalues],
                             "residuals": [float(v) for v in d.residuals], "iterations": d.iterations,
                             "applies": d.applies, "restarts": d.restarts, "converged": d.converged, "tol": tol_davidson}
    return out


def heisenberg_opsum(qk, N, dtype):
    os_ = qk.OpSum(dtype=dtype)
    for i in range(N):
        j = (i + 1) % N
        os_.add_term(1.0, "Sz", i, "Sz", j)
        os_.add_term(0.5, "Sp", i, "Sm", j)
        os_.add_term(0.5, "Sm", i, "Sp", j)
    return os_


def mem_available_gb():
    """Host memory available to this process (MemAvailable), in GB."""
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024 / 1e9
    except OSError:
        pass
    return 0.0


# Peak host memory of the reference's H.x set-up on the Heisenberg chain at
# N sites, Sz=0 (its CSR build: the int32/complex128 `reserve(dim * terms)`
# of matrix_free_hamiltonian.cpp:45-94, the final CSR and the hashed basis),
# in GB: about 100 GB at N = 28, 25 GB at N = 26, 6 GB at N = 24.
def reference_peak_gb(N):
    from math import comb
    dim = comb(N, N // 2)
    return dim * (3 * N * 20 + 43 * 20 + 64) / 1e9


def reference_sizes(force_n=None):
    """Sizes of the reference arm: N = 28 (the headline configuration) when
    its CSR fits with a 2.5x margin in the available host memory, else the
    two largest that do among 26 and 24.  Returns (sizes, infeasible-or-None)."""
    if force_n:
        return [int(force_n)], None
    mem = mem_available_gb()
    if mem >= 2.5 * reference_peak_gb(28):
        return [28], None
    sizes = [n for n in (26, 24) if mem >= 2.5 * reference_peak_gb(n)] or [24]
    return sizes, {"N": 28, "reason": f"the reference's CSR set-up needs ~{reference_peak_gb(28):.0f} GB of host "
                   f"memory (2.5x margin: {2.5 * reference_peak_gb(28):.0f} GB), MemAvailable {mem:.0f} GB",
                   "mem_available_gb": round(mem, 1)}


def cpu_reference_gbs(N=24, steps=5, warmup=1, use_ref=True):
    """Reference CPU H.x (its CSR SpMV through the host-pointer apply,
    matrix_free_hamiltonian.cpp:173-201) on all host threads, `steps`
    timed applies after `warmup`; returns GB/s on the same effective-bytes
    metric (mean over the timed applies)."""
    import oracle as O
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    kind = "reference" if use_ref and O.have_ref() else "port"
    back = O.ref() if kind == "reference" else O.port()
    t0 = time.perf_counter()
    H = back.hamiltonian("spin", N, dict(use_sz=1, sz2=0), O.heisenberg_chain(N))
    setup = time.perf_counter() - t0
    rng = np.random.default_rng(0)
    x = rng.standard_normal(H.dim) + 1j * rng.standard_normal(H.dim)
    y = np.zeros_like(x)
    for _ in range(max(1, warmup)):
        H.apply_into(x, y)
    t0 = time.perf_counter()
    for _ in range(steps):
        H.apply_into(x, y)
    t = (time.perf_counter() - t0) / steps
    del H
    return dict(value=H_dim_bytes(N) / t / 1e9, unit="GB/s", cores=int(os.environ.get("OMP_NUM_THREADS", threads)),
                kind=kind, sample=f"Heisenberg N={N} Sz=0 complex128 H.x, {steps} timed applies after {warmup}; "
                f"setup (basis + CSR build) {setup:.1f} s",
                seconds_per_apply=t, setup_seconds=setup, N=N)


def H_dim_bytes(N):
    from math import comb
    return comb(N, N // 2) * 32


def cpu_reference_solvers(qk, N=22, tj_N=14, R=64, M=100, j1j2_N=24, j1j2_k=100, hub=(4, 3)):
    """The reference's own CPU solvers (its unchanged sources, oracle/_ref,
    all host threads) beside the library's GPU solvers on the same models at
    sizes the CPU finishes in seconds:
      lanczos  Heisenberg chain N, Sz=0: lanczos_ground_state(maxiter 200,
               tol 1e-12), the reference's start vector on both sides
      j1j2_coupling  the warm-start workload's chain (J1-J2, j1j2_N, Sz=0) at
               one coupling J2 = j1j2_k / 255: the reference's time per
               coupling (set-up and Lanczos) against the GPU's
               reference-semantics Lanczos and the mixed-precision form
      hubbard  a periodic hub[0] x hub[1] Hubbard lattice at half filling
               (the reference cannot build the 4x4 one): reference Lanczos on
               both sides, and the GPU's mixed-precision form
      ftlm     t-J chain tj_N (2 holes): the reference's ftlm at one
               temperature (R complex Gaussian vectors, M steps) against the
               GPU's reference-semantics ftlm at one temperature and the
               batched block (R Rademacher vectors, M steps) at 200."""
    import oracle as O
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    kind = "reference" if O.have_ref() else "port"
    back = O.ref() if kind == "reference" else O.port()
    out = {"kind": kind, "cores": int(os.environ.get("OMP_NUM_THREADS", threads))}
    sec = dict(use_sz=1, sz2=0)
    t0 = time.perf_counter()
    Hc = back.hamiltonian("spin", N, sec, O.heisenberg_chain(N))
    setup = time.perf_counter() - t0
    t0 = time.perf_counter()
    rc = Hc.lanczos(200, 1e-12, want_vector=False)
    t_cpu = time.perf_counter() - t0
    del Hc
    Hg = qk.MatrixFreeHamiltonian(qk.SpinHalfBasis(N, sz=0), qk.SpinHalfSite(), heisenberg_opsum(qk, N, np.float64),
                                  dtype=np.float64)
    qk.lanczos_ground_state(Hg, 20, 1e-12)  # warm-up
    t0 = time.perf_counter()
    rg = qk.lanczos_ground_state(Hg, 200, 1e-12)
    t_gpu = time.perf_counter() - t0
    out["lanczos"] = {"workload": f"heisenberg_chain_N{N}_Sz0", "cpu_setup_seconds": setup, "cpu_seconds": t_cpu,
                      "cpu_iterations": rc["iterations"], "gpu_seconds": t_gpu, "gpu_iterations": rg.iterations,
                      "dE": abs(rc["energy"] - rg.energy), "speedup": t_cpu / t_gpu}
    del Hg
    for leg, model, Hg_make in (
            ("j1j2_coupling", ("spin", j1j2_N, sec, O.j1j2_chain(j1j2_N, 1.0, j1j2_k / 255.0)),
             lambda: qk.MatrixFreeHamiltonian(qk.SpinHalfBasis(j1j2_N, sz=0), qk.SpinHalfSite(),
                                              j1j2_opsum(qk, j1j2_N, 1.0, j1j2_k / 255.0), dtype=np.float64)),
            ("hubbard", ("hubbard", hub[0] * hub[1],
                         dict(use_nup=1, nup=hub[0] * hub[1] // 2, use_ndn=1, ndn=hub[0] * hub[1] // 2),
                         O.hubbard_square(hub[0], hub[1], 1.0, 4.0)),
             lambda: qk.MatrixFreeHamiltonian(qk.HubbardBasis(hub[0] * hub[1], nup=hub[0] * hub[1] // 2,
                                                              ndn=hub[0] * hub[1] // 2), qk.HubbardSite(),
                                              hubbard_opsum(qk, hub[0], hub[1], 1.0, 4.0), dtype=np.float64))):
        t0 = time.perf_counter()
        Hc = back.hamiltonian(*model)
        setup = time.perf_counter() - t0
        t0 = time.perf_counter()
        rc = Hc.lanczos(200, 1e-12, want_vector=False)
        t_cpu = time.perf_counter() - t0
        del Hc
        t0 = time.perf_counter()
        Hg = Hg_make()
        g_setup = time.perf_counter() - t0
        qk.lanczos_ground_state(Hg, 20, 1e-12)  # warm-up
        t0 = time.perf_counter()
        rg = qk.lanczos_ground_state(Hg, 200, 1e-12)
        t_gpu = time.perf_counter() - t0
        qk.lanczos_mixed(Hg, seed=1, tol=1e-10)  # warm-up
        t0 = time.perf_counter()
        rm = qk.lanczos_mixed(Hg, seed=1, tol=1e-10)
        t_mix = time.perf_counter() - t0
        out[leg] = {"workload": (f"j1j2_chain_N{j1j2_N}_Sz0_J2_{j1j2_k}/255" if leg == "j1j2_coupling"
                                 else f"hubbard_{hub[0]}x{hub[1]}_U4_half_filling"),
                    "dim": Hg.dimension, "cpu_setup_seconds": setup, "cpu_seconds": t_cpu,
                    "cpu_iterations": rc["iterations"], "gpu_setup_seconds": g_setup, "gpu_seconds": t_gpu,
                    "gpu_iterations": rg.iterations, "gpu_mixed_seconds": t_mix, "gpu_mixed_residual": rm.residual,
                    "dE": abs(rc["energy"] - rg.energy), "dE_mixed": abs(rc["energy"] - rm.energy),
                    "speedup": t_cpu / t_gpu, "speedup_with_setup": (setup + t_cpu) / (g_setup + t_gpu),
                    "speedup_mixed": t_cpu / t_mix}
        del Hg
    ne = tj_N - 2
    tsec = dict(use_nup=1, nup=ne // 2, use_ndn=1, ndn=ne - ne // 2)
    Hc = back.hamiltonian("tj", tj_N, tsec, O.tj_chain(tj_N, 1.0, 0.4))
    t0 = time.perf_counter()
    fc = Hc.ftlm(1.0, R, M)
    t_cpu = time.perf_counter() - t0
    del Hc
    B = qk.TJBasis(tj_N, conserve_nup=True, nup=ne // 2, conserve_ndn=True, ndn=ne - ne // 2)
    Hg = qk.MatrixFreeHamiltonian(B, qk.TJSite(), tj_opsum(qk, tj_N, 1.0, 0.4), dtype=np.float64)
    qk.ftlm(Hg, 1.0, 4, M)  # warm-up
    t0 = time.perf_counter()
    fg = qk.ftlm(Hg, 1.0, R, M)
    t_one = time.perf_counter() - t0
    T = 0.01 * 1000.0 ** (np.arange(200) / 199.0)
    qk.ftlm_block(Hg, T, n_random=R, n_steps=M, seed=5, precision=64)  # tunes the tile shape
    t0 = time.perf_counter()
    qk.ftlm_block(Hg, T, n_random=R, n_steps=M, seed=5, precision=64)
    t_blk = time.perf_counter() - t0
    out["ftlm"] = {"workload": f"tj_chain_N{tj_N}_2holes_Sz0", "dim": Hg.dimension, "R": R, "M": M,
                   "cpu_seconds_per_temperature": t_cpu, "gpu_seconds_per_temperature": t_one,
                   "gpu_block_seconds_200_temperatures": t_blk,
                   "cpu_seconds_200_temperatures": 200 * t_cpu,
                   "U_cpu_T1": fc["U"], "U_gpu_T1": fg.internal_energy}
    return out


def time_to_e0(qk, N, tol=1e-10, seed=1):
    """Plain FP64 GPU Lanczos vs the mixed-precision form on the Heisenberg
    chain, both from a GPU random start, both stopped at the explicit FP64
    residual ||H psi - E psi|| / |E| <= tol; the mixed form with partial
    reorthogonalisation (the default) and with full reorthogonalisation of
    every FP32 step; each form runs twice and the second (warm) run is
    reported."""
    H = qk.MatrixFreeHamiltonian(qk.SpinHalfBasis(N, sz=0), qk.SpinHalfSite(), heisenberg_opsum(qk, N, np.float64),
                                 dtype=np.float64)
    out = {"workload": f"heisenberg_chain_N{N}_Sz0", "dim": H.dimension, "tol_residual": tol,
           "start": f"GPU uniform [-1,1) from seed {seed}"}
    legs = (("plain_fp64", qk.lanczos_fp64), ("mixed", qk.lanczos_mixed),
            ("mixed_full_reorth", lambda H, **kw: qk.lanczos_mixed(H, reorth="full", **kw)))
    for name, fn in legs:
        r = None
        for _ in range(2):
            t0 = time.perf_counter()
            r = fn(H, seed=seed, tol=tol)
            wall = time.perf_counter() - t0
        out[name] = {"seconds": wall, "energy": r.energy, "residual": r.residual, "converged": r.converged,
                     "iterations_fp32": r.iterations_low, "iterations_fp64": r.iterations_high,
                     "restarts": r.restarts}
    out["dE_mixed_vs_plain"] = abs(out["mixed"]["energy"] - out["plain_fp64"]["energy"])
    try:  # the independent FP64 oracle of this model: the Bethe-ansatz energy
        from oracle import bethe
        eb = bethe.ground_energy(N)
        out["E0_bethe"] = eb
        out["dE_vs_bethe"] = {k: abs(out[k]["energy"] - eb) for k in ("plain_fp64", "mixed", "mixed_full_reorth")}
    except Exception as e:
        out["E0_bethe"] = {"error": str(e)}
    out["speedup_mixed"] = out["plain_fp64"]["seconds"] / out["mixed"]["seconds"]
    out["speedup_mixed_full_reorth"] = out["plain_fp64"]["seconds"] / out["mixed_full_reorth"]["seconds"]
    del H
    return out


def batched_ftlm(qk, N=20, R=64, M=100, loop_vectors=64, seed=5):
    """Batched FTLM (R Rademacher vectors as one block, FP32 vectors, FP64
    dots, CUDA graph) vs the one-vector FP64 loop on the same vectors, on
    the periodic t-J chain (2 holes, Sz=0), 200 temperatures in [0.01, 10].
    The loop runs all R vectors (loop_vectors < R times the first ones and
    scales to R; the vectors are independent and equal in cost)."""
    ne = N - 2
    B = qk.TJBasis(N, conserve_nup=True, nup=ne // 2, conserve_ndn=True, ndn=ne - ne // 2)
    H = qk.MatrixFreeHamiltonian(B, qk.TJSite(), tj_opsum(qk, N, 1.0, 0.4), dtype=np.float64)
    T = 0.01 * 1000.0 ** (np.arange(200) / 199.0)
    out = {"workload": f"tj_chain_N{N}_2holes_Sz0", "dim": H.dimension, "R": R, "M": M, "temperatures": 200}
    for prec in (32, 64):
        r = qk.ftlm_block(H, T, n_random=R, n_steps=M, seed=seed, precision=prec)   # tunes the tile shape
        r = qk.ftlm_block(H, T, n_random=R, n_steps=M, seed=seed, precision=prec)
        out[f"block_fp{prec}"] = {"seconds": r.seconds, "seconds_device": r.seconds_device,
                                  "lanes_per_row": r.lanes_per_row, "graph": r.graph}
        if prec == 32:
            r32 = r
        else:
            r64 = r
    l = qk.ftlm_loop(H, T, n_random=R, n_steps=M, seed=seed, precision=64, n_vectors=loop_vectors)
    loop_s = l.seconds_device * R / loop_vectors
    out["loop_fp64"] = {"seconds": loop_s, "measured_vectors": loop_vectors}
    out["speedup_block_fp32"] = loop_s / out["block_fp32"]["seconds"]
    out["speedup_block_fp64"] = loop_s / out["block_fp64"]["seconds"]
    out["max_rel_dU_fp32_vs_fp64"] = float(np.max(np.abs(r32.U - r64.U) / np.abs(r64.U)))
    del H
    return out


def j1j2_opsum(qk, N, J1, J2):
    """Periodic J1-J2 chain: per bond (nearest, then next-nearest)
    J Sz Sz + J/2 (Sp Sm + Sm Sp)."""
    os_ = qk.OpSum(dtype=np.float64)
    for d, J in ((1, J1), (2, J2)):
        for i in range(N):
            j = (i + d) % N
            os_.add_term(J, "Sz", i, "Sz", j)
            os_.add_term(0.5 * J, "Sp", i, "Sm", j)
            os_.add_term(0.5 * J, "Sm", i, "Sp", j)
    return os_


def warm_start(qk, N=24, eval_every=1, eval_offset=1, steps=1500, batch=8192, tol=1e-10):
    """J1-J2 chain, Sz=0: plain FP64 Lanczos ground states at J2_k = k/255
    for k = 0, 8, ..., 248 train the warm-start network on the GPU; at the
    untrained couplings k = eval_offset, eval_offset + eval_every, ... the
    plain FP64 GPU Lanczos (random start), the mixed-precision form (random
    start) and the mixed form from the network's start vector (inference
    included) are each timed to the explicit residual tol."""
    B = qk.SpinHalfBasis(N, sz=0)
    t0 = time.perf_counter()
    net = qk.WarmStartMLP(B, seed=0)
    train_k = list(range(0, 256, 8))
    gs_s = 0.0
    for k in train_k:
        H = qk.MatrixFreeHamiltonian(B, qk.SpinHalfSite(), j1j2_opsum(qk, N, 1.0, k / 255.0), dtype=np.float64)
        t1 = time.perf_counter()
        r = qk.lanczos_fp64(H, seed=1, tol=tol, eigenvector=True)
        gs_s += time.perf_counter() - t1
        net.add_target(k / 255.0, r.eigenvector)
        del H
    t1 = time.perf_counter()
    loss = net.train(steps=steps, batch=batch, lr=2e-3, seed=3)
    train_s = time.perf_counter() - t1
    net.start_vector(train_k[1] / 255.0)  # warm-up of the inference kernel (module load, shared-memory attribute)
    rows = []
    for k in range(eval_offset, 256, eval_every):
        if k % 8 == 0:
            continue
        j2 = k / 255.0
        H = qk.MatrixFreeHamiltonian(B, qk.SpinHalfSite(), j1j2_opsum(qk, N, 1.0, j2), dtype=np.float64)
        qk.lanczos_mixed(H, seed=2, tol=tol)  # warm-up of this operator's kernels
        res = {}
        for name, fn in (("plain_fp64", lambda: qk.lanczos_fp64(H, seed=2, tol=tol)),
                         ("mixed", lambda: qk.lanczos_mixed(H, seed=2, tol=tol)),
                         ("mixed_warm", lambda: qk.lanczos_warm(H, net, j2, tol=tol))):
            t1 = time.perf_counter()
            r = fn()
            res[name] = (time.perf_counter() - t1, r)
        e_ref = res["plain_fp64"][1].energy
        rows.append({"J2": j2,
                     "seconds": {n: v[0] for n, v in res.items()},
                     "iterations": {n: v[1].iterations_low + v[1].iterations_high for n, v in res.items()},
                     "inference_s": res["mixed_warm"][1].seconds_inference,
                     "dE": {n: abs(v[1].energy - e_ref) for n, v in res.items()},
                     "converged": all(v[1].converged for v in res.values())})
        del H
    tot = {n: sum(r["seconds"][n] for r in rows) for n in ("plain_fp64", "mixed", "mixed_warm")}
    regimes = {}
    for name, sel in (("J2_below_0.5", lambda j: j < 0.5), ("J2_from_0.5", lambda j: j >= 0.5)):
        rr = [r for r in rows if sel(r["J2"])]
        if rr:
            t = {n: sum(r["seconds"][n] for r in rr) for n in ("plain_fp64", "mixed", "mixed_warm")}
            regimes[name] = {"couplings": len(rr), "speedup_mixed_warm": t["plain_fp64"] / t["mixed_warm"],
                             "speedup_mixed": t["plain_fp64"] / t["mixed"],
                             "mean_iterations": {n: float(np.mean([r["iterations"][n] for r in rr]))
                                                 for n in ("plain_fp64", "mixed", "mixed_warm")}}
    return net, {"workload": f"j1j2_chain_N{N}_Sz0", "dim": B.size, "train_J2": len(train_k),
            "eval_J2": {"count": len(rows), "first": rows[0]["J2"] if rows else None,
                        "last": rows[-1]["J2"] if rows else None}, "regimes": regimes,
            "train_steps": steps, "batch": batch,
            "train_seconds": train_s, "ground_state_seconds": gs_s, "loss_first": float(loss[:20].mean()),
            "loss_last": float(loss[-20:].mean()), "params": net.n_params,
            "total_seconds": tot, "speedup_mixed": tot["plain_fp64"] / tot["mixed"],
            "speedup_mixed_warm": tot["plain_fp64"] / tot["mixed_warm"],
            "max_dE": max(max(r["dE"].values()) for r in rows), "all_converged": all(r["converged"] for r in rows),
            "mean_iterations": {n: float(np.mean([r["iterations"][n] for r in rows]))
                                for n in ("plain_fp64", "mixed", "mixed_warm")},
            "mean_inference_s": float(np.mean([r["inference_s"] for r in rows])),
            "max_inference_s": float(np.max([r["inference_s"] for r in rows])),
            "wall_seconds": time.perf_counter() - t0}


def dynamics(qk, N, steps=300, eta=0.05, npts=2001, tol=1e-10):
    """Dynamical structure factor of the Heisenberg chain: ground state by
    the mixed-precision Lanczos, phi0 = Sz(q=pi)|psi0> = N^-1/2 sum_j (-1)^j
    Sz_j |psi0> applied as an OpSum-defined operator through the same H.x
    path (apply_operator: the OpSum compiled and applied once, no
    Hamiltonian kept), `steps` continued-fraction Lanczos steps from phi0
    (host vector in, coefficients out, through the reference-facing API),
    then S(omega) on `npts` points of [0, 4] with broadening eta in one
    batched GPU call."""
    B = qk.SpinHalfBasis(N, sz=0)
    H = qk.MatrixFreeHamiltonian(B, qk.SpinHalfSite(), heisenberg_opsum(qk, N, np.float64), dtype=np.float64)
    t0 = time.perf_counter()
    r = qk.lanczos_mixed(H, seed=1, tol=tol, eigenvector=True)
    t_gs = time.perf_counter() - t0
    sz = qk.OpSum(dtype=np.float64)
    for j in range(N):
        sz.add_term((-1.0) ** j / np.sqrt(N), "Sz", j)
    t0 = time.perf_counter()
    phi = qk.apply_operator(B, qk.SpinHalfSite(), sz, r.eigenvector).astype(np.complex128)
    t_phi = time.perf_counter() - t0
    t0 = time.perf_counter()
    cf = qk.continued_fraction_coeffs(H, phi, steps)
    t_cf = time.perf_counter() - t0
    omega = np.linspace(0.0, 4.0, npts)
    t0 = time.perf_counter()
    S = qk.spectral_function_batch(cf, omega, r.energy, eta)
    t_s = time.perf_counter() - t0
    return {"workload": f"heisenberg_chain_N{N}_Sz0_SzPi", "dim": H.dimension, "steps": len(cf.alphas),
            "E0": r.energy, "ground_state_seconds": t_gs, "phi0_seconds": t_phi, "norm_phi0": cf.norm_phi0,
            "cf_seconds": t_cf, "ms_per_cf_step": t_cf / max(1, len(cf.alphas)) * 1e3,
            "spectral_points": npts, "spectral_seconds": t_s, "eta": eta,
            "omega_peak": float(omega[int(np.argmax(S))]),
            "weight_0_4": float(np.sum(S) * (omega[1] - omega[0])),
            "note": "cf_seconds includes the host-to-device copy of phi0 (complex128, 642 MB at N=28)"}


def coupling_sweep(qk, N=24, tol=1e-10, sequential=True, net=None):
    """J1-J2 chain, Sz=0, at the 32 couplings J2_k = k/255, k = 4, 12, ...,
    252: the batched sweep (one FP64 block of 32 Lanczos recurrences over
    H0 = J1 part and H1 = unit J2 part) against the plain FP64 GPU Lanczos
    and the mixed-precision form run one coupling at a time from random
    starts, all to the explicit residual tol; with the warm-start network
    (trained on k = 0, 8, ..., 248) also the sweep from its start vectors
    (inference included)."""
    B = qk.SpinHalfBasis(N, sz=0)
    os0, os1 = qk.OpSum(dtype=np.float64), qk.OpSum(dtype=np.float64)
    for d, os_ in ((1, os0), (2, os1)):
        for i in range(N):
            j = (i + d) % N
            os_.add_term(1.0, "Sz", i, "Sz", j)
            os_.add_term(0.5, "Sp", i, "Sm", j)
            os_.add_term(0.5, "Sm", i, "Sp", j)
    H0 = qk.MatrixFreeHamiltonian(B, qk.SpinHalfSite(), os0, dtype=np.float64)
    H1 = qk.MatrixFreeHamiltonian(B, qk.SpinHalfSite(), os1, dtype=np.float64)
    g = np.array([k / 255.0 for k in range(4, 256, 8)])
    qk.lanczos_sweep(H0, H1, g, tol=1e-6)  # warm-up: block tile tuning of both operators, memory pool
    t0 = time.perf_counter()
    sw = qk.lanczos_sweep(H0, H1, g, tol=tol)
    t_sweep = time.perf_counter() - t0
    warm = None
    if net is not None:
        t0 = time.perf_counter()
        sww = qk.lanczos_sweep(H0, H1, g, tol=tol, net=net)
        warm = {"seconds": time.perf_counter() - t0, "steps": sww.steps, "passes": sww.passes,
                "inference_seconds": sww.seconds_inference, "all_converged": bool(sww.converged.all()),
                "max_dE_vs_random_start_sweep": float(np.max(np.abs(sww.energies - sw.energies)))}
    if not sequential:
        return {"workload": f"j1j2_chain_N{N}_Sz0_32_couplings", "dim": B.size, "couplings": len(g),
                "block": sw.block, "sweep_seconds": t_sweep, "sweep_steps": sw.steps, "sweep_passes": sw.passes,
                "sweep_all_converged": bool(sw.converged.all()), "sweep_warm": warm}
    seq = {"plain_fp64": 0.0, "mixed": 0.0}
    dE = 0.0
    for q, j2 in enumerate(g):
        H = qk.MatrixFreeHamiltonian(B, qk.SpinHalfSite(), j1j2_opsum(qk, N, 1.0, j2), dtype=np.float64)
        qk.lanczos_mixed(H, seed=2, tol=tol)  # warm-up of this operator's kernels
        for name, fn in (("plain_fp64", qk.lanczos_fp64), ("mixed", qk.lanczos_mixed)):
            t1 = time.perf_counter()
            r = fn(H, seed=2, tol=tol)
            seq[name] += time.perf_counter() - t1
            if name == "plain_fp64":
                dE = max(dE, abs(r.energy - sw.energies[q]))
        del H
    return {"workload": f"j1j2_chain_N{N}_Sz0_32_couplings", "dim": B.size, "couplings": len(g), "block": sw.block,
            "sweep_seconds": t_sweep, "sweep_steps": sw.steps, "sweep_passes": sw.passes,
            "sweep_pass_len": 64, "sweep_memory_gb": (64 + 4) * B.size * sw.block * 8 / 1e9,
            "sweep_max_residual": float(sw.residuals.max()), "sweep_all_converged": bool(sw.converged.all()),
            "sequential_seconds": seq, "speedup_vs_plain_fp64": seq["plain_fp64"] / t_sweep,
            "speedup_vs_mixed": seq["mixed"] / t_sweep, "max_dE_vs_plain_fp64": dE,
            "sweep_warm": warm,
            "speedup_warm_vs_plain_fp64": seq["plain_fp64"] / warm["seconds"] if warm else None}


def dynamics_all_momenta(qk, N=24, steps=300):
    """S(q, omega) for every momentum q = 2 pi k / N (k = 1 .. N/2) of the
    Heisenberg chain: the real start vectors cos- and sin-weighted
    sum_j Sz_j |psi0> / sqrt(N) (their fractions add up to the complex
    Sz(q)|psi0> one) as one block continued fraction (FP64 and FP32
    vectors), against one complex continued fraction per momentum (all N/2
    timed)."""
    H = qk.MatrixFreeHamiltonian(qk.SpinHalfBasis(N, sz=0), qk.SpinHalfSite(), heisenberg_opsum(qk, N, np.float64),
                                 dtype=np.float64)
    g = qk.lanczos_fp64(H, seed=1, tol=1e-10, eigenvector=True)
    st = qk.SpinHalfBasis(N, sz=0).states()
    cols, pairs = [], []
    for k in range(1, N // 2 + 1):
        q = 2 * np.pi * k / N
        pair = []
        for w in (np.cos(q * np.arange(N)), np.sin(q * np.arange(N))):
            w[np.abs(w) < 1e-12] = 0.0
            if not w.any():
                continue
            acc = np.zeros(len(st))
            for j in range(N):
                if w[j]:
                    acc += w[j] * (((st >> np.uint64(j)) & np.uint64(1)).astype(np.float64) - 0.5)
            pair.append(len(cols))
            cols.append(g.eigenvector * acc / np.sqrt(N))
        pairs.append(pair)
    X = np.stack(cols, 1)
    out = {"workload": f"heisenberg_chain_N{N}_Sz0_all_q", "momenta": N // 2, "columns": X.shape[1], "steps": steps}
    for prec in (64, 32):
        qk.cf_block(H, X, 20, precision=prec)  # warm-up (tile tuning)
        t0 = time.perf_counter()
        qk.cf_block(H, X, steps, precision=prec)
        out[f"block_fp{prec}_seconds"] = time.perf_counter() - t0
    qk.continued_fraction_coeffs(H, X[:, 0].astype(np.complex128), 20)  # warm-up
    t0 = time.perf_counter()
    for p in pairs:
        z = X[:, p[0]] + (1j * X[:, p[1]] if len(p) > 1 else 0)
        qk.continued_fraction_coeffs(H, z.astype(np.complex128), steps)
    out["one_at_a_time_seconds"] = time.perf_counter() - t0
    out["speedup_block_fp64"] = out["one_at_a_time_seconds"] / out["block_fp64_seconds"]
    out["speedup_block_fp32"] = out["one_at_a_time_seconds"] / out["block_fp32_seconds"]
    return out


def profile_case(qk, name):
    """Small, self-contained launches of one kernel family for ncu captures
    (each runs a few launches on a few GB at most):
      tj20-hx          t-J N=20 (2 holes) two-part row kernel, float64, 4 applies
      tj20-ftlm-block  batched FTLM on the same chain, R=64 FP32 vectors, 4 steps
                       without graph capture (after one tuning run)
      mdot             the reorthogonalisation multi-dot / multi-update of the
                       solvers on 32 float64 vectors of 16 M elements (the
                       kernels of the Davidson projection and the Lanczos
                       reorthogonalisation, at C3's vector length / 10)
      sweep-n20        the batched coupling sweep on the J1-J2 chain N=20 (its
                       column multi-dot / multi-update kernels)
      davidson-n24     block Davidson (block 8, subspace 64, float64) on the
                       Heisenberg chain N=24 (dim 2,704,156; a 64-vector basis
                       is 1.4 GB), 8 iterations: its many-against-many
                       projection and combination kernels at C3's shapes
      hub44-hx         Hubbard 4x4, U=4, 8 up 8 down (dim 165,636,900) H.x on
                       its default path (spin-product), float64, 3 applies
      hub44-hx-two-part  the same on the two-part row kernel"""
    import torch
    out = {}
    if name in ("tj20-hx", "tj20-ftlm-block"):
        N = 20
        B = qk.TJBasis(N, conserve_nup=True, nup=9, conserve_ndn=True, ndn=9)
        H = qk.MatrixFreeHamiltonian(B, qk.TJSite(), tj_opsum(qk, N, 1.0, 0.4), dtype=np.float64)
        out["dim"] = H.dimension
        if name == "tj20-hx":
            x = torch.randn(H.dimension, dtype=torch.float64, device="cuda")
            y = torch.empty_like(x)
            torch.cuda.synchronize()  # x comes from torch's stream, the applies run on the library's
            for _ in range(4):
                H.apply_device(x.data_ptr(), y.data_ptr(), qk.DTYPE_F64)
            torch.cuda.synchronize()
        else:
            T = [0.5, 1.0]
            qk.ftlm_block(H, T, n_random=64, n_steps=4, seed=5, precision=32, graph=False)
            r = qk.ftlm_block(H, T, n_random=64, n_steps=4, seed=5, precision=32, graph=False)
            out["lanes_per_row"] = r.lanes_per_row
    elif name == "mdot":
        n, k = 16 * 1024 * 1024, 32
        V = [torch.randn(n, dtype=torch.float64, device="cuda") for _ in range(k)]
        x = torch.randn(n, dtype=torch.float64, device="cuda")
        L = qk.lib()
        import ctypes
        ptrs = (ctypes.c_void_p * k)(*[v.data_ptr() for v in V])
        o = np.zeros(2 * k)
        for _ in range(3):
            L.qkrylov_b200_multi_dot(torch.cuda.current_device(), qk.DTYPE_F64, n, k, ptrs,
                                     ctypes.c_void_p(x.data_ptr()), o.ctypes.data)
        out.update(n=n, k=k)
    elif name in ("hub44-hx", "hub44-hx-two-part"):
        if name == "hub44-hx-two-part":
            qk.set_kernel_policy("no-spin-product")
        H = qk.MatrixFreeHamiltonian(qk.HubbardBasis(16, nup=8, ndn=8), qk.HubbardSite(),
                                     hubbard_opsum(qk, 4, 4, 1.0, 4.0), dtype=np.float64)
        out["dim"] = H.dimension
        x = torch.randn(H.dimension, dtype=torch.float64, device="cuda")
        y = torch.empty_like(x)
        torch.cuda.synchronize()
        for _ in range(3):
            H.apply_device(x.data_ptr(), y.data_ptr(), qk.DTYPE_F64)
        torch.cuda.synchronize()
    elif name == "sweep-n20":
        out.update(coupling_sweep(qk, N=20, sequential=False))
    elif name == "davidson-n24":
        N = 24
        H = qk.MatrixFreeHamiltonian(qk.SpinHalfBasis(N, sz=0), qk.SpinHalfSite(), heisenberg_opsum(qk, N, np.float64),
                                     dtype=np.float64)
        d = qk.davidson_block(H, n_eig=4, block=8, max_subspace=64, tol=1e-12, seed=1, maxiter=8, precision=64)
        out.update(dim=H.dimension, iterations=d.iterations, applies=d.applies)
    else:
        raise ValueError(f"unknown profile case {name}")
    return out


def run_reference(args):
    """The reference arm: the reference's own CPU H.x (oracle/_ref, its
    unchanged sources, OpenMP on all host threads) on the headline workload
    where the host memory allows, else on the largest Heisenberg chains that
    fit (the line says which and why)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sizes, infeasible = reference_sizes(args.ref_n)
    runs = [cpu_reference_gbs(N=n, steps=max(1, args.steps), warmup=max(1, args.warmup)) for n in sizes]
    cb = runs[0]
    same = cb["N"] == 28
    line = {"metric": "Hx effective HBM GB/s (Heisenberg N=28 Sz=0)", "value": cb["value"], "unit": "GB/s",
            "impl": "reference", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": cb["seconds_per_apply"] * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {"workload": "heisenberg_chain_N28_Sz0_Hx", "N": 28, "dim": 40116600,
                       "sample_N": cb["N"], "same_config": same, "parallelism": "cpu-openmp"},
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if infeasible:
        line["infeasible"] = infeasible
    if len(runs) > 1:
        line["other_samples"] = [{k: r[k] for k in ("N", "value", "seconds_per_apply", "setup_seconds")}
                                 for r in runs[1:]]
    print(json.dumps(line), flush=True)


def run_b200(args):
    import torch
    import qkrylov_b200 as qk

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    N = args.n
    H = qk.MatrixFreeHamiltonian(qk.SpinHalfBasis(N, sz=0), qk.SpinHalfSite(), heisenberg_opsum(qk, N, np.float64),
                                 device=f"cuda:{local}", dtype=np.float64)
    D = H.dimension
    stream = torch.cuda.ExternalStream(H.stream)
    g = torch.Generator(device="cuda").manual_seed(1234 + rank)

    def time_apply(dt_code, tdt, bytes_per, steps, warmup):
        x = torch.randn(D, dtype=tdt, device="cuda", generator=g)
        y = torch.empty_like(x)
        torch.cuda.synchronize()
        for _ in range(warmup):
            H.apply_device(x.data_ptr(), y.data_ptr(), dt_code)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        l0 = qk.lib().qkrylov_b200_launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            H.apply_device(x.data_ptr(), y.data_ptr(), dt_code)
        e1.record(stream)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        ms = e0.elapsed_time(e1) / steps
        launches = int(qk.lib().qkrylov_b200_launch_count() - l0)
        del x, y
        return ms, launches

    peak, peak_kind = peaks()
    if args.profile_case:
        if rank == 0:
            print(json.dumps({"profile_case": args.profile_case, **profile_case(qk, args.profile_case)}), flush=True)
        if dist:
            dist.destroy_process_group()
        return
    if args.hubbard:
        if rank == 0:
            print(json.dumps({"hubbard_only": True, **hubbard_c3(qk)}), flush=True)
        if dist:
            dist.destroy_process_group()
        return
    if args.sweep_only:
        if rank == 0:
            print(json.dumps({"sweep_only": True, **coupling_sweep(qk, N=args.n, sequential=False)}), flush=True)
        if dist:
            dist.destroy_process_group()
        return
    if args.kernel_only:
        qk.set_kernel_policy(args.policy)
        code, tdt, b = {"c128": (qk.DTYPE_C128, torch.complex128, 32), "c64": (qk.DTYPE_C64, torch.complex64, 16),
                        "f64": (qk.DTYPE_F64, torch.float64, 16), "f32": (qk.DTYPE_F32, torch.float32, 8)}[args.kernel_dtype]
        ms, _ = time_apply(code, tdt, b, args.steps, args.warmup)
        if rank == 0:
            print(json.dumps({"kernel_only": True, "N": N, "dim": D, "dtype": args.kernel_dtype, "policy": args.policy,
                              "ms_per_step": ms, "GBs_effective": D * b / (ms * 1e-3) / 1e9, "kernel": H.kernel}),
                  flush=True)
        if dist:
            dist.destroy_process_group()
        return
    with ClockSampler(local) as clk:
        ms, launches = time_apply(qk.DTYPE_C128, torch.complex128, 32, args.steps, args.warmup)
    bytes_step = D * 32
    ms, value = replica_throughput(ms, bytes_step, world, dist, "cuda")

    variants = {}
    for name, code, tdt, b in [("c64", qk.DTYPE_C64, torch.complex64, 16), ("f64", qk.DTYPE_F64, torch.float64, 16),
                               ("f32", qk.DTYPE_F32, torch.float32, 8)]:
        vms, _ = time_apply(code, tdt, b, max(3, args.steps // 2), 2)
        variants[name] = {"ms_per_apply": vms, "GBs_effective": D * b / (vms * 1e-3) / 1e9,
                          "frac_of_measured_hbm": D * b / (vms * 1e-3) / 1e9 / peak}

    # e2e through the C ABI with pinned host buffers
    xh = torch.randn(D, dtype=torch.complex128, generator=torch.Generator().manual_seed(7)).pin_memory()
    yh = torch.empty_like(xh).pin_memory()
    L = qk.lib()
    for _ in range(2):
        L.qkrylov_hamiltonian_apply_complex_f64(H._h, xh.data_ptr(), yh.data_ptr())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ke2e = max(3, args.steps // 2)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(ke2e):
        rc = L.qkrylov_hamiltonian_apply_complex_f64(H._h, xh.data_ptr(), yh.data_ptr())
        assert rc == 0
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / ke2e
    if dist is not None and world > 1:  # the slowest rank's host round trip
        t = torch.tensor([e2e_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())

    traffic = profiled_traffic() if N == 28 else None

    line = {"metric": "Hx effective HBM GB/s (Heisenberg N=28 Sz=0)", "value": value, "unit": "GB/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "data": "synthetic",
            "config": {"workload": "heisenberg_chain_N28_Sz0_Hx", "N": N, "dim": D, "terms": 3 * N,
                       "vector": "complex128", "l2": "inputs larger than L2 (x = 642 MB)",
                       "parallelism": "replicas" if world > 1 else "single-gpu"},
            "roofline": {"bound": "hbm", "achieved": bytes_step / (ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": bytes_step / (ms * 1e-3) / 1e9 / peak, "traffic": traffic,
                         "peak_source": peak_kind, "kernel": H.kernel},
            "e2e": {"value": world * bytes_step / (e2e_ms * 1e-3) / 1e9, "unit": "GB/s",
                    "h2d_bytes_per_step": D * 16, "d2h_bytes_per_step": D * 16, "ms_per_step": e2e_ms,
                    "path": "qkrylov_hamiltonian_apply_complex_f64, pinned host buffers"},
            "variants": variants,
            "gpu_launches": launches,
            "clocks": clk.summary()}
    # the solver legs and the CPU baseline are single-GPU measurements: they
    # run with one rank (N=1) only
    if rank == 0 and world == 1 and not args.no_solvers:
        try:
            torch.cuda.empty_cache()
            line["time_to_e0"] = time_to_e0(qk, N)
        except Exception as e:  # reported, never silently replaced
            line["time_to_e0"] = {"error": str(e)}
        try:
            torch.cuda.empty_cache()
            line["batched_ftlm"] = batched_ftlm(qk)
        except Exception as e:
            line["batched_ftlm"] = {"error": str(e)}
        try:
            torch.cuda.empty_cache()
            line["dynamics"] = dynamics(qk, N)
            line["dynamics"]["all_momenta"] = dynamics_all_momenta(qk)
        except Exception as e:
            line["dynamics"] = {"error": str(e)}
        net = None
        try:
            torch.cuda.empty_cache()
            net, line["warm_start"] = warm_start(qk)
        except Exception as e:
            line["warm_start"] = {"error": str(e)}
        try:
            torch.cuda.empty_cache()
            line["coupling_sweep"] = coupling_sweep(qk, net=net)
        except Exception as e:
            line["coupling_sweep"] = {"error": str(e)}
        del net
        try:
            torch.cuda.empty_cache()
            line["hubbard_c3"] = hubbard_c3(qk)
        except Exception as e:
            line["hubbard_c3"] = {"error": str(e)}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cb = cpu_reference_gbs(N=24, steps=5)
            line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
            if not args.no_solvers:
                line["cpu_baseline"]["solvers"] = cpu_reference_solvers(qk)
        except Exception as e:  # reported, never silently replaced
            line["cpu_baseline"] = {"value": None, "unit": "GB/s", "error": str(e)}
    if rank == 0:
        line["summary"] = summary(line)  # last key: the headline numbers of every leg, compactly
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def summary(line):
    """The headline figure of each leg in a few short keys (None where a leg
    did not run or failed)."""
    def get(*path):
        v = line
        for k in path:
            if not isinstance(v, dict) or k not in v:
                return None
            v = v[k]
        return round(v, 4) if isinstance(v, float) else v
    return {"hx_c128_frac": get("roofline", "frac"), "hx_f32_ms": get("variants", "f32", "ms_per_apply"),
            "e2e_GBs": get("e2e", "value"),
            "t2e0_mixed_vs_fp64": get("time_to_e0", "speedup_mixed"),
            "t2e0_mixed_full_reorth_vs_fp64": get("time_to_e0", "speedup_mixed_full_reorth"),
            "dE_bethe": get("time_to_e0", "dE_vs_bethe"),
            "ftlm_fp64_vs_loop": get("batched_ftlm", "speedup_block_fp64"),
            "ftlm_fp32_vs_loop": get("batched_ftlm", "speedup_block_fp32"),
            "warm_vs_fp64": get("warm_start", "speedup_mixed_warm"),
            "sweep_vs_fp64": get("coupling_sweep", "speedup_vs_plain_fp64"),
            "cf_all_q_vs_one": get("dynamics", "all_momenta", "speedup_block_fp64"),
            "hubbard_hx_ms": get("hubbard_c3", "hx_f64_ms"),
            "hubbard_mixed_vs_fp64": get("hubbard_c3", "speedup_mixed_vs_fp64"),
            "hubbard_davidson_ok": get("hubbard_c3", "davidson_block", "converged"),
            "cpu_ref_GBs": get("cpu_baseline", "value"),
            "j1j2_coupling_cpu_vs_gpu_mixed": get("cpu_baseline", "solvers", "j1j2_coupling", "speedup_mixed")}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=28)
    ap.add_argument("--ref-n", type=int, default=None,
                    help="reference arm: chain length (default: 28 when its CSR fits in host memory, else 26/24)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-solvers", action="store_true", help="skip the time-to-E0 Lanczos comparison")
    ap.add_argument("--kernel-only", action="store_true",
                    help="time only the device apply (profiling runs)")
    ap.add_argument("--kernel-dtype", default="c128", choices=["c128", "c64", "f64", "f32"],
                    help="vector type of --kernel-only")
    ap.add_argument("--policy", default="auto", help="H.x kernel policy of --kernel-only (qkrylov_b200.set_kernel_policy)")
    ap.add_argument("--hubbard", action="store_true",
                    help="only the Hubbard 4x4 (8 up, 8 down) H.x, mixed-precision Lanczos and block Davidson")
    ap.add_argument("--profile-case", default=None,
                    help="run one small kernel case for an ncu capture (see profile_case) and exit")
    ap.add_argument("--sweep-only", action="store_true",
                    help="only the batched coupling sweep on the J1-J2 chain of --n sites (no one-at-a-time runs)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
