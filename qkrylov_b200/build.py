"""Build recipe for libqkrylov_b200.so (in-tree, sm_100a only).

    python -m qkrylov_b200.build            # incremental
    python -m qkrylov_b200.build --clean

CUDA sources are compiled by nvcc for sm_100a, host C++20 sources by g++
(the C++ API layer twice: fp64 and fp32 precision namespaces, the way the
qkrylov library ships both), and everything is linked into one shared
library next to this file.  Objects go to qkrylov_b200/_build/.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libqkrylov_b200.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
GXX = shutil.which("g++", path="/usr/bin:" + os.environ.get("PATH", "")) or "g++"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
INCLUDES = ["-I" + os.path.join(ROOT, "include"), "-I" + CSRC, "-I" + os.path.join(CUDA_HOME, "include")]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                     "-ccbin", GXX] + INCLUDES
CXX_FLAGS = ["-O3", "-std=c++20", "-fPIC", "-Wall", "-Wno-unused-function"] + INCLUDES

CU_SOURCES = ["kernels/vec.cu", "kernels/hx.cu", "kernels/krylov.cu", "kernels/block.cu", "kernels/mlp.cu", "kernels/mlp_tc.cu", "kernels/noalloc.cu",
              "kernels/hx_spin.cu", "kernels/hx_pair.cu", "kernels/topology.cu", "kernels/spectral.cu"]
ENGINE_SOURCES = ["engine/sector.cpp", "engine/compile.cpp", "engine/operator.cpp", "engine/runtime.cpp",
                  "engine/solvers.cpp", "engine/npy.cpp", "engine/ftlm_block.cpp", "engine/warmstart.cpp", "engine/sweep.cpp"]
API_SOURCES = ["api/objects.cpp", "api/solvers_api.cpp"]  # compiled for fp64 and fp32
C_ABI_SOURCES = ["api/common.cpp", "api/c_api.cpp", "api/c_api_ext.cpp"]


def _sources():
    out = []
    for s in CU_SOURCES:
        if os.path.exists(os.path.join(CSRC, s)):
            out.append(("cu", s, []))
    for s in ENGINE_SOURCES + C_ABI_SOURCES:
        if os.path.exists(os.path.join(CSRC, s)):
            out.append(("cxx", s, []))
    for s in API_SOURCES:
        if os.path.exists(os.path.join(CSRC, s)):
            out.append(("cxx", s, ["-DQKRYLOV_DOUBLE_PRECISION"]))
            out.append(("cxx", s, []))
    return out


def _obj_path(src, defs):
    tag = "_fp64" if "-DQKRYLOV_DOUBLE_PRECISION" in defs else ""
    return os.path.join(BUILD, src.replace("/", "_").rsplit(".", 1)[0] + tag + ".o")


def _headers_mtime():
    newest = 0.0
    for base in (CSRC, os.path.join(ROOT, "include")):
        for dp, _, fs in os.walk(base):
            for f in fs:
                if f.endswith((".h", ".hpp", ".cuh")):
                    newest = max(newest, os.path.getmtime(os.path.join(dp, f)))
    return newest


def _compile(job):
    kind, src, defs = job
    obj = _obj_path(src, defs)
    path = os.path.join(CSRC, src)
    if kind == "cu":
        cmd = [NVCC] + NVCC_FLAGS + defs + ["-c", path, "-o", obj]
    else:
        cmd = [GXX] + CXX_FLAGS + defs + ["-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj


def build(verbose=False, jobs=None):
    os.makedirs(BUILD, exist_ok=True)
    hdr = _headers_mtime()
    todo, objs = [], []
    for job in _sources():
        obj = _obj_path(job[1], job[2])
        objs.append(obj)
        src_m = os.path.getmtime(os.path.join(CSRC, job[1]))
        if not os.path.exists(obj) or os.path.getmtime(obj) < max(src_m, hdr):
            todo.append(job)
    if todo:
        with cf.ThreadPoolExecutor(jobs or os.cpu_count() or 4) as ex:
            for obj in ex.map(_compile, todo):
                if verbose:
                    print("built", os.path.relpath(obj, ROOT))
    if todo or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-ccbin", GXX, "-o", LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose:
            print("linked", os.path.relpath(LIB, ROOT))
    return LIB


def clean():
    shutil.rmtree(BUILD, ignore_errors=True)
    if os.path.exists(LIB):
        os.remove(LIB)


if __name__ == "__main__":
    if "--clean" in sys.argv:
        clean()
    build(verbose=True)
