"""In-tree build of libda_b200.so (CUDA for sm_100a + host C++), no torch extension machinery.

Each translation unit is compiled on its own so that the FP64 kernels can be built without
FMA contraction (bit-exact against the CPU reference) while the FP32-split kernels keep it.
Objects go to discrete_adjoint_b200/_build/, the shared library next to this file.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libda_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + INCLUDE, "-I" + CSRC] + ARCH

# (source, extra flags)
UNITS = [
    ("capi.cu", []),
    ("forward_fp64.cu", ["--fmad=false"]),
    ("forward_fp32.cu", ["-prec-div=false", "-prec-sqrt=false"]),
    ("adjoint_fp64.cu", ["--fmad=false"]),
    ("adjoint_fp32.cu", ["-prec-div=false", "-prec-sqrt=false"]),
    ("adjoint_host.cu", []),
    ("adjoint_ref.cu", ["--fmad=false"]),
    ("noalloc.cu", ["--fmad=false"]),
    ("domain.cu", []),
    ("snapshot.cu", []),
    ("ensemble.cu", []),
    ("dwr.cu", []),
    ("stats.cu", []),
    ("mesh_host.cpp", []),
    ("solution_io.cpp", []),
    ("restart_io.cpp", []),
]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libda_b200")
    return cand


def _headers() -> list[str]:
    out = []
    for d in (CSRC, INCLUDE):
        for f in os.listdir(d):
            if f.endswith((".h", ".cuh", ".hpp")):
                out.append(os.path.join(d, f))
    return out


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    hdrs = _headers()
    objs, jobs = [], []
    for src, extra in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, [s, __file__] + hdrs):
            if src.endswith(".cpp"):
                cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-I" + INCLUDE, "-I" + CSRC, "-c", s, "-o", o]
            else:
                cmd = [nvcc] + NVCC_COMMON + extra + ["-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            jobs.append(cmd)
    # the translation units compile independently: run them side by side
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as pool:
        for r in list(pool.map(lambda c: subprocess.run(c, capture_output=True, text=True), jobs)):
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise subprocess.CalledProcessError(r.returncode, r.args)
    if force or _stale(LIB, objs):
        cmd = [nvcc, "-shared", "-Xcompiler", "-fPIC"] + ARCH + objs + ["-o", LIB, "-cudart", "static", "-lz"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
