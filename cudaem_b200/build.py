"""Builds libcudaem_b200.so in-tree for sm_100a.

Sources under cudaem_b200/csrc are compiled with nvcc (CUDA files) and g++
(host files) into cudaem_b200/_build/*.o and linked into
cudaem_b200/libcudaem_b200.so.  Objects are rebuilt only when a source or a
header is newer than the object.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcudaem_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["kernels.cu", "passes_128.cu", "passes_256.cu", "passes_512.cu", "passes_1024.cu", "passes_2048.cu",
              "engine.cu", "noalloc.cu"]
CPP_SOURCES = ["host.cpp", "abi.cpp", "tune.cpp"]


def _host_cxx() -> str:
    for cand in ("/usr/bin/g++", shutil.which("g++") or ""):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("no host C++ compiler found")


def _headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh", ".h"))]
    hs.append(os.path.join(INCLUDE, "cudaem_b200.h"))
    return hs


def _stale(obj: str, src: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in [src] + deps)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr, file=sys.stderr)


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> str:
    """Compile every source for sm_100a and link the shared library; returns its path."""
    os.makedirs(BUILD, exist_ok=True)
    cxx = _host_cxx()
    deps = _headers()
    jobs = []
    objs = []
    for f in CU_SOURCES:
        src = os.path.join(CSRC, f)
        obj = os.path.join(BUILD, f + ".o")
        objs.append(obj)
        if force or _stale(obj, src, deps):
            cmd = [NVCC, "-ccbin", cxx, *ARCH, "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
                   "-Xcompiler", "-fPIC,-ffp-contract=off", "-I", INCLUDE, "-c", src, "-o", obj]
            if ptxas_verbose:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append(cmd)
    for f in CPP_SOURCES:
        src = os.path.join(CSRC, f)
        obj = os.path.join(BUILD, f + ".o")
        objs.append(obj)
        if force or _stale(obj, src, deps):
            jobs.append([cxx, "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall",
                         "-I", os.path.join(CUDA_HOME, "include"), "-I", INCLUDE, "-c", src, "-o", obj])
    if jobs:
        with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
            list(ex.map(lambda c: _run(c, verbose), jobs))
    if force or jobs or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        tmp = LIB + ".tmp"
        _run([NVCC, "-ccbin", cxx, *ARCH, "-shared", "-o", tmp, *objs, "-cudart", "static", "-lpthread"], verbose)
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, ptxas_verbose="--ptxas" in sys.argv))
