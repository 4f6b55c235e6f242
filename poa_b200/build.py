"""Build the native library in-tree.

    python -m poa_b200.build          # or poa_b200.build.build() from Python

Compiles the CUDA sources for sm_100a only (nvcc cross-compiles without a
GPU), the host C++ sources with g++, and links ``poa_b200/libpoa_b200.so``
(CUDA runtime linked statically) and the drop-in CLI ``poa_b200/minipoa_b200``.
Objects go to ``poa_b200/_build/``; a source newer than its object is rebuilt.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
ROOT = os.path.dirname(PKG)
LIB = os.path.join(PKG, "libpoa_b200.so")
CLI = os.path.join(PKG, "minipoa_b200")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")

CU_SRCS = ["gpu_engine.cu", "batch.cu", "noalloc.cu", "proposer.cu", "intpeak.cu"]
CPP_SRCS = ["graph.cpp", "driver.cpp", "seeding.cpp", "capi.cpp", "multi.cpp", "stream.cpp", "reader.cpp"]
HEADERS = [f for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))] if os.path.isdir(CSRC) else []

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-Xptxas", "-v", "--expt-relaxed-constexpr"]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall", "-Wextra", "-I" + os.path.join(CUDA, "include")]


def _newest_header() -> float:
    hs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "poa_b200.h")]
    return max(os.path.getmtime(h) for h in hs if os.path.exists(h))


def _stale(obj: str, src: str) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return os.path.getmtime(src) > t or _newest_header() > t


def _run(cmd, log=None):
    res = subprocess.run(cmd, capture_output=True, text=True)
    if log is not None:
        with open(log, "w") as fh:
            fh.write(" ".join(cmd) + "\n" + res.stdout + res.stderr)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd[:3]) + " ...")
    return res


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    for s in CU_SRCS:
        src, obj = os.path.join(CSRC, s), os.path.join(BUILD, s + ".o")
        if _stale(obj, src):
            _run([NVCC] + NVCC_FLAGS + ["-c", src, "-o", obj], log=os.path.join(BUILD, s + ".ptxas.txt"))
        objs.append(obj)
    for s in CPP_SRCS:
        src, obj = os.path.join(CSRC, s), os.path.join(BUILD, s + ".o")
        if _stale(obj, src):
            _run(["g++"] + CXX_FLAGS + ["-c", src, "-o", obj])
        objs.append(obj)
    if not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        _run(["g++", "-shared", "-o", LIB] + objs +
             ["-L" + os.path.join(CUDA, "lib64"), "-lcudart_static", "-lz", "-ldl", "-lrt", "-lpthread"])
    main = os.path.join(CSRC, "main.cpp")
    if os.path.exists(main) and (not os.path.exists(CLI) or os.path.getmtime(main) > os.path.getmtime(CLI)
                                 or os.path.getmtime(LIB) > os.path.getmtime(CLI)):
        _run(["g++", "-O2", "-std=c++17", "-I" + CSRC, main, "-o", CLI, "-L" + PKG, "-lpoa_b200",
              "-Wl,-rpath,$ORIGIN", "-lz"])
    if verbose:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    build(verbose=True)
