"""Build libkfb.so (the CUDA library behind include/kfb.h) in-tree.

Every translation unit is compiled by nvcc for sm_100a only
(-gencode arch=compute_100a,code=sm_100a) and linked against the CUDA runtime,
cuBLAS of the CUDA toolkit.  The result is
kernelforge_b200/libkfb.so; it is loaded with ctypes by kernelforge_b200._lib.

Usage: python -m kernelforge_b200.build [--force] [-v]
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libkfb.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

SOURCES = ["kfb_common.cpp", "scalar_simt.cu", "scalar_tc.cu", "derivs.cu", "solve.cu",
           "capi.cu", "scalar_noalloc.cu", "tc_gemm.cu", "features.cu",
           "matvec.cu", "repr.cu", "trsv.cu", "ozaki.cu", "chol.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler",
         "-fvisibility=hidden", "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC]


def _headers_mtime() -> float:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(INCLUDE, "kfb.h"))
    return max(os.path.getmtime(h) for h in hs)


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, src + ".o")
    cmd = [NVCC, *ARCH, *FLAGS, "-x", "cu", "-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{res.stderr}")
    if verbose and res.stderr:
        sys.stderr.write(res.stderr)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdr = _headers_mtime()
    stale = []
    for src in SOURCES:
        obj = os.path.join(BUILD, src + ".o")
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < max(
                os.path.getmtime(os.path.join(CSRC, src)), hdr):
            stale.append(src)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        list(ex.map(lambda s: _compile(s, verbose), stale))
    objs = [os.path.join(BUILD, s + ".o") for s in SOURCES]
    if stale or not os.path.exists(LIB):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcublas",
               "-Xlinker", f"-rpath={CUDA_HOME}/lib64"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
