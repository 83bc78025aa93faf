"""Builds the native parts of eqtl_b200 in-tree.

    python -m eqtl_b200.build          # libeqtl_cuda.so + the eqtl CLI

* eqtl_b200/lib/libeqtl_cuda.so : every CUDA kernel (sm_100a only) and the C
  ABI declared in include/eqtl_b200.h;
* eqtl_b200/bin/eqtl            : the host C++ program with the reference's
  command line, linked against the library (rpath $ORIGIN/../lib).

Objects are rebuilt only when a source or header is newer than them.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
HOST = os.path.join(PKG, "host")
OBJ = os.path.join(PKG, "_obj")
LIB = os.path.join(PKG, "lib", "libeqtl_cuda.so")
BIN = os.path.join(PKG, "bin", "eqtl")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = "/usr/bin/g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stderr


def build_lib(verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "*.h*")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        [os.path.join(ROOT, "include", "eqtl_b200.h")]
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    jobs = []
    for s in srcs:
        o = os.path.join(OBJ, os.path.basename(s) + ".o")
        if _newer(o, [s] + headers):
            cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-ccbin", CXX, "-Xcompiler", "-fPIC",
                   "-Xptxas", "-v", "-c", s, "-o", o]
            jobs.append(cmd)
    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        logs = list(ex.map(_run, jobs))
    if verbose:
        for lg in logs:
            sys.stderr.write(lg)
    objs = [os.path.join(OBJ, os.path.basename(s) + ".o") for s in srcs]
    if jobs or _newer(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-ccbin", CXX, "-o", LIB, *objs, "-lcublas", "-lcusolver",
              "-Xlinker", "-rpath=/usr/local/cuda/lib64"])
    return LIB


def build_cli() -> str:
    srcs = sorted(glob.glob(os.path.join(HOST, "*.cpp")))
    if not srcs:
        return ""
    os.makedirs(os.path.dirname(BIN), exist_ok=True)
    headers = glob.glob(os.path.join(HOST, "*.hpp")) + [os.path.join(ROOT, "include", "eqtl_b200.h"),
                                                         os.path.join(CSRC, "tstat.hpp")]
    if _newer(BIN, srcs + headers + [LIB]):
        _run([CXX, "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC, *srcs, "-o", BIN,
              "-L" + os.path.dirname(LIB), "-leqtl_cuda", "-lz", "-Wl,-rpath,$ORIGIN/../lib"])
    return BIN


def build(verbose: bool = False) -> None:
    build_lib(verbose)
    build_cli()


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)
