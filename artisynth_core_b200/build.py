"""Builds libb200fem.so in-tree with nvcc for sm_100a.

The library is the product boundary (C ABI declared in include/b200fem.h);
the Python package only loads it through ctypes.  Every source compiles to
its own object (in parallel, into csrc/_build/) and nvcc links them; no
device code crosses file boundaries, so no relocatable device code is
needed.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(CSRC, "_build")
LIB = os.path.join(HERE, "libb200fem.so")
SOURCES = ["api.cu", "kernels.cu", "pcg.cu", "pcg_cluster.cu", "tet_rows.cu", "attach.cu", "point_cons.cu", "setup.cpp", "serve.cpp"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "-ccbin", "g++",
]


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(HERE, "..", "include", "b200fem.h"))
    return [h for h in hs if os.path.exists(h)]


def _stale(target, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(p) > t for p in deps)


def needs_build() -> bool:
    deps = [os.path.join(CSRC, s) for s in SOURCES] + _headers()
    return _stale(LIB, deps)


def build(force: bool = False, verbose: bool = False, extra=None) -> str:
    if not force and not needs_build():
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    hdrs = _headers()
    jobs = []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(OBJ, os.path.splitext(s)[0] + ".o")
        if force or extra or _stale(obj, [src] + hdrs):
            jobs.append([NVCC, *FLAGS, *(extra or []), "-c", "-o", obj, src])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        return subprocess.run(cmd, capture_output=not verbose, text=True)

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(run, jobs))
    for cmd, r in zip(jobs, results):
        if r.returncode != 0:
            if r.stderr:
                sys.stderr.write(r.stderr)
            raise subprocess.CalledProcessError(r.returncode, cmd)
        if r.stderr and verbose is False and "ptxas info" in r.stderr:
            sys.stderr.write(r.stderr)
    objs = [os.path.join(OBJ, os.path.splitext(s)[0] + ".o") for s in SOURCES]
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB, *objs]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else None)
