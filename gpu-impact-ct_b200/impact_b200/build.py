"""Build libimpact_b200.so (the CUDA kernels and the C ABI) in-tree for sm_100a.

    python -m impact_b200.build        (from gpu-impact-ct_b200/)

Each translation unit is compiled separately with nvcc and linked into one shared library
next to this file; a unit is rebuilt only when its sources are newer than its object.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(ROOT, "csrc")
INCLUDE = os.path.join(os.path.dirname(ROOT), "include")
OBJ = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "libimpact_b200.so")

SOURCES = ["kernels.cu", "stencil25d.cu", "solver.cu", "engine.cu", "step.cu", "capi.cu", "prof.cu", "noalloc.cu", "rhs.cu", "ibm.cu", "march.cu", "coeffs.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
              "--expt-relaxed-constexpr", "-I", CSRC, "-I", INCLUDE]


def _nvcc():
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _ccbin():
    for c in ("/usr/bin/g++",):
        if os.path.exists(c):
            return ["-ccbin", c]
    return []


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return hs


def _compile(src, extra, verbose):
    s = os.path.join(CSRC, src)
    o = os.path.join(OBJ, src + ".o")
    newest = max([os.path.getmtime(s)] + [os.path.getmtime(h) for h in _headers()])
    if os.path.exists(o) and os.path.getmtime(o) >= newest:
        return o
    cmd = [_nvcc()] + _ccbin() + ARCH + NVCC_FLAGS + extra + ["-c", s, "-o", o]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr.strip():
        print(r.stderr, flush=True)
    return o


def build(verbose=False, ptxas_info=False):
    os.makedirs(OBJ, exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra, verbose), SOURCES))
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(o) for o in objs):
        return LIB
    cmd = [_nvcc()] + _ccbin() + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="-v" in sys.argv))
