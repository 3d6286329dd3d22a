"""Build the hyteg_b200 shared library in-tree with nvcc for sm_100a.

Usage: python -m hyteg_b200.build   (or hyteg_b200.build.build() from Python)
Produces hyteg_b200/libhyteg_b200.so next to this file.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libhyteg_b200.so")
OBJ_DIR = os.path.join(HERE, "_build")

SOURCES = ["topology.cpp", "mesh_gen.cpp", "p1_kernels.cu", "p1_elementwise.cu", "p2_constant.cu", "capi.cu", "serve.cu", "dataexport.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build hyteg_b200")
    return cand


def _needs_build(obj, src, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src] + deps)


def build(verbose: bool = False, force: bool = False) -> str:
    nvcc = _nvcc()
    os.makedirs(OBJ_DIR, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "hyteg_b200.h"))
    common = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-I", CSRC, "-I", os.path.join(ROOT, "include")]
    jobs = []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(OBJ_DIR, s + ".o")
        flags = common + ARCH
        if s.endswith(".cpp"):
            flags = flags + ["-x", "cu"]
        cmd = [nvcc, *flags, "-c", src, "-o", obj]
        if force or _needs_build(obj, src, headers):
            jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {cmd[-3]}:\n{r.stdout}\n{r.stderr}")
        return r.stderr

    with ThreadPoolExecutor(max_workers=min(4, max(1, len(jobs)))) as ex:
        for out in ex.map(run, jobs):
            if verbose and out:
                print(out)
    objs = [os.path.join(OBJ_DIR, s + ".o") for s in SOURCES]
    if force or jobs or not os.path.exists(LIB):
        cmd = [nvcc, "-shared", *ARCH, "-o", LIB, *objs, "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
