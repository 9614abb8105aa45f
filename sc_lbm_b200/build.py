"""Build libsclbm_b200.so in-tree with nvcc for sm_100a.

The FP64 operator kernels (ops_fp64.cu) are compiled with ``-fmad=false`` so
every multiply and add rounds separately, in the reference's order; the other
translation units use the default contraction rules.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
HOST = os.path.join(HERE, "host")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libsclbm_b200.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
          f"-I{os.path.join(ROOT, 'include')}", f"-I{os.path.join(HOST, 'include')}"]
EXACT = {"ops_fp64.cu"}


def _sources():
    srcs = []
    for d in (CSRC, os.path.join(HOST, "src")):
        if os.path.isdir(d):
            for f in sorted(os.listdir(d)):
                if f.endswith((".cu", ".cpp")):
                    srcs.append(os.path.join(d, f))
    return srcs


def _headers():
    hs = [os.path.join(ROOT, "include", "sclbm.h")]
    for d in (CSRC, os.path.join(HOST, "include")):
        for r, _, fs in os.walk(d):
            hs += [os.path.join(r, f) for f in fs if f.endswith((".h", ".cuh"))]
    return hs


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = _headers()
    objs = []
    for src in _sources():
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            flags = ARCH + COMMON + (["-fmad=false"] if os.path.basename(src) in EXACT else [])
            if src.endswith(".cpp"):
                flags += ["-x", "cu"] if "csrc" in src else []
            cmd = [NVCC] + flags + ["-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
