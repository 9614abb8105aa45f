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

GEN = os.path.join(BUILD, "gen")
TUNING_JSON = os.path.join(HERE, "tuning", "b200.json")
TUNED_HEADER = os.path.join(GEN, "sclbm_tuned_table.h")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
          f"-I{os.path.join(ROOT, 'include')}", f"-I{os.path.join(HOST, 'include')}", f"-I{GEN}"]
EXACT = {"ops_fp64.cu"}
PRECISIONS = ("fp64", "fp32s", "fp16s")  # sclbm_precision order


def tuned_table_source(path: str = TUNING_JSON) -> str:
    """C table of the autotuner's size classes (empty when no results exist)."""
    import json
    lines = [f"// generated by sc_lbm_b200/build.py from {os.path.relpath(path, ROOT)}",
             "#pragma once", "// included after tuning.h (SclbmTunedClass)"]
    classes, batch = [], {}
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        classes = d.get("classes", [])
        batch = d.get("batch_default", {})
    rows = []
    for c in classes:
        shapes = ", ".join("{%d, %d}" % (int(c["shapes"][p]["variant"]), int(c["shapes"][p]["tile_y"]))
                           for p in PRECISIONS)
        rows.append("    {%d, %d, %d, %d, %d, {%s}}," % (c["nx"][0], c["nx"][1], c["ny"][0], c["ny"][1],
                                                      PRECISIONS.index(c["precision"]), shapes))
    lines.append(f"#define SCLBM_TUNED_COUNT {len(rows)}")
    lines.append("static const SclbmTunedClass kSclbmTuned[%d] = {" % max(1, len(rows)))
    lines += rows or ["    {0, 0, 0, 0, 0, {{0, 0}, {0, 0}, {0, 0}}},"]
    lines.append("};")
    # the body the mixed-ensemble sweep found fastest for batches with solid
    # nodes, per storage precision ({0, 0}: the size-class table decides)
    bd = ", ".join("{%d, %d}" % (int(batch.get(p, {}).get("variant", 0)), int(batch.get(p, {}).get("rows", 0)))
                   for p in PRECISIONS)
    lines.append("static const SclbmTunedShape kSclbmBatchDefault[3] = {%s};" % bd)
    return "\n".join(lines) + "\n"


def _gen_tuning_header():
    os.makedirs(GEN, exist_ok=True)
    src = tuned_table_source()
    old = open(TUNED_HEADER).read() if os.path.exists(TUNED_HEADER) else None
    if src != old:
        with open(TUNED_HEADER, "w") as fh:
            fh.write(src)


def _sources():
    srcs = []
    for d in (CSRC, os.path.join(HOST, "src")):
        if os.path.isdir(d):
            for f in sorted(os.listdir(d)):
                if f.endswith((".cu", ".cpp")):
                    srcs.append(os.path.join(d, f))
    return srcs


def _headers():
    hs = [os.path.join(ROOT, "include", "sclbm.h"), TUNED_HEADER]
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
    _gen_tuning_header()
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
