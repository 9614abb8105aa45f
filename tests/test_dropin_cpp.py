"""The C++ drop-in: the reference's Geometry / Fluid / LBM classes
(sc_lbm_b200/host/include, implemented in libsclbm_b200.so over the C ABI).

One driver source, oracle/ref_runner.cpp, is written only against the
reference's public classes (include/geometry.h, include/fluid.h,
include/lbm.h).  Built against the reference's own sources it produced the
golden digests; built here against the drop-in headers and linked to
libsclbm_b200.so it must reproduce them bit for bit -- the claim that a
reference user recompiles unchanged and gets the same numbers.

CPU tests: the runner builds and links; the geometry half (host code behind
the ABI) matches every golden mask and error; the reference's own benchmark
drivers compile and link against the drop-in headers (when its sources are
present).  GPU tests: every simulation case bit for bit, and the fused
LBM::step extension against the per-method sequence (tests/cpp/dropin_step.cpp).
"""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

import cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "sc_lbm_b200")
HOST_INC = os.path.join(PKG, "host", "include")
RUNNER_SRC = os.path.join(ROOT, "oracle", "ref_runner.cpp")
STEP_SRC = os.path.join(ROOT, "tests", "cpp", "dropin_step.cpp")
REF_SRC = os.environ.get("SCLBM_REF", "/root/reference")

ALL = cases.all_cases()
MASKS = {k: v for k, v in ALL.items() if v["mode"] == "mask"}
SIM = {k: v for k, v in ALL.items() if v["mode"] != "mask"}


def _link_flags():
    return [f"-L{PKG}", "-lsclbm_b200", f"-Wl,-rpath,{PKG}"]


def _compile(src, out, extra_inc=()):
    cmd = ["g++", "-std=c++11", "-O2", "-Wall", f"-I{HOST_INC}", *[f"-I{d}" for d in extra_inc],
           src, "-o", out, *_link_flags()]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, f"{' '.join(cmd)}\n{r.stdout}\n{r.stderr}"
    return out


@pytest.fixture(scope="module")
def lib_built(sclbm):
    from sc_lbm_b200 import capi
    assert os.path.exists(capi.LIB_PATH)
    return capi.LIB_PATH


@pytest.fixture(scope="module")
def runner(lib_built, tmp_path_factory):
    """oracle/ref_runner.cpp built against the drop-in headers."""
    d = tmp_path_factory.mktemp("dropin")
    return _compile(RUNNER_SRC, str(d / "dropin_runner"))


def _golden():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "golden_digests.json")) as fh:
        return json.load(fh)["cases"]


def _digest(a):
    import hashlib
    a = np.ascontiguousarray(a)
    a = a.astype("<f8") if a.dtype.kind == "f" else a.astype("<i4")
    return hashlib.sha256(a.tobytes()).hexdigest()


def _assert_golden(name, res):
    want = _golden()[name]
    keys = [k for k in want if k in res]
    assert keys, f"{name}: no outputs"
    missing = [k for k in want if k not in res]
    assert not missing, f"{name}: the drop-in runner did not write {missing}"
    bad = [k for k in keys if _digest(res[k]) != want[k][0]]
    assert not bad, f"{name}: differ from the reference: {bad}"


# ------------------------------------------------------------------ CPU
def test_dropin_runner_builds(runner):
    assert os.access(runner, os.X_OK)


@pytest.mark.parametrize("name", sorted(MASKS))
def test_dropin_geometry_matches_reference(runner, name):
    """Geometry construction through the drop-in: masks and exception types
    (error codes) equal the reference's, including partly built masks."""
    from oracle import pyoracle
    res = pyoracle.run_ref(MASKS[name], runner=runner)
    _assert_golden(name, res)


def _reference_drivers():
    if not os.path.isdir(os.path.join(REF_SRC, "benchmarks")):
        return []
    out = []
    for dirpath, _, files in os.walk(os.path.join(REF_SRC, "benchmarks")):
        for f in files:
            if f.endswith(".cpp"):
                p = os.path.join(dirpath, f)
                txt = open(p, errors="replace").read()
                # drivers of the library (not its test harness)
                if re.search(r'#include\s+"(\.\./)+include/lbm\.h"', txt) and "test_utils" not in txt:
                    out.append(os.path.relpath(p, REF_SRC))
    return sorted(out)


@pytest.mark.parametrize("rel", _reference_drivers() or ["(reference sources absent)"])
def test_reference_driver_compiles_against_dropin(lib_built, tmp_path, rel):
    """The reference's benchmark drivers compile and link, unchanged, against
    the drop-in headers: their relative includes ("../include/lbm.h",
    "../../../include/geometry.h") are pointed at sc_lbm_b200/host/include by
    placing a copy of the driver at the matching depth of a scratch tree."""
    if rel.startswith("("):
        pytest.skip("reference sources are not present on this machine")
    src = os.path.join(REF_SRC, rel)
    txt = open(src, errors="replace").read()
    depth = max(len(m) // 3 for m in re.findall(r'#include\s+"((?:\.\./)+)include/', txt))
    os.symlink(HOST_INC, tmp_path / "include")
    d = tmp_path
    for k in range(depth - 1):
        d = d / f"d{k}"
    d = d / "drv"
    d.mkdir(parents=True)
    local = d / os.path.basename(src)
    shutil.copy(src, local)
    _compile(str(local), str(d / "driver"))


# ------------------------------------------------------------------ GPU
@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(SIM))
def test_dropin_bit_exact(runner, name):
    """Every simulation case through the drop-in classes: every array the
    reference driver dumps (f, f_eq, rho, u, u_eq, F_repulsive, F_solid) is
    bit-identical to the reference's."""
    from oracle import pyoracle
    res = pyoracle.run_ref(SIM[name], runner=runner)
    _assert_golden(name, res)


@pytest.mark.gpu
def test_dropin_fused_step_extension(lib_built, tmp_path):
    """LBM::step (one fused kernel per step) equals the per-method sequence
    bit for bit, across host edits of populations between steps; the text
    output of write_density carries the density at 6 significant digits."""
    exe = _compile(STEP_SRC, str(tmp_path / "dropin_step"))
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    f1 = np.fromfile(tmp_path / "f1.bin", dtype="<f8").reshape(9, 48, 96)
    rho_txt = np.loadtxt(tmp_path / "rho1.txt")
    assert rho_txt.shape == (48, 96)
    np.testing.assert_allclose(rho_txt, f1.sum(axis=0), rtol=6e-6, atol=1e-12)
