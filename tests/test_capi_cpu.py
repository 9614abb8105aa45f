"""CPU checks of the C ABI (no GPU needed).

* libsclbm_b200.so loads and exports every function declared in
  include/sclbm.h;
* the host geometry builder behind the ABI reproduces the reference masks
  bit for bit (via the oracle, itself pinned to the reference) and raises the
  reference's exception types on the reference's error cases;
* device entry points fail with a clean status when no device is present.
"""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "sclbm.h")


def declared_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w\s\*]*?\b(sclbm_\w+)\s*\(", txt, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(sclbm):
    from sc_lbm_b200 import capi
    names = declared_functions()
    assert len(names) >= 50
    L = capi.lib()
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # and the binding declares exactly those
    assert sorted(capi.SIGNATURES) == names
    out = subprocess.run(["nm", "-D", "--defined-only", capi.LIB_PATH], capture_output=True,
                         text=True).stdout
    exported = set(re.findall(r"\b(sclbm_\w+)\b", out))
    assert set(names) <= exported


def _apply(geom, cmds):
    for cmd in cmds:
        k = cmd[0]
        if k == "walls":
            geom.add_walls(cmd[1], cmd[2])
        elif k == "rectangle":
            geom.add_rectangle(*cmd[1:5])
        elif k == "square":
            geom.add_square(*cmd[1:4])
        elif k == "ellipse":
            geom.add_ellipse(*cmd[1:5])
        elif k == "circle":
            geom.add_circle(*cmd[1:4])
        elif k == "array_n":
            _, typ, props, b, a1, a2 = cmd
            geom.add_array(props, [[b[0], b[1]], [b[2], b[3]]], [a1, a2], typ)
        elif k == "array_d":
            _, typ, props, b, a1, a2 = cmd
            geom.add_array(props, [[b[0], b[1]], [b[2], b[3]]], a1, a2, typ)
        elif k == "fluid_node":
            geom.set_node_fluid(cmd[1], cmd[2])
        elif k == "solid_node":
            geom.set_node_solid(cmd[1], cmd[2])


ERRORS = {1: ValueError, 2: RuntimeError, 3: IndexError}


@pytest.mark.parametrize("name", sorted(cases.MASK_CASES))
def test_geometry_mask_matches_reference(sclbm, oracle, name):
    case = cases.MASK_CASES[name]
    want, err = oracle.build_mask(case["nx"], case["ny"], case["geom"])
    g = sclbm.Geometry(case["nx"], case["ny"])
    if err:
        with pytest.raises(ERRORS[err]):
            _apply(g, case["geom"])
    else:
        _apply(g, case["geom"])
    assert np.array_equal(g.get_geom(), want.astype(np.int32))
    assert g.Nx() == case["nx"] and g.Ny() == case["ny"]


def test_geometry_random_objects_match_oracle(sclbm, oracle):
    rng = np.random.default_rng(5)
    for trial in range(40):
        nx, ny = int(rng.integers(10, 90)), int(rng.integers(10, 70))
        cmds = []
        for _ in range(int(rng.integers(1, 6))):
            kind = rng.choice(["circle", "ellipse", "rectangle", "square"])
            a, b = int(rng.integers(0, 16)), int(rng.integers(0, 16))
            x, y = int(rng.integers(0, nx)), int(rng.integers(0, ny))
            cmds.append({"circle": ("circle", a, x, y), "square": ("square", a, x, y),
                         "ellipse": ("ellipse", a, b, x, y),
                         "rectangle": ("rectangle", a, b, x, y)}[kind])
        g = sclbm.Geometry(nx, ny)
        mask = np.ones(nx * ny, np.uint8)
        for cmd in cmds:
            m, err = _oracle_step(oracle, mask, nx, ny, cmd)
            if err:
                with pytest.raises(ERRORS[err]):
                    _apply(g, [cmd])
            else:
                _apply(g, [cmd])
            mask = m
            assert np.array_equal(g.get_geom(), mask.astype(np.int32)), (trial, cmd)


def _oracle_step(oracle, mask, nx, ny, cmd):
    import ctypes
    L = oracle.lib()
    m = mask.copy()
    p = m.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
    k = cmd[0]
    if k == "circle":
        rc = L.orc_geom_add_circle(p, nx, ny, *cmd[1:4])
    elif k == "square":
        rc = L.orc_geom_add_square(p, nx, ny, *cmd[1:4])
    elif k == "ellipse":
        rc = L.orc_geom_add_ellipse(p, nx, ny, *cmd[1:5])
    else:
        rc = L.orc_geom_add_rectangle(p, nx, ny, *cmd[1:5])
    return m, rc


def test_device_calls_fail_cleanly_without_gpu(sclbm):
    from sc_lbm_b200 import capi
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    h = C.c_void_p()
    rc = capi.lib().sclbm_fluid_create(4, 4, 1.0, C.byref(h))
    assert rc == capi.E_NO_DEVICE
    assert "device" in capi.last_error()
    with pytest.raises(capi.SclbmError):
        sclbm.Domain(4, 4, np.ones(16, np.int32), sclbm.make_params())
