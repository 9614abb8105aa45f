"""Text output in the reference's format, checked on the CPU.

The library writes lattice fields the way Fluid::write_var does
(src/fluid.cpp:303-343 through LbmIO::write_vector): rows of nx values, 6
significant digits, a space after every value, and write_var's own corner
cases (empty file for a 1 x 1 lattice, one value dropped when nx == 1).  The
reference itself, compiled from its sources (oracle/_ref), writes the files of
the same populations; the bytes must agree.  The fields are computed by the
oracle (bit-exact with the reference), so any difference is the formatting.
"""
import os
import subprocess

import numpy as np
import pytest

import cases


def _fields(oracle, f, nx, ny):
    L = oracle.lib()
    N = nx * ny
    g = np.ones(N, np.uint8)
    rho, ux, uy = np.zeros(N), np.zeros(N), np.zeros(N)
    L.orc_compute_density(N, oracle._p(f), oracle._p(rho))
    L.orc_compute_velocities(N, oracle._p(g), oracle._p(f), oracle._p(rho), oracle._p(ux),
                             oracle._p(uy))
    return rho, ux, uy


def _populations(seed, nx, ny):
    # wide range of magnitudes and both signs, so exponents and rounding show
    N = nx * ny
    u = cases.uniform(seed, 9 * N)
    scale = 10.0 ** np.floor(12 * cases.uniform(seed + 1, 9 * N) - 6)
    return (u - 0.3) * scale + 1.0 / 9.0 * (u > 0.5)


@pytest.mark.parametrize("nx,ny", [(5, 4), (17, 3), (1, 6), (1, 2), (1, 1), (7, 1), (2, 1)])
def test_text_matches_reference_bytes(sclbm, oracle, tmp_path, nx, ny):
    if not oracle.have_ref():
        pytest.skip("the reference was not compiled here (oracle/_ref)")
    f = _populations(7 + nx * 31 + ny, nx, ny)
    fbin = tmp_path / "f.bin"
    f.astype("<f8").tofile(fbin)
    ref = tmp_path / "ref"
    subprocess.run([oracle.REF_RUNNER, "text", str(fbin), str(nx), str(ny), str(ref)], check=True,
                   stdout=subprocess.DEVNULL)
    rho, ux, uy = _fields(oracle, f, nx, ny)
    for name, v in (("rho", rho), ("ux", ux), ("uy", uy)):
        ours = tmp_path / f"ours_{name}.txt"
        sclbm.write_rows(ours, v, nx, ny)
        assert ours.read_bytes() == (tmp_path / f"ref_{name}.txt").read_bytes(), name
    N = nx * ny
    for i in range(9):
        ours = tmp_path / f"ours_f_{i}.txt"
        sclbm.write_rows(ours, f[i * N:(i + 1) * N], nx, ny)
        assert ours.read_bytes() == (tmp_path / f"ref_f_{i}.txt").read_bytes(), i


def test_write_var_corner_cases(sclbm, tmp_path):
    p = tmp_path / "a.txt"
    sclbm.write_rows(p, [3.5], 1, 1)
    assert p.read_bytes() == b""
    sclbm.write_rows(p, [1.0, 2.0, 3.0, 4.0], 1, 4)   # nx == 1 drops the next-to-last value
    assert p.read_text() == "1 \n2 \n4 \n"
    sclbm.write_rows(p, [1.0, 2.5e-7, -3.0, 123456789.0], 2, 2)
    assert p.read_text() == "1 2.5e-07 \n-3 1.23457e+08 \n"


def test_read_rows_round_trip_and_errors(sclbm, tmp_path):
    v = np.linspace(-2, 3, 12)
    p = tmp_path / "r.txt"
    sclbm.write_rows(p, v, 4, 3)
    back = sclbm.read_rows(p, 4, 3)
    assert np.array_equal(back, np.array([float(f"{x:.6g}") for x in v]))
    with pytest.raises(IndexError):
        sclbm.read_rows(p, 5, 3)   # rows of 4 values
    with pytest.raises(IndexError):
        sclbm.read_rows(p, 4, 4)   # only 3 rows
    with pytest.raises(RuntimeError):
        sclbm.read_rows(tmp_path / "missing.txt", 4, 3)
    with pytest.raises(RuntimeError):
        sclbm.write_rows(tmp_path / "no" / "dir.txt", v, 4, 3)
