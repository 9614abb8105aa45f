"""The numpy restatement of the reference's Laplace-law post-processing
(oracle/post.py: laplace) against the pressure jumps, radii and fit the
unmodified script computed on the same synthetic droplets
(tests/golden/laplace_golden.json, made by make_laplace_golden.py) (CPU).

The GPU tests check the device measurement (sclbm_domain_laplace_measure)
against this restatement's arithmetic on the downloaded fields.
"""
import json
import os

import numpy as np

import laplace_fields
from oracle import post

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "laplace_golden.json")


def test_restatement_matches_reference_script():
    with open(GOLDEN) as fh:
        g = json.load(fh)
    dps, Rs = [], []
    for key, dp_want, R_want in zip(g["cases"], g["p_final"], g["R_final"]):
        rb, rd = laplace_fields.fields(key)
        got = post.laplace(rb, rd, laplace_fields.NX, laplace_fields.NY, G=0.9,
                           p_in=(200, 200), p_out=(370, 370), rho_bulk=1.9, rho_disp=0.06)
        assert got["dp"] == dp_want, key
        assert got["R"] == R_want, key
        dps.append(got["dp"])
        Rs.append(got["R"])
    fit = np.polyfit(1 / np.asarray(Rs), np.asarray(dps), 1)
    assert fit.tolist() == g["fit"]


def test_gpu_checker_equals_restatement():
    """The inline checker of tests/test_gpu_analysis.py computes the same
    numbers as the pinned restatement."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "gpu_analysis", os.path.join(os.path.dirname(__file__), "test_gpu_analysis.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    for key in ("80", "20"):
        rb, rd = laplace_fields.fields(key)
        want = post.laplace(rb, rd, 400, 400, 0.9, (200, 200), (370, 370), 1.9, 0.06)
        # the checker takes (x, y) points and flattened fields
        dp, R, band = mod._numpy_laplace(rb.ravel(), rd.ravel(), 0.9, 1.9, 0.06, (200, 200),
                                         (370, 370), 400, 400)
        assert dp == want["dp"] and R == want["R"] and band == want["band_nodes"]
