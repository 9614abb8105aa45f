"""The numpy restatement of the reference's contact-angle script
(oracle/post.py) against what the unmodified script printed on the same
synthetic fields and on the reduced benchmark's density files written by the
compiled reference (tests/golden/contact_angle_golden.json, made by
make_contact_angle_golden.py), its failure cases, and the contact-angle
workload's initial state against the oracle's rectangle initialiser (CPU).
"""
import json
import os

import numpy as np
import pytest

import contact_fields
from oracle import post

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "contact_angle_golden.json")


def test_restatement_matches_reference_script():
    with open(GOLDEN) as fh:
        golden = json.load(fh)["theta_deg"]
    assert set(golden) == set(contact_fields.CASES)
    for key, theta in golden.items():
        rb, rd = contact_fields.fields(key)
        ny, nx = rb.shape
        got = post.contact_angle(rb, rd, nx, ny)
        assert got["theta"] == theta, key


def test_restatement_covers_both_sides_of_90_degrees():
    with open(GOLDEN) as fh:
        th = list(json.load(fh)["theta_deg"].values())
    assert min(th) < 90.0 < max(th) and 90.0 in th


def test_restatement_failures():
    nx, ny = 20, 10
    rb, rd = np.full((ny, nx), 2.0), np.full((ny, nx), 0.06)
    with pytest.raises(ValueError):
        post.contact_angle(rb, rd, nx, ny)
    rb[4, 3:9], rd[4, 3:9] = 0.7, 1.3
    with pytest.raises(ValueError):
        post.contact_angle(rb, rd, nx, ny)
    rb[5, 4:8], rd[5, 4:8] = 0.7, 1.3
    r = post.contact_angle(rb, rd, nx, ny)
    assert r["y_min"] == 4 and r["y_max"] == 5 and r["band_nodes"] == 10


def test_contact_workload_matches_reference_initialiser(sclbm, oracle):
    """workloads.contact_angle: the shelf of contact_angles.cpp:62-63 and the
    populations of initialize_fluid_rectangle (src/lbm.cpp:51-99)."""
    from sc_lbm_b200 import workloads as W
    w = W.contact_angle(-0.3)
    case = dict(nx=400, ny=306, geom=[("rectangle", 341, 20, 199, 152)], mode="two",
                fluid1=(1.0, 0.9, 0.3), fluid2=(1.0, 0.9, -0.3),
                init=("rectangle", 2.0, 2.0, 0.06, 0.06, 199, 192, 30, 30),
                force=(0, [0.0] * 9), steps=0)
    r = oracle.run_case(case)
    assert np.array_equal(np.asarray(w["mask"]).ravel(), r["mask"])
    assert np.array_equal(w["f1"], r["c1_f"])
    assert np.array_equal(w["f2"], r["c2_f"])
    assert w["Gs"] == (0.3, -0.3)


def test_reduced_benchmark_angle_matches_reference_text_route(oracle):
    """The reduced contact-angle benchmark (golden case contact_120x90): the
    restatement on the oracle's final densities (bit-identical to the compiled
    reference's) gives the angle the reference's script printed on the density
    files the reference itself wrote in six-digit text."""
    import cases
    with open(GOLDEN) as fh:
        want = json.load(fh)["reduced_benchmark"]
    case = cases.all_cases()[want["case"]]
    r = oracle.run_case(case)
    got = post.contact_angle(r["c1_rho_final"], r["c2_rho_final"], case["nx"], case["ny"])
    assert got["theta"] == want["theta_deg"]
