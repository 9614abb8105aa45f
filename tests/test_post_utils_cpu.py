"""The restatements of the reference's scripts/benchmark_utils.py in
oracle/post.py (analytic channel profile; largest and mean nonzero |u|, the
quantities the device's sclbm_domain_profile / sclbm_domain_velocity_stats
are compared with) against the values the reference's own functions returned
(tests/golden/utils_golden.json, made by make_utils_golden.py) (CPU)."""
import json
import os

import numpy as np
import pytest

import make_utils_golden
from oracle import post

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "utils_golden.json")


def _golden():
    with open(GOLDEN) as fh:
        return json.load(fh)


def test_channel_profile_matches_reference():
    for ch in _golden()["channels"]:
        lat, u = post.channel_profile(*ch["args"])
        assert lat.tolist() == ch["lat"]
        assert u.tolist() == ch["u"]


def test_velocity_stats_match_reference():
    for v in _golden()["velocity"]:
        ux, uy = make_utils_golden.velocity_fields(v["seed"])
        got = post.velocity_stats(ux, uy)
        assert got["max_u"] == v["max_u"]
        # the reference averages the transposed field: same terms, other order
        assert got["mean_nonzero_u"] == pytest.approx(v["mean_nonzero_u"], rel=1e-14)
        assert 0 < got["nonzero"] < ux.size


def test_poiseuille_check_uses_the_reference_profile():
    """The 200 x 50 channel check of the GPU tests (h = (ny - 2)/2,
    u = g h^2 / (2 mu) (1 - (y/h)^2) at y = -h + 0.5 ...) is the reference's
    profile without its wall zeros."""
    g, ny, mu = 1e-6, 50, (1.0 - 0.5) / 3.0
    h = (ny - 2) / 2.0
    lat = np.arange(-h, h) + 0.5
    ua = g * h * h / (2 * mu) * (1 - (lat / h) ** 2)
    _, u = post.channel_profile(200, ny, g, "x", mu)
    np.testing.assert_allclose(ua, u[1:-1], rtol=1e-15, atol=0)
