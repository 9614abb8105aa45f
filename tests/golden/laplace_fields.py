"""Seeded synthetic droplet fields for the Laplace-law fixtures
(deterministic integer geometry: the same fields on every machine and numpy
version).

Field ``key`` (the radius label the reference's script iterates over) is a
400 x 400 lattice holding a disk of the droplet fluid of radius r around
(cy, cx): nodes within two nodes of its rim form the interface band (rho_d
0.8, rho_b 1.2), nodes deeper inside hold the droplet phase (rho_d 2 + 0.3/r,
rho_b 0.06: a Laplace-like pressure excess), all others the bulk phase
(rho_d 0.06, rho_b 2.0).
"""
from __future__ import annotations

import numpy as np

# key -> (r, cy, cx)
CASES = {"80": (80, 200, 200), "70": (70, 199, 202), "60": (60, 201, 198),
         "50": (50, 200, 203), "40": (40, 197, 200), "30": (30, 202, 201),
         "20": (20, 200, 199)}
NX = NY = 400


def fields(key: str) -> tuple[np.ndarray, np.ndarray]:
    """(rho_bulk_fluid, rho_droplet_fluid), each NY x NX float64."""
    r, cy, cx = CASES[key]
    yy, xx = np.mgrid[0:NY, 0:NX]
    d2 = (yy - cy) ** 2 + (xx - cx) ** 2
    drop = d2 <= r * r
    band = drop & (d2 > (r - 2) ** 2)
    core = drop & ~band
    rb = np.full((NY, NX), 2.0)
    rd = np.full((NY, NX), 0.06)
    rb[band], rd[band] = 1.2, 0.8
    rb[core], rd[core] = 0.06, 2.0 + 0.3 / r
    return rb, rd
