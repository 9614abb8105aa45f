"""Seeded synthetic density fields of a droplet resting on a solid shelf, the
inputs of the contact-angle fixtures (deterministic integer geometry: the same
fields on every machine and numpy version).

A field is ``ny x nx``: the shelf occupies rows [shelf_y0, ys) (both densities
0, as the reference's solid nodes), the droplet is the part of the disk of
radius ``r`` around (xc, yc) at rows y >= ys.  Nodes of the droplet within two
nodes of its rim form the interface band (rho_d 1.3, rho_b 0.7), nodes deeper
inside hold the droplet phase (rho_d 2.0, rho_b 0.06, or 0.0601 at the seeded
"wet" nodes, which then join the band), all others the bulk phase (rho_d 0.06,
rho_b 2.0).
"""
from __future__ import annotations

import numpy as np

# key -> (nx, ny, shelf_y0, ys, xc, yc, r, wet_fraction, seed); the keys are
# the solid-interaction parameters the reference's script iterates over
CASES = {
    "-0.4": (120, 90, 20, 30, 60, 20, 24, 0.0, 1),    # flat cap, angle well below 90
    "-0.3": (120, 90, 20, 30, 58, 25, 22, 0.0, 2),
    "-0.2": (120, 90, 20, 30, 61, 30, 20, 0.0, 3),    # hemisphere: steep lowest rows
    "-0.1": (140, 100, 10, 16, 70, 22, 25, 0.02, 4),
    "0.1": (140, 100, 10, 16, 69, 30, 21, 0.0, 5),    # angle above 90
    "0.2": (100, 100, 30, 40, 50, 55, 18, 0.05, 6),
    "0.3": (100, 100, 30, 40, 47, 60, 22, 0.0, 7),
    "0.4": (160, 120, 5, 12, 81, 38, 30, 0.01, 8),
}


def fields(key: str) -> tuple[np.ndarray, np.ndarray]:
    """(rho_bulk_fluid, rho_droplet_fluid), each ny x nx float64."""
    nx, ny, shelf_y0, ys, xc, yc, r, wet, seed = CASES[key]
    yy, xx = np.mgrid[0:ny, 0:nx]
    d2 = (xx - xc) ** 2 + (yy - yc) ** 2
    drop = (d2 <= r * r) & (yy >= ys)
    band = drop & (d2 > (r - 2) ** 2)
    core = drop & ~band
    solid = (yy >= shelf_y0) & (yy < ys)
    rb = np.full((ny, nx), 2.0)
    rd = np.full((ny, nx), 0.06)
    rb[band], rd[band] = 0.7, 1.3
    rb[core], rd[core] = 0.06, 2.0
    if wet > 0:
        h = ((xx * 73856093) ^ (yy * 19349663) ^ (seed * 83492791)) % 1000
        rb[core & (h < int(wet * 1000))] = 0.0601
    rb[solid] = rd[solid] = 0.0
    return rb, rd
