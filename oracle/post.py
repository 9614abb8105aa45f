"""numpy restatements of the reference's post-processing scripts (TEST
INFRASTRUCTURE ONLY): the checkers of the library's on-device measurements.

* ``contact_angle`` -- benchmarks/two_phase_two_components_flows/
  contact_angles/compute_contact_angles.py:45-106, on density fields held in
  memory instead of the loaded text files;
* ``laplace`` -- benchmarks/two_phase_two_components_flows/laplace_law/
  compute_surface_tension.py:64-72 (pressure jump and radius of one droplet);
* ``channel_profile``, ``velocity_stats`` -- scripts/benchmark_utils.py:8-60
  (the analytic channel profile, the largest |u| and the mean nonzero |u|).

Pinned against the scripts themselves: tests/golden/make_contact_angle_golden.py,
tests/golden/make_laplace_golden.py and tests/golden/make_utils_golden.py run
the unmodified scripts on seeded synthetic inputs and record what they compute
(tests/golden/contact_angle_golden.json, laplace_golden.json,
utils_golden.json).
"""
from __future__ import annotations

import numpy as np


def contact_angle(rho_b: np.ndarray, rho_d: np.ndarray, nx: int, ny: int,
                  rho_bulk: float = 2.0, rho_disp: float = 0.06) -> dict:
    """Contact angle of the droplet (density rho_d) on a flat solid below it.

    The interface band (compute_contact_angles.py:46) is rho_b - rho_d <= 0,
    rho_d <= rho_bulk, rho_b > rho_disp.  Its lowest row y2 and the row above,
    y1 (:48-55), give each end of the base: the smallest (left) and largest
    (right) x on both rows, one node apart at least (:62-79), extended by the
    line through them to half a node below the lowest row (:72-90).  The cap
    height is the band's row extent + 0.5 (:96), its radius
    R = (4H^2 + L^2) / (8H) (:99) and the angle atan(L / (2(R - H))) in
    degrees, moved into [0, 180) (:102-106).  Raises ValueError on an empty
    band or a band of one row, where the script's reductions fail.
    """
    rb = np.asarray(rho_b, dtype=np.float64).reshape(ny, nx)
    rd = np.asarray(rho_d, dtype=np.float64).reshape(ny, nx)
    ys, xs = np.where((rb - rd <= 0) & (rd <= rho_bulk) & (rb > rho_disp))
    if ys.size == 0:
        raise ValueError("no interface nodes")
    y2 = int(ys.min())
    y1 = y2 + 1
    row2, row1 = xs[ys == y2], xs[ys == y1]
    if row1.size == 0:
        raise ValueError("no interface nodes above the lowest row")
    xL1, xL2 = float(row1.min()), float(row2.min())
    xR1, xR2 = float(row1.max()), float(row2.max())
    y_base = y2 - 0.5
    if xL1 == xL2:
        xL1 -= 1
    if xR1 == xR2:
        xR1 -= 1
    slope_l = (y1 - y2) / (xL1 - xL2)
    slope_r = (y1 - y2) / (xR1 - xR2)
    inter_l = y2 - slope_l * xL2
    inter_r = y2 - slope_r * xR2
    xL = 1 / slope_l * (y_base - inter_l)
    xR = 1 / slope_r * (y_base - inter_r)
    L = xR - xL
    H = float(ys.max() - ys.min()) + 0.5
    R = (4 * H * H + L * L) / (8 * H)
    with np.errstate(divide="ignore"):
        theta = float(np.degrees(np.arctan(np.float64(L) / (2 * (R - H)))))
    if theta < 0:
        theta += 180
    return {"theta": theta, "L": L, "H": H, "R": R, "xL": xL, "xR": xR, "y_min": y2,
            "y_max": int(ys.max()), "band_nodes": int(ys.size)}


def laplace(rho_b: np.ndarray, rho_d: np.ndarray, nx: int, ny: int, G: float = 0.9,
            p_in=(200, 200), p_out=(370, 370), rho_bulk: float = 1.9,
            rho_disp: float = 0.06) -> dict:
    """Pressure jump and radius of a droplet (density rho_d) in the bulk fluid.

    p = (rho_b + rho_d)/3 + G/3 rho_b rho_d (compute_surface_tension.py:65),
    dp = p[p_in] - p[p_out] with the points given as [row, column] (:66), the
    radius as half the row extent and half the column extent of the band
    rho_d - rho_b < 0, rho_disp < rho_b <= rho_bulk, averaged (:69-72).
    """
    rb = np.asarray(rho_b, dtype=np.float64).reshape(ny, nx)
    rd = np.asarray(rho_d, dtype=np.float64).reshape(ny, nx)
    p = 1.0 / 3.0 * (rb + rd) + G / 3.0 * rb * rd
    dp = p[p_in[0], p_in[1]] - p[p_out[0], p_out[1]]
    sel = np.where((rd - rb < 0) & (rb <= rho_bulk) & (rb > rho_disp))
    if sel[0].size == 0:
        raise ValueError("no interface nodes")
    Rx = (np.amax(sel[0]) - np.amin(sel[0])) / 2.0
    Ry = (np.amax(sel[1]) - np.amin(sel[1])) / 2.0
    return {"dp": float(dp), "R": float(0.5 * (Rx + Ry)), "R_rows": float(Rx), "R_cols": float(Ry),
            "band_nodes": int(sel[0].size)}


def channel_profile(nx: int, ny: int, dPdL: float, direction: str, mu: float):
    """Analytic laminar profile between plates one node thick
    (benchmark_utils.py:8-52): lateral node positions and u, the half width
    h = (n_lat - 2)/2, u = u_max (1 - (y/h)^2), u_max = dPdL h^2 / (2 mu), and
    a zero at each wall node."""
    n_lat = ny if direction == "x" else nx
    h = (n_lat - 2.0) / 2.0
    u_max = dPdL * (h * h) / (2.0 * mu)
    lat = np.arange(-h, h) + 0.5
    u = u_max * (1.0 - (lat / h) * (lat / h))
    return (np.concatenate([[lat[0] - 1], lat, [lat[-1] + 1]]),
            np.concatenate([[0.0], u, [0.0]]))


def velocity_stats(ux: np.ndarray, uy: np.ndarray) -> dict:
    """Largest |u| and mean of the nonzero |u| (vel_mag and ave,
    benchmark_utils.py:54-60)."""
    m = np.sqrt(np.asarray(ux) * ux + np.asarray(uy) * uy).ravel()
    nz = m[np.flatnonzero(m)]
    return {"max_u": float(m.max()), "mean_nonzero_u": float(np.mean(nz)), "nonzero": int(nz.size)}
