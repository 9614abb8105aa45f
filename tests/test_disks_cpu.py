"""The native seeded disk packer (sclbm_geometry_add_random_disks) against a
plain numpy restatement of the same random sequential addition (CPU).

Both draw the splitmix64 stream of sc_lbm_b200/workloads.py, reject disks
that leave the bounds or come within one node of a solid, stop at the target
solid fraction, the try limit or a run of failed draws, and build the mask
with add_circle -- so the masks must be identical.
"""
import numpy as np
import pytest


def _python_disks(sc, W, nx, ny, porosity, rmin, rmax, seed, walls, max_tries, max_misses):
    s = W.Stream(seed)
    occ = np.zeros((ny, nx), dtype=bool)
    wall_rows = 0
    if walls == "x":
        occ[0, :] = occ[-1, :] = True
        wall_rows = 1
    yy, xx = np.mgrid[0:ny, 0:nx]
    disks, solid, tries, misses = [], occ.sum(), 0, 0
    target = (1.0 - porosity) * nx * ny
    while solid < target and tries < max_tries and misses < max_misses:
        tries += 1
        misses += 1
        r = s.integer(rmin, rmax)
        xc = s.integer(r, nx - 1 - r)
        yc = s.integer(r + wall_rows, ny - 1 - r - wall_rows)
        if xc - r < 0 or yc - r < 0 or xc + r >= nx or yc + r >= ny:
            continue
        y0, y1 = max(0, yc - r - 1), min(ny, yc + r + 2)
        x0, x1 = max(0, xc - r - 1), min(nx, xc + r + 2)
        win = (yy[y0:y1, x0:x1] - yc) ** 2 + (xx[y0:y1, x0:x1] - xc) ** 2 <= (r + 1.5) ** 2
        if np.any(occ[y0:y1, x0:x1] & win):
            continue
        occ[y0:y1, x0:x1] |= win
        misses = 0
        disks.append((2 * r + 1, xc, yc))
        solid += np.pi * (r + 0.5) ** 2
    g = sc.Geometry(nx, ny)
    if walls:
        g.add_walls(1, walls)
    for D, xc, yc in disks:
        g.add_circle(D, xc, yc)
    return g.get_geom(), len(disks)


@pytest.mark.parametrize("nx,ny,phi,rmin,rmax,seed,walls,tries,misses", [
    (512, 256, 0.6, 8, 20, 11, "x", 20000, 300),     # drainage-like
    (224, 96, 0.7, 2, 8, 7919, None, 4000, 300),     # ensemble member
    (64, 64, 0.5, 2, 8, 3, None, 4000, 300),         # jams before the target
    (40, 30, 0.2, 5, 30, 5, "x", 500, 50),           # radii larger than the lattice allows
    (96, 96, 1.0, 2, 4, 1, None, 100, 10),           # nothing to place
])
def test_native_packer_matches_restatement(sclbm, nx, ny, phi, rmin, rmax, seed, walls, tries,
                                           misses):
    from sc_lbm_b200 import workloads as W
    want, nwant = _python_disks(sclbm, W, nx, ny, phi, rmin, rmax, seed, walls, tries, misses)
    got, ngot, frac = W.disk_mask(nx, ny, phi, rmin, rmax, seed, walls=walls, max_tries=tries,
                                  max_misses=misses)
    assert ngot == nwant
    assert np.array_equal(got, want)
    assert frac == float(want.mean())


def test_native_packer_arguments(sclbm):
    g = sclbm.Geometry(32, 32)
    with pytest.raises(ValueError):
        g.add_random_disks(1.5, 2, 4, 1)
    with pytest.raises(ValueError):
        g.add_random_disks(0.5, 5, 4, 1)
