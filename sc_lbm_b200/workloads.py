"""Seeded synthetic workloads of the sc_lbm configurations (host side).

Each generator returns plain numpy data (masks as int32 0/1 ``[y*nx + x]``,
populations as float64 in the reference layout ``f[i*N + y*nx + x]``) plus the
physical parameters, so the same inputs feed the GPU domain, the batch, the
drop-in classes and the CPU checks.  Random numbers come from a splitmix64
stream indexed by node, identical on every machine and numpy version.

Configurations (lattice sizes and parameters of the reference's benchmark
drivers, scaled as the project's measurement plan states):

* ``poiseuille``  -- 200 x 50 channel, walls at y = 0 and 49, tau = 1,
  rho = 1, body force 1e-6 along x (laminar_flow_x_dir.cpp:17-68);
* ``laplace``     -- 256 x 256 periodic, a disk of component 1 (rho 2.0 inside,
  0.06 outside; component 2 the reverse), G = 0.9, +-1e-3 noise
  (laplace_law.cpp:67-133 with a disk instead of a square);
* ``drainage``    -- 2048 x 1024 porous medium of non-overlapping disks
  (radius 8-20, porosity ~0.6), walls top and bottom, G = 0.9, Gs = -+0.2,
  force 1e-5 along x on component 1, component 1 in the left 10%;
* ``ensemble``    -- 512 two-component domains, Nx in {64..512}, Ny in
  {64..256} (multiples of 16), disks to porosity 0.5-0.9, G in [0.8, 1.2],
  Gs in [-0.3, 0.3], tau in [0.6, 1.5];
* ``spinodal``    -- periodic, tau = 1, G = 1.2, rho = 1 +- 1% per component
  (phase_separation.cpp:57-116).
* ``contact_angle`` -- 400 x 306, a droplet on a solid shelf, one solid
  interaction parameter per domain (contact_angles.cpp:39-109).
"""
from __future__ import annotations

import numpy as np

CX = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1], dtype=np.float64)
CY = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1], dtype=np.float64)


def uniform(seed: int, n: int, offset: int = 0) -> np.ndarray:
    """n uniforms in [0,1) from splitmix64(seed + offset + i)."""
    with np.errstate(over="ignore"):
        z = (np.arange(offset, offset + n, dtype=np.uint64) + np.uint64(seed) *
             np.uint64(0x9E3779B97F4A7C15) + np.uint64(0x632BE59BD9B4E019))
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


class Stream:
    """Sequential draws from one splitmix64 stream (generated in blocks)."""

    BLOCK = 4096

    def __init__(self, seed: int):
        self.seed, self.pos = int(seed), 0
        self.buf, self.i = uniform(self.seed, self.BLOCK, 0).tolist(), 0

    def next(self) -> float:
        if self.i == len(self.buf):
            self.pos += len(self.buf)
            self.buf, self.i = uniform(self.seed, self.BLOCK, self.pos).tolist(), 0
        self.i += 1
        return self.buf[self.i - 1]

    def uniform(self, lo: float, hi: float) -> float:
        return lo + (hi - lo) * self.next()

    def integer(self, lo: int, hi: int) -> int:
        """integer in [lo, hi]"""
        return lo + min(hi - lo, int(self.next() * (hi - lo + 1)))


def force_vec(g: float, direction: str = "x") -> np.ndarray:
    """Body force g along x or y as the drivers write it: F_i = g/6 c_i
    (laminar_flow_x_dir.cpp:21-24); sum_i F_i c_i = g."""
    return (g / 6.0) * (CX if direction == "x" else CY)


def populations(rho: np.ndarray, mask=None) -> np.ndarray:
    """f_i = rho/9 (the reference initialisers), zero on solid nodes."""
    r = np.asarray(rho, dtype=np.float64).ravel()
    if mask is not None:
        r = np.where(np.asarray(mask).ravel() != 0, r, 0.0)
    return np.tile(r / 9.0, 9)


def disk_mask(nx: int, ny: int, porosity: float, rmin: int, rmax: int, seed: int,
              walls: str | None = None, max_tries: int = 20000, max_misses: int = 300):
    """Non-overlapping disks (add_circle with D = 2r + 1, placed inside the
    bounds the reference's check_object_bounds accepts, one node apart) added
    in seeded random order until the fluid fraction drops to `porosity`, or
    `max_tries` draws were made, or `max_misses` draws in a row found no room
    (jammed).  Runs in the library (sclbm_geometry_add_random_disks) on a
    Geometry with the walls, so the mask follows the reference's rules.
    Returns (mask int32 [ny*nx], number of disks, fluid fraction)."""
    from .api import Geometry
    g = Geometry(nx, ny)
    if walls:
        g.add_walls(1, walls)
    n = g.add_random_disks(porosity, rmin, rmax, seed, wall_rows=1 if walls == "x" else 0,
                           max_tries=max_tries, max_misses=max_misses)
    m = g.get_geom()
    return m, n, float(m.mean())


# ----------------------------------------------------------------------------- configs
def poiseuille(nx: int = 200, ny: int = 50):
    m = np.ones(nx * ny, np.int32).reshape(ny, nx)
    m[0, :] = m[-1, :] = 0
    m = m.ravel()
    return dict(nx=nx, ny=ny, mask=m, tau=1.0, rho0=1.0, g=1e-6,
                force=force_vec(1e-6, "x"), f=populations(np.ones(nx * ny), m))


def laplace(radius: float, nx: int = 256, ny: int = 256, seed: int = 7, G: float = 0.9,
            rho_in: float = 2.0, rho_out: float = 0.06, noise: float = 1e-3):
    N = nx * ny
    yy, xx = np.divmod(np.arange(N), nx)
    inside = (xx - nx / 2) ** 2 + (yy - ny / 2) ** 2 <= radius ** 2
    r1 = np.where(inside, rho_in, rho_out) * (1 + noise * (2 * uniform(seed, N) - 1))
    r2 = np.where(inside, rho_out, rho_in) * (1 + noise * (2 * uniform(seed + 1, N) - 1))
    return dict(nx=nx, ny=ny, mask=np.ones(N, np.int32), tau=(1.0, 1.0), G=G, Gs=(0.0, 0.0),
                f1=populations(r1), f2=populations(r2), radius=radius)


def drainage(nx: int = 2048, ny: int = 1024, seed: int = 11, porosity: float = 0.6):
    m, disks, phi = disk_mask(nx, ny, porosity, 8, 20, seed, walls="x")
    x = np.arange(nx * ny) % nx
    left = x < 0.1 * nx
    r1 = np.where(left, 2.0, 0.06)
    r2 = np.where(left, 0.06, 2.0)
    return dict(nx=nx, ny=ny, mask=m, tau=(1.0, 1.0), G=0.9, Gs=(-0.2, 0.2),
                force1=force_vec(1e-5, "x"), f1=populations(r1, m), f2=populations(r2, m),
                porosity=phi, disks=disks)


def contact_angle(gs_droplet: float, nx: int = 400, ny: int = 306):
    """A droplet on a solid shelf (contact_angles.cpp:39-109): the rectangle
    341 x 20 around (199, 152) is solid; component 1 (the bulk, Gs = -gs) at
    rho 2.0 with 0.06 of component 2 (the droplet, Gs = +gs), except the
    square of half-width 30 around (199, 192), which holds the reverse
    (initialize_fluid_rectangle, src/lbm.cpp:51-99: nodes xc - 29 .. xc + 29,
    yc - 29 .. yc + 29).  G = 0.9, tau = 1, no volume force."""
    from .api import Geometry
    g = Geometry(nx, ny)
    g.add_rectangle(341, 20, 199, 152)
    m = g.get_geom()
    N = nx * ny
    yy, xx = np.divmod(np.arange(N), nx)
    sq = (xx >= 199 - 30 + 1) & (xx <= 199 + 30 - 1) & (yy >= 192 - 30 + 1) & (yy <= 192 + 30 - 1)
    r1 = np.where(sq, 0.06, 2.0)
    r2 = np.where(sq, 2.0, 0.06)
    return dict(nx=nx, ny=ny, mask=m, tau=(1.0, 1.0), G=0.9, Gs=(-gs_droplet, gs_droplet),
                f1=populations(r1, m), f2=populations(r2, m), gs_droplet=gs_droplet)


def spinodal(nx: int, ny: int, seed: int = 101, amp: float = 0.01):
    N = nx * ny
    f = [populations(1.0 + amp * (2.0 * uniform(seed + k, N) - 1.0)) for k in range(2)]
    return dict(nx=nx, ny=ny, mask=np.ones(N, np.int32), tau=(1.0, 1.0), G=1.2, Gs=(0.0, 0.0),
                f1=f[0], f2=f[1])


def ensemble_draws(k: int, seed: int = 2024, size=None) -> dict:
    """The seeded draws of ensemble domain k: size, target fluid fraction,
    G, Gs, tau, and the arguments of its disk packing."""
    s = Stream(seed * 100003 + k)
    if size is None:
        nx = 16 * s.integer(4, 32)
        ny = 16 * s.integer(4, 16)
    else:
        nx, ny = size
    phi = s.uniform(0.5, 0.9)
    G = s.uniform(0.8, 1.2)
    gs = s.uniform(-0.3, 0.3)
    tau = s.uniform(0.6, 1.5)
    return dict(nx=nx, ny=ny, phi=phi, G=G, gs=gs, tau=tau,
                disks=dict(porosity=phi, rmin=2, rmax=8, seed=seed * 7919 + k, wall_rows=0,
                           max_tries=4000, max_misses=300))


def ensemble_member(k: int, seed: int = 2024, size=None):
    """Domain k of the seeded ensemble (its own stream: members are
    independent of how many are drawn)."""
    e = ensemble_draws(k, seed, size)
    nx, ny, phi, G, gs, tau = e["nx"], e["ny"], e["phi"], e["G"], e["gs"], e["tau"]
    m, disks, phi_got = disk_mask(nx, ny, phi, 2, 8, seed * 7919 + k, max_tries=4000)
    N = nx * ny
    r1 = 1.0 + 0.01 * (2 * uniform(seed + 3 * k, N) - 1)
    r2 = 1.0 + 0.01 * (2 * uniform(seed + 3 * k + 1, N) - 1)
    return dict(nx=nx, ny=ny, mask=m, tau=(tau, tau), G=G, Gs=(gs, -gs), porosity=phi_got,
                f1=populations(r1, m), f2=populations(r2, m))


def ensemble(n: int = 512, seed: int = 2024):
    return [ensemble_member(k, seed) for k in range(n)]


def params_of(w, sc, rho_ref=(1.0, 1.0)):
    """sclbm_params for a two-component workload dict."""
    F1 = w.get("force1")
    F2 = w.get("force2")
    return sc.make_params(ncomp=2, tau=w["tau"], g_fluid=(w["G"], w["G"]), g_solid=w["Gs"],
                          rho_ref=rho_ref, force=(F1, F2))
