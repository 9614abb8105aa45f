"""Seeded parity cases shared by the golden-fixture generator and the tests.

The cases restate the reference's own test structure with the compiled
reference (oracle/_ref) as the source of truth instead of its MATLAB files:

* the six test geometries of tests/lbm/create_geometries.cpp:7-92 plus the
  shape and error cases of tests/geometry/{add_objects_test,misc_geom_tests}.cpp;
* single-component runs on those geometries with uniform and multi-direction
  body forces (tests/lbm/{no_force,uni_force,multi_force}_tests.cpp) and a
  per-operator snapshot (tests/lbm/lbm_tests.cpp:12-44);
* the one-step two-component droplet with exaggerated parameters
  (tests/lbm/droplet_tests.cpp:61-252) in its four variants, its per-operator
  snapshot, and multi-step droplet / porous-medium / spinodal runs shaped like
  the benchmark drivers (laplace_law.cpp, droplet_in_a_channel.cpp,
  phase_separation.cpp).

Random initial states use a self-contained splitmix64 generator so they are
identical on every machine and numpy version.
"""
from __future__ import annotations

import numpy as np

CX = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1], dtype=np.float64)
CY = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1], dtype=np.float64)
W = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)


def uniform(seed: int, n: int) -> np.ndarray:
    """n uniforms in [0,1) from splitmix64(seed + i) (bit-reproducible)."""
    with np.errstate(over="ignore"):
        z = (np.arange(n, dtype=np.uint64) + np.uint64(seed) * np.uint64(0x9E3779B97F4A7C15)
             + np.uint64(0x632BE59BD9B4E019))
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def noisy_f(seed: int, nx: int, ny: int, rho: float, amp: float, mask=None) -> np.ndarray:
    """f_i = rho(1 + amp*(2u-1))/9 per node (the reference initialisers' f = rho/9
    shape with a seeded perturbation); zero on solid nodes."""
    N = nx * ny
    r = rho * (1.0 + amp * (2.0 * uniform(seed, N) - 1.0))
    f = np.tile(r / 9.0, 9)
    if mask is not None:
        f = f.reshape(9, N)
        f[:, np.asarray(mask).ravel() == 0] = 0.0
        f = f.ravel()
    return f


def noisy_f_equilibrium(seed: int, nx: int, ny: int, rho: float, amp: float, uamp: float,
                        mask=None) -> np.ndarray:
    """Equilibrium populations of a seeded density and velocity field."""
    N = nx * ny
    r = rho * (1.0 + amp * (2.0 * uniform(seed, N) - 1.0))
    ux = uamp * (2.0 * uniform(seed + 1, N) - 1.0)
    uy = uamp * (2.0 * uniform(seed + 2, N) - 1.0)
    cu = CX[:, None] * ux[None, :] + CY[:, None] * uy[None, :]
    f = W[:, None] * r[None, :] * (1 + 3 * cu + 4.5 * cu * cu - 1.5 * (ux * ux + uy * uy)[None, :])
    if mask is not None:
        f[:, np.asarray(mask).ravel() == 0] = 0.0
    return f.ravel()


def force_vec(g: float, direction: str = "x") -> list[float]:
    """g/6 * c (the drivers' beta*dPdL*{...}, laminar_flow_x_dir.cpp:21-24)."""
    c = CX if direction == "x" else CY
    return list((g / 6.0) * c)


ARRAY_ELLIPSES = ("array_n", "ellipse", [5, 7, 10, 15], [5, 190, 3, 70], 20, 5)

MASK_CASES = {
    "empty_5x10": dict(nx=5, ny=10, geom=[]),
    "x_walls_20x10": dict(nx=20, ny=10, geom=[("walls", 3, "x")]),
    "y_walls_20x10": dict(nx=20, ny=10, geom=[("walls", 3, "y")]),
    "array_no_walls_200x100": dict(nx=200, ny=100, geom=[ARRAY_ELLIPSES]),
    "array_x_walls_200x100": dict(nx=200, ny=100, geom=[("walls", 3, "x"), ARRAY_ELLIPSES]),
    "array_y_walls_200x100": dict(nx=200, ny=100, geom=[("walls", 2, "y"), ARRAY_ELLIPSES]),
    "shapes_64x48": dict(nx=64, ny=48, geom=[("walls", 1, "y"), ("circle", 11, 30, 20),
                                             ("rectangle", 6, 4, 10, 10), ("square", 5, 50, 30),
                                             ("ellipse", 9, 6, 40, 35), ("circle", 8, 20, 38)]),
    "array_spacing_120x90": dict(nx=120, ny=90, geom=[("array_d", "Circle", [7, 10, 10],
                                                       [4, 110, 4, 80], 6, 9),
                                                      ("array_d", "rectangle", [3, 5, 100, 8],
                                                       [95, 118, 5, 60], 2, 3)]),
    "array_square_100x60": dict(nx=100, ny=60, geom=[("array_n", "SQUARE", [4, 6, 6],
                                                      [3, 95, 3, 55], 8, 4)]),
    "nodes_30x20": dict(nx=30, ny=20, geom=[("walls", 2, "x"), ("fluid_node", 5, 0),
                                            ("solid_node", 10, 10), ("solid_node", 11, 10)]),
    # error cases (the reference throws; the mask shows how far it got)
    "err_circle_low_40x40": dict(nx=40, ny=40, geom=[("circle", 11, 4, 20)]),
    "err_circle_high_40x40": dict(nx=40, ny=40, geom=[("circle", 11, 20, 36)]),
    "err_walls_thick_10x8": dict(nx=10, ny=8, geom=[("walls", 9, "x")]),
    "err_walls_dir_10x8": dict(nx=10, ny=8, geom=[("walls", 1, "z")]),
    "err_array_type_50x50": dict(nx=50, ny=50, geom=[("array_n", "triangle", [3, 3, 5, 5],
                                                      [2, 40, 2, 40], 3, 3)]),
    "err_array_outside_50x50": dict(nx=50, ny=50, geom=[("walls", 1, "x"),
                                                        ("array_d", "square", [5, 10, 10],
                                                         [5, 80, 5, 70], 2, 2)]),
}


def single_cases() -> dict:
    c = {}
    for name, geom_name, steps, fx in (
            ("empty_5x10_multi", "empty_5x10", 50, "multi"),
            ("x_walls_20x10_uni", "x_walls_20x10", 200, "x"),
            ("y_walls_20x10_uni", "y_walls_20x10", 200, "y"),
            ("array_x_walls_200x100_uni", "array_x_walls_200x100", 30, "x"),
            ("array_y_walls_200x100_multi", "array_y_walls_200x100", 30, "multi")):
        m = MASK_CASES[geom_name]
        if fx == "multi":
            force = list(1e-3 / 6 * np.array([0, 1, 1, -1, 0, 1, -1, -1, 1]))
        else:
            force = force_vec(1e-3, fx)
        c[name] = dict(nx=m["nx"], ny=m["ny"], geom=m["geom"], mode="single",
                       fluid1=(0.8, 0.0, 0.0), init=("simple", 2.0), force=(1, force),
                       steps=steps)
    # noisy start, tau != 1, no force (tests/lbm/no_force_tests.cpp shape)
    m = MASK_CASES["shapes_64x48"]
    c["shapes_64x48_noise"] = dict(nx=64, ny=48, geom=m["geom"], mode="single",
                                   fluid1=(1.3, 0, 0),
                                   init=("file", noisy_f_equilibrium(11, 64, 48, 1.0, 0.01, 0.02)),
                                   force=(0, [0.0] * 9), steps=40)
    c["poiseuille_200x50"] = dict(nx=200, ny=50, geom=[("walls", 1, "x")], mode="single",
                                  fluid1=(1.0, 0, 0), init=("simple", 1.0),
                                  force=(1, force_vec(1e-6, "x")), steps=100)
    # Poiseuille channel at the full length of the measurement plan (10,000 steps)
    c["poiseuille_200x50_10k"] = dict(nx=200, ny=50, geom=[("walls", 1, "x")], mode="single",
                                      fluid1=(1.0, 0, 0), init=("simple", 1.0),
                                      force=(1, force_vec(1e-6, "x")), steps=10000)
    c["ops1_y_walls_20x10"] = dict(nx=20, ny=10, geom=[("walls", 3, "y")], mode="ops1",
                                   fluid1=(1.0, 0, 0),
                                   init=("file", noisy_f(3, 20, 10, 1.0, 0.05)),
                                   force=(1, force_vec(1e-3, "y")), steps=1)
    return c


def droplet_params(gs: float, flow: bool):
    """tests/lbm/droplet_tests.cpp:222-252 defaults (200x99, y walls)."""
    force = list(-10.5 / 6.0 * np.array([0, 0, -1, 0, 1, -1, -1, 1, 1])) if flow else [0.0] * 9
    return dict(nx=200, ny=99, geom=[("walls", 1, "y")], mode="two",
                fluid1=(1.0, 109.0, gs), fluid2=(1.0, 109.0, -gs),
                init=("rectangle", 2.0, 2.0, 0.6, 0.6, 99, 58, 21, 21),
                force=(3 if flow else 0, force), steps=1)


def two_cases() -> dict:
    c = {
        "droplet_zero_solid_zero_flow": droplet_params(0.0, False),
        "droplet_zero_solid_flow": droplet_params(0.0, True),
        "droplet_solid_zero_flow": droplet_params(20.3, False),
        "droplet_solid_flow": droplet_params(20.3, True),
    }
    ops = dict(droplet_params(20.3, True))
    ops.update(mode="ops2", nx=64, ny=33, init=("rectangle", 2.0, 2.0, 0.6, 0.6, 31, 19, 10, 10))
    c["ops2_droplet_64x33"] = ops
    # Laplace-type droplet (laplace_law.cpp:67-133, smaller), periodic, noisy
    nx = ny = 64
    f1 = noisy_f(21, nx, ny, 0.06, 1e-3)
    f2 = noisy_f(22, nx, ny, 2.0, 1e-3)
    yy, xx = np.divmod(np.arange(nx * ny), nx)
    inside = (xx - 32.0) ** 2 + (yy - 32.0) ** 2 <= 12.0 ** 2
    f1 = f1.reshape(9, -1)
    f2 = f2.reshape(9, -1)
    f1[:, inside], f2[:, inside] = (2.0 / 9) * (1 + 0 * f1[:, inside]), (0.06 / 9) * (1 + 0 * f2[:, inside])
    c["laplace_64x64"] = dict(nx=nx, ny=ny, geom=[], mode="two", fluid1=(1.0, 0.9, 0.0),
                              fluid2=(1.0, 0.9, 0.0),
                              init=("file", np.concatenate([f1.ravel(), f2.ravel()])),
                              force=(0, [0.0] * 9), steps=150)
    # droplet initialiser + solids + unequal tau + force on component 1 only
    c["porous_96x48"] = dict(nx=96, ny=48,
                             geom=[("walls", 1, "x"), ("circle", 9, 30, 20), ("circle", 13, 60, 28),
                                   ("circle", 7, 80, 12), ("square", 5, 15, 35)],
                             mode="two", fluid1=(0.7, 0.9, -0.2), fluid2=(1.3, 0.9, 0.2),
                             init=("droplet", 2.0, 2.0, 0.06, 0.06, 48, 24, 10),
                             force=(1, force_vec(1e-5, "x")), steps=120)
    # spinodal-type (phase_separation.cpp:57-116), periodic, +-1% noise
    nx, ny = 48, 40
    f = np.concatenate([noisy_f(31, nx, ny, 1.0, 0.01), noisy_f(32, nx, ny, 1.0, 0.01)])
    c["spinodal_48x40"] = dict(nx=nx, ny=ny, geom=[], mode="two", fluid1=(1.0, 1.2, 0.0),
                               fluid2=(1.0, 1.2, 0.0), init=("file", f), force=(0, [0.0] * 9),
                               steps=200)
    # flowing droplet (droplet_in_a_channel.cpp:85-156), rectangle init, both fluids forced
    c["channel_80x32"] = dict(nx=80, ny=32, geom=[("walls", 1, "x")], mode="two",
                              fluid1=(1.0, 0.9, -0.294), fluid2=(1.0, 0.9, 0.294),
                              init=("rectangle", 2.0, 2.0, 0.06, 0.06, 40, 16, 14, 15),
                              force=(3, force_vec(1e-4, "x")), steps=100)
    # droplet on a solid shelf (contact_angles.cpp:39-137, reduced): periodic,
    # rectangle initialiser, solid interaction -0.2 / +0.2, no volume force
    c["contact_120x90"] = dict(nx=120, ny=90, geom=[("rectangle", 101, 8, 59, 30)], mode="two",
                               fluid1=(1.0, 0.9, 0.2), fluid2=(1.0, 0.9, -0.2),
                               init=("rectangle", 2.0, 2.0, 0.06, 0.06, 59, 50, 14, 14),
                               force=(0, [0.0] * 9), steps=2000)
    # a component absent from part of the lattice (rho = 0 keeps the previous u_eq)
    nx, ny = 24, 16
    f1 = noisy_f(41, nx, ny, 1.0, 0.01).reshape(9, -1)
    f2 = noisy_f(42, nx, ny, 0.5, 0.01).reshape(9, -1)
    f2[:, : nx * 4] = 0.0
    c["absent_24x16"] = dict(nx=nx, ny=ny, geom=[("walls", 1, "y")], mode="two",
                             fluid1=(1.0, 0.9, 0.1), fluid2=(1.0, 0.9, -0.1),
                             init=("file", np.concatenate([f1.ravel(), f2.ravel()])),
                             force=(0, [0.0] * 9), steps=1)
    return c


def all_cases() -> dict:
    c = {k: dict(v, mode="mask") for k, v in MASK_CASES.items()}
    c.update(single_cases())
    c.update(two_cases())
    return c


def long_cases() -> dict:
    """Full-size runs whose reference results take minutes on the CPU: pinned
    by digests of the compiled reference only (no oracle re-run in the CPU
    suite); the GPU suite compares its FP64 results with them bit for bit."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
    from sc_lbm_b200 import workloads as W
    w = W.laplace(40.0)   # configuration 2: 256 x 256, disk of radius 40, G = 0.9, +-1e-3 noise
    return {"laplace_256x256_r40_20k": dict(
        nx=256, ny=256, geom=[], mode="two", fluid1=(1.0, 0.9, 0.0), fluid2=(1.0, 0.9, 0.0),
        init=("file", np.concatenate([w["f1"], w["f2"]])), force=(0, [0.0] * 9), steps=20000)}


# cases whose full arrays are committed (small enough to diagnose a mismatch)
FULL_ARRAY_CASES = ("x_walls_20x10_uni", "ops1_y_walls_20x10", "absent_24x16", "empty_5x10_multi")
