"""Generate tests/golden/utils_golden.json from the reference's own
scripts/benchmark_utils.py (imported from the reference checkout):
channel_flow_analytical for the Poiseuille configuration and a second channel,
vel_mag / ave on seeded velocity fields with zeros.

    python tests/golden/make_utils_golden.py

Needs the reference sources; the committed fixture is what the tests read.
"""
from __future__ import annotations

import importlib.util
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference checkout whose unmodified scripts generate the fixtures
REF_ROOT = os.environ.get("SCLBM_REF", "/root/reference")
UTILS = os.path.join(REF_ROOT, "scripts/benchmark_utils.py")

# (nx, ny, dPdL, direction, mu)
CHANNELS = [(200, 50, 1e-6, "x", 1.0 / 6.0), (30, 80, 2.5e-5, "y", 0.1)]


def velocity_fields(seed: int, nx: int = 37, ny: int = 23):
    """Seeded u fields (splitmix64 of the node index) with a third of the
    nodes at rest."""
    n = np.arange(nx * ny, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = n + np.uint64(seed) * np.uint64(0x9E3779B97F4A7C15) + np.uint64(0x632BE59BD9B4E019)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    u = (z >> np.uint64(11)).astype(np.float64) / 9007199254740992.0
    ux = (u - 0.5) * 1e-3
    uy = (0.5 - u * u) * 2e-3
    rest = (z % np.uint64(3)) == 0
    ux[rest] = 0.0
    uy[rest] = 0.0
    return ux.reshape(ny, nx), uy.reshape(ny, nx)


def main() -> None:
    spec = importlib.util.spec_from_file_location("benchmark_utils", UTILS)
    bu = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bu)
    out = {"script": "scripts/benchmark_utils.py", "channels": [], "velocity": []}
    for nx, ny, dpdl, d, mu in CHANNELS:
        lat, u = bu.channel_flow_analytical(nx, ny, dpdl, d, mu)
        out["channels"].append({"args": [nx, ny, dpdl, d, mu], "lat": lat.tolist(), "u": u.tolist()})
    for seed in (3, 4):
        ux, uy = velocity_fields(seed)
        m = bu.vel_mag(ux, uy)
        out["velocity"].append({"seed": seed, "max_u": float(m.max()), "mean_nonzero_u": float(bu.ave(m))})
    with open(os.path.join(HERE, "utils_golden.json"), "w") as fh:
        json.dump(out, fh, indent=1)
        fh.write("\n")
    print(json.dumps(out["velocity"], indent=1))


if __name__ == "__main__":
    main()
