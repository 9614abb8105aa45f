"""Generate tests/golden/laplace_golden.json by running the reference's own
Laplace-law script on the synthetic droplets of laplace_fields.py.

    python tests/golden/make_laplace_golden.py

The unmodified script
(benchmarks/two_phase_two_components_flows/laplace_law/
compute_surface_tension.py, read from the reference checkout) runs in a
scratch directory holding output/{bulk,droplet}_<key>_final.txt for the seven
keys it iterates over, written with 17 significant digits so that np.loadtxt
reads the fields back exactly.  Its plotting modules are replaced by no-op
stubs; the pressure jumps, radii and fit it computes are read from the
script's own variables after it ran.  Needs the reference sources; the
committed fixture is what the tests read.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference checkout whose unmodified scripts generate the fixtures
REF_ROOT = os.environ.get("SCLBM_REF", "/root/reference")
sys.path.insert(0, HERE)

import laplace_fields  # noqa: E402

SCRIPT = os.path.join(REF_ROOT, "benchmarks/two_phase_two_components_flows/laplace_law/"
                      "compute_surface_tension.py")

RUNNER = r"""
import json, runpy, sys, types
class _Any:
    def __getattr__(self, name):
        return self
    def __call__(self, *a, **k):
        return self
vis = types.ModuleType("visualization")
vis.plot_3D_flat = lambda *a, **k: None
sys.modules["visualization"] = vis
mpl = types.ModuleType("matplotlib")
mpl.pyplot = _Any()
sys.modules.setdefault("matplotlib", mpl)
sys.modules.setdefault("matplotlib.pyplot", mpl.pyplot)
g = runpy.run_path(sys.argv[1], run_name="__main__")
print("RESULT " + json.dumps({"cases": g["cases"], "p_final": g["p_final"].tolist(),
                              "R_final": g["R_final"].tolist(),
                              "fit": g["fit_params"].tolist()}))
"""


def main() -> None:
    with tempfile.TemporaryDirectory() as tmp:
        os.makedirs(os.path.join(tmp, "output"))
        for k in laplace_fields.CASES:
            rb, rd = laplace_fields.fields(k)
            for name, v in (("bulk", rb), ("droplet", rd)):
                np.savetxt(os.path.join(tmp, "output", f"{name}_{k}_final.txt"), v, fmt="%.17g")
        out = subprocess.run([sys.executable, "-c", RUNNER, SCRIPT], cwd=tmp, check=True,
                             capture_output=True, text=True).stdout
    line = [l for l in out.splitlines() if l.startswith("RESULT ")][-1]
    res = json.loads(line[len("RESULT "):])
    golden = {"script": "benchmarks/two_phase_two_components_flows/laplace_law/"
                        "compute_surface_tension.py",
              "fields": "tests/golden/laplace_fields.py", **res}
    with open(os.path.join(HERE, "laplace_golden.json"), "w") as fh:
        json.dump(golden, fh, indent=1)
        fh.write("\n")
    print(json.dumps(res, indent=1))


if __name__ == "__main__":
    main()
