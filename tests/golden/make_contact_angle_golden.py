"""Generate tests/golden/contact_angle_golden.json by running the reference's
own contact-angle script on the synthetic fields of contact_fields.py.

    python tests/golden/make_contact_angle_golden.py

The unmodified script
(benchmarks/two_phase_two_components_flows/contact_angles/
compute_contact_angles.py, read from the reference checkout) runs in a
scratch directory holding output/contact_angle_{bulk,droplet}_fluid_final_
<key>.txt for the eight keys it iterates over, written with 17 significant
digits so that np.loadtxt reads the fields back exactly.  Its plotting module
and matplotlib are replaced by no-op stubs; the angle it prints for each key
is recorded.  Needs the reference sources; the committed fixture is what the
tests read.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import contact_fields  # noqa: E402

SCRIPT = ("/root/reference/benchmarks/two_phase_two_components_flows/contact_angles/"
          "compute_contact_angles.py")

RUNNER = r"""
import runpy, sys, types
vis = types.ModuleType("visualization")
vis.plot_3D_flat = lambda *a, **k: None
sys.modules["visualization"] = vis
mpl = types.ModuleType("matplotlib")
plt = types.ModuleType("matplotlib.pyplot")
mpl.pyplot = plt
sys.modules.setdefault("matplotlib", mpl)
sys.modules.setdefault("matplotlib.pyplot", plt)
runpy.run_path(sys.argv[1], run_name="__main__")
"""


def main() -> None:
    keys = list(contact_fields.CASES)
    with tempfile.TemporaryDirectory() as tmp:
        os.makedirs(os.path.join(tmp, "output"))
        for k in keys:
            rb, rd = contact_fields.fields(k)
            for name, v in (("bulk", rb), ("droplet", rd)):
                np.savetxt(os.path.join(tmp, "output", f"contact_angle_{name}_fluid_final_{k}.txt"),
                           v, fmt="%.17g")
        out = subprocess.run([sys.executable, "-c", RUNNER, SCRIPT], cwd=tmp, check=True,
                             capture_output=True, text=True).stdout
    # the script prints, per key, the list of files it found and then the angle
    thetas = [float(line) for line in out.splitlines() if line and not line.startswith("[")]
    if len(thetas) != len(keys):
        raise SystemExit("unexpected script output:\n" + out)
    golden = {"script": "benchmarks/two_phase_two_components_flows/contact_angles/"
                        "compute_contact_angles.py",
              "fields": "tests/golden/contact_fields.py",
              "theta_deg": dict(zip(keys, thetas))}
    with open(os.path.join(HERE, "contact_angle_golden.json"), "w") as fh:
        json.dump(golden, fh, indent=1)
        fh.write("\n")
    print(json.dumps(golden["theta_deg"], indent=1))


if __name__ == "__main__":
    main()
