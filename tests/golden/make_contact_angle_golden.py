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
is recorded.

A second run feeds the script, under the key -0.2, the final densities of the
reduced contact-angle benchmark (golden case contact_120x90: 2,000 steps of
the compiled reference, oracle/_ref) written by the reference itself
(Fluid::write_density, six significant digits) -- the text route the
reference's own post-processing takes; its angle is recorded as
``reduced_benchmark``.  Needs the reference sources; the committed fixture is
what the tests read.
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

import contact_fields  # noqa: E402
import cases  # noqa: E402

sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import pyoracle  # noqa: E402

SCRIPT = os.path.join(REF_ROOT, "benchmarks/two_phase_two_components_flows/contact_angles/"
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


def run_script(keys, write) -> list[float]:
    """Run the script on the files write(dir, key) puts under output/."""
    with tempfile.TemporaryDirectory() as tmp:
        os.makedirs(os.path.join(tmp, "output"))
        for k in keys:
            write(os.path.join(tmp, "output"), k)
        out = subprocess.run([sys.executable, "-c", RUNNER, SCRIPT], cwd=tmp, check=True,
                             capture_output=True, text=True).stdout
    # the script prints, per key, the list of files it found and then the angle
    thetas = [float(line) for line in out.splitlines() if line and not line.startswith("[")]
    if len(thetas) != len(keys):
        raise SystemExit("unexpected script output:\n" + out)
    return thetas


def write_synthetic(outdir, k):
    rb, rd = contact_fields.fields(k)
    for name, v in (("bulk", rb), ("droplet", rd)):
        np.savetxt(os.path.join(outdir, f"contact_angle_{name}_fluid_final_{k}.txt"), v, fmt="%.17g")


def reference_density_text(f, nx, ny, path):
    """The reference's Fluid::write_density of populations f (oracle/_ref)."""
    with tempfile.TemporaryDirectory() as tmp:
        fbin = os.path.join(tmp, "f.bin")
        np.asarray(f, dtype="<f8").tofile(fbin)
        subprocess.run([pyoracle.REF_RUNNER, "text", fbin, str(nx), str(ny),
                        os.path.join(tmp, "ref")], check=True, stdout=subprocess.DEVNULL)
        with open(os.path.join(tmp, "ref_rho.txt")) as src, open(path, "w") as dst:
            dst.write(src.read())


def main() -> None:
    if not pyoracle.have_ref():
        pyoracle.build(ref=True)
    keys = list(contact_fields.CASES)
    thetas = run_script(keys, write_synthetic)
    # the reduced benchmark (bulk = component 1, droplet = component 2)
    case = cases.all_cases()["contact_120x90"]
    res = pyoracle.run_ref(case)

    def write_reduced(outdir, k):
        if k != "-0.2":
            write_synthetic(outdir, k)
            return
        for name, comp in (("bulk", "c1_f"), ("droplet", "c2_f")):
            reference_density_text(res[comp], case["nx"], case["ny"],
                                   os.path.join(outdir, f"contact_angle_{name}_fluid_final_{k}.txt"))

    reduced = run_script(keys, write_reduced)[keys.index("-0.2")]
    golden = {"script": "benchmarks/two_phase_two_components_flows/contact_angles/"
                        "compute_contact_angles.py",
              "fields": "tests/golden/contact_fields.py",
              "theta_deg": dict(zip(keys, thetas)),
              "reduced_benchmark": {"case": "contact_120x90", "bulk": "component 1",
                                    "text": "Fluid::write_density of the compiled reference",
                                    "theta_deg": reduced}}
    with open(os.path.join(HERE, "contact_angle_golden.json"), "w") as fh:
        json.dump(golden, fh, indent=1)
        fh.write("\n")
    print(json.dumps({k: golden[k] for k in ("theta_deg", "reduced_benchmark")}, indent=1))


if __name__ == "__main__":
    main()
