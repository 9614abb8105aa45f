"""The ensemble members that go non-finite do so in the reference too.

The 512-domain ensemble samples tau down to 0.6 with |Gs| up to 0.3 and G up
to 1.2; about a third of its members become non-finite in FP64 on the GPU.
Here the unmodified reference (oracle/_ref, compiled from its own sources) runs
two of those members on the CPU with the same mask, parameters and initial
populations: every population is finite one step before the recorded step and
some population is not at that step.  The C restatement gives the same arrays
bit for bit one step before the blow-up, so the GPU's FP64 form (bit-exact
with both, tests/test_gpu_workloads.py) blows up at the same step.  Reference
code: src/lbm.cpp:144-312 (repulsive force, equilibrium velocity, collide).
"""
import numpy as np
import pytest

from oracle import pyoracle
from sc_lbm_b200 import workloads as W

# ensemble member -> first step (1-based) after which a population is non-finite
BLOWUP = {3: 75, 4: 57}


def member_case(k, steps):
    m = W.ensemble_member(k)
    nx, ny = m["nx"], m["ny"]
    mask = np.asarray(m["mask"]).reshape(ny, nx)
    ys, xs = np.nonzero(mask == 0)
    geom = [("solid_node", int(x), int(y)) for y, x in zip(ys, xs)]
    return dict(nx=nx, ny=ny, geom=geom, mode="two",
                fluid1=(m["tau"][0], m["G"], m["Gs"][0]),
                fluid2=(m["tau"][1], m["G"], m["Gs"][1]),
                init=("file", np.concatenate([m["f1"], m["f2"]])),
                force=(0, [0.0] * 9), steps=steps), m


def _finite(out):
    return bool(np.isfinite(out["c1_f"]).all() and np.isfinite(out["c2_f"]).all())


@pytest.mark.skipif(not pyoracle.have_ref(), reason="oracle/_ref not built")
@pytest.mark.parametrize("k", sorted(BLOWUP))
def test_reference_blows_up_at_the_recorded_step(k):
    s = BLOWUP[k]
    before, m = member_case(k, s - 1)
    ref_before = pyoracle.run_ref(before)
    assert (ref_before["mask"] == np.asarray(m["mask"])).all()
    assert _finite(ref_before), f"member {k}: reference non-finite before step {s}"
    ref_at = pyoracle.run_ref(member_case(k, s)[0])
    assert not _finite(ref_at), f"member {k}: reference still finite at step {s}"
    # the restatement agrees bit for bit while the values are finite
    orc = pyoracle.run_case(before)
    for key in ("c1_f", "c2_f"):
        assert orc[key].tobytes() == ref_before[key].tobytes(), (k, key)
    assert not _finite(pyoracle.run_case(member_case(k, s)[0]))
