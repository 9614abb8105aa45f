"""CPU check of the shifted storage algebra used by the GPU FP32/FP16 path.

oracle/shifted_emul.py restates the step in deviation form
(d_i = f_i - w_i*rho_ref, solid force from the mask, neighbour sums as
sum w c drho - rho_ref*S).  Evaluated in float64 it must reproduce the FP64
oracle (itself bit-exact with the reference) to rounding level, so any
difference of the GPU shifted forms from FP64 is storage/arithmetic precision,
not algebra.
"""
import numpy as np
import pytest

import cases

RUNS = cases.all_cases()


@pytest.mark.parametrize("name,steps", [("laplace_64x64", 40), ("channel_80x32", 40),
                                        ("porous_96x48", 40), ("spinodal_48x40", 40),
                                        ("droplet_solid_flow", 1)])
def test_deviation_form_is_exact_in_float64(oracle, name, steps):
    from oracle import shifted_emul
    case = dict(RUNS[name], steps=steps)
    want = oracle.run_case(case)
    g = want["mask"].astype(np.uint8)
    f1, f2 = oracle._init_two(case, g)
    case["_mask"] = g
    for rr in ((1.0, 1.0), (0.3, 1.7)):
        rho = shifted_emul.run(case, f1, f2, steps, rr, store=np.float64, compute=np.float64)
        for k in range(2):
            w = want[f"c{k + 1}_rho_final"]
            m = g.astype(bool)
            err = np.max(np.abs(rho[k][m] - w[m])) / np.mean(np.abs(w[m]))
            assert err < 1e-11, (name, rr, k, err)
