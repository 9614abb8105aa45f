"""Generate the golden fixtures from the compiled reference (oracle/_ref).

    python tests/golden/make_golden.py [case ...]

For every case of tests/golden/cases.py it runs the unmodified reference
library (LBMFluids/sc_lbm compiled from its own sources by oracle/Makefile,
driven by oracle/ref_runner.cpp) and records, per output array, the SHA-256
of its little-endian bytes (golden_digests.json).  The arrays of the few
smallest cases are stored in full (golden_arrays.npz) so a mismatch can be
located.  Needs the reference sources (it builds oracle/_ref when missing);
the committed fixtures are what the tests read.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

from oracle import pyoracle  # noqa: E402
import cases  # noqa: E402


def digest(a: np.ndarray) -> str:
    a = np.ascontiguousarray(a)
    a = a.astype("<f8") if a.dtype.kind == "f" else a.astype("<i4")
    return hashlib.sha256(a.tobytes()).hexdigest()


def main() -> None:
    """All cases, or only those named on the command line (the digests of the
    others are kept from the committed fixture)."""
    if not pyoracle.have_ref():
        pyoracle.build(ref=True)
    names = sys.argv[1:]
    out, arrays = {}, {}
    if names:
        with open(os.path.join(HERE, "golden_digests.json")) as fh:
            out = json.load(fh)["cases"]
        with np.load(os.path.join(HERE, "golden_arrays.npz")) as z:
            arrays = {k: z[k] for k in z.files}
    for name, case in list(cases.all_cases().items()) + list(cases.long_cases().items()):
        if names and name not in names:
            continue
        res = pyoracle.run_ref(case)
        out[name] = {k: [digest(v), int(v.size)] for k, v in sorted(res.items())}
        if name in cases.FULL_ARRAY_CASES:
            for k, v in res.items():
                arrays[f"{name}/{k}"] = v
        print(f"{name:32s} {len(res):3d} arrays  error={int(res['error'][0])}")
    with open(os.path.join(HERE, "golden_digests.json"), "w") as fh:
        json.dump({"generator": "oracle/_ref/sclbm_ref_runner (reference compiled from its "
                                "own sources, g++ -std=c++11 -O3)", "cases": out}, fh, indent=1,
                  sort_keys=True)
    np.savez_compressed(os.path.join(HERE, "golden_arrays.npz"), **arrays)


if __name__ == "__main__":
    main()
