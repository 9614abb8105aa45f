"""The autotuned size-class table (CPU: host-only lookup, no device needed).

sc_lbm_b200/autotune.py measured the launch shapes on B200 and wrote
sc_lbm_b200/tuning/b200.json; sc_lbm_b200/build.py compiles that file into the
library, and sclbm_tuned_config answers from the compiled table.  These tests
check that the library answers what the committed measurements say.
"""
import json
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TUNING = os.path.join(ROOT, "sc_lbm_b200", "tuning", "b200.json")
PREC = ("fp64", "fp32s", "fp16s")


def _classes():
    with open(TUNING) as fh:
        return json.load(fh)["classes"]


def test_committed_table_is_complete():
    cls = _classes()
    assert len(cls) >= 6
    for c in cls:
        assert c["precision"] in PREC
        for p in PREC:
            assert c["shapes"][p]["variant"] in (2, 3)
            assert c["shapes"][p]["tile_y"] >= 1
        # the recommended storage met the accuracy bound it was chosen under
        assert c["error_vs_fp64"][c["precision"]] <= 1e-5


@pytest.mark.parametrize("k", range(6))
def test_library_answers_from_the_table(sclbm, k):
    c = _classes()[k]
    for nx in (c["nx"][0], c["nx"][1] - 1, c["representative"][0]):
        for ny in (c["ny"][0], c["ny"][1] - 1):
            rec = sclbm.tuned_config(nx, ny)
            assert rec["recommended_precision"] == PREC.index(c["precision"])
            for p, name in enumerate(PREC):
                got = sclbm.tuned_config(nx, ny, precision=p)
                assert (got["variant"], got["tile_y"]) == (c["shapes"][name]["variant"],
                                                           c["shapes"][name]["tile_y"])


def test_sizes_outside_the_table_take_the_nearest_class(sclbm):
    cls = _classes()
    big = max(cls, key=lambda c: (c["nx"][1], c["ny"][1]))
    got = sclbm.tuned_config(100000, 100000, precision=1)
    assert (got["variant"], got["tile_y"]) == (big["shapes"]["fp32s"]["variant"],
                                               big["shapes"]["fp32s"]["tile_y"])
    small = min(cls, key=lambda c: (c["nx"][0], c["ny"][0]))
    got = sclbm.tuned_config(8, 8, precision=1)
    assert (got["variant"], got["tile_y"]) == (small["shapes"]["fp32s"]["variant"],
                                               small["shapes"]["fp32s"]["tile_y"])


def test_invalid_arguments(sclbm):
    with pytest.raises(ValueError):
        sclbm.tuned_config(0, 10)
    with pytest.raises(ValueError):
        sclbm.tuned_config(10, 10, precision=7)


def test_table_generator(tmp_path):
    from sc_lbm_b200 import build
    j = tmp_path / "t.json"
    j.write_text(json.dumps({"classes": [{"nx": [1, 5], "ny": [2, 6], "precision": "fp16s",
                                          "shapes": {"fp64": {"variant": 3, "tile_y": 16},
                                                     "fp32s": {"variant": 2, "tile_y": 8},
                                                     "fp16s": {"variant": 2, "tile_y": 4}}}]}))
    src = build.tuned_table_source(str(j))
    assert "#define SCLBM_TUNED_COUNT 1" in src
    assert "{1, 5, 2, 6, 2, {{3, 16}, {2, 8}, {2, 4}}}," in src
    empty = build.tuned_table_source(str(tmp_path / "missing.json"))
    assert "#define SCLBM_TUNED_COUNT 0" in empty
