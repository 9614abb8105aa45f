"""Shared-memory layout of the ring kernels (sc_lbm_b200/csrc/fused_ring.cuh,
RingLayout), printed by a host-only program compiled with nvcc from the
library's own header and run on the CPU: tensor-copy destinations on
128-byte boundaries, the edge buffer of the form without halo boxes large
enough for both halo lanes' two slots, and the resident CTAs per SM that the
shared memory allows -- the figures the kernels' launch bounds and the design
notes rely on (four FP32 CTAs with halo boxes, five without)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
SMEM_PER_SM = 228 * 1024   # B200 (sm_100): shared memory per SM
RESERVED_PER_CTA = 1024    # shared memory the runtime reserves per resident CTA
ELEM = {"ring_fp64": 8, "ring_fp32": 4, "ring_fp32_edge": 4, "ring_fp16": 2, "batch_fp64": 8,
        "batch_fp32": 4, "batch_fp32_w64": 4, "batch_fp16": 2}


@pytest.fixture(scope="module")
def layouts(tmp_path_factory):
    if not (os.path.exists(NVCC) or shutil.which("nvcc")):
        pytest.skip("nvcc not found")
    exe = str(tmp_path_factory.mktemp("ring") / "ring_layout")
    subprocess.run([NVCC if os.path.exists(NVCC) else "nvcc", "-std=c++17", "-O0",
                    "-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(ROOT, "sc_lbm_b200", "csrc"),
                    "-gencode", "arch=compute_100a,code=sm_100a",
                    os.path.join(ROOT, "tests", "cpp", "ring_layout.cu"), "-o", exe], check=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    keys = ["R", "W", "HB", "A", "comp", "halo", "stage", "pops", "edge_at", "edge", "bars", "bytes"]
    rows = {}
    for line in out.split("\n"):
        if line.strip():
            name, *vals = line.split()
            rows[name] = dict(zip(keys, map(int, vals)))
    return rows


def ctas_by_smem(row):
    return SMEM_PER_SM // (row["bytes"] + RESERVED_PER_CTA)


def test_tensor_copy_destinations_are_aligned(layouts):
    for name, L in layouts.items():
        s = ELEM[name]
        assert L["A"] * s == 16, name                       # a box starts on a 16-byte boundary
        assert L["comp"] % 128 == 0 and L["stage"] % 128 == 0, name
        assert L["comp"] >= 9 * (L["W"] + 2 * L["A"]) * s, name  # one row box per component
        assert 9 * L["A"] * s <= L["halo"], name
        assert L["stage"] == 2 * L["comp"] + (4 * L["halo"] if L["HB"] else 0), name
        assert L["pops"] == L["R"] * L["stage"], name
        assert L["edge_at"] % 16 == 0 and L["bars"] % 16 == 0, name
        assert L["bytes"] >= L["bars"] + 8 * L["R"] + 16, name


def test_edge_buffer_holds_both_halo_lanes_two_slots(layouts):
    for name, L in layouts.items():
        if L["HB"]:
            assert L["edge"] == 0, name
            continue
        s = ELEM[name]
        assert s in (4, 8), name                            # cp.async element copies of 4 or 8 bytes
        # slot of ring row j for lane hl: ((j & 1) * 2 + (0 if left else 1)) * 18 + k * 9 + i
        last = ((1 * 2 + 1) * 18 + 1 * 9 + 8) * s
        assert last + s <= L["edge"], name
        assert L["edge_at"] + L["edge"] <= L["bars"], name


def test_resident_ctas_the_shared_memory_allows(layouts):
    assert ctas_by_smem(layouts["ring_fp32"]) == 4          # 48.9 KB: four CTAs per SM
    assert ctas_by_smem(layouts["ring_fp32_edge"]) == 5     # without halo boxes: five
    assert ctas_by_smem(layouts["ring_fp16"]) >= 6          # the registers' six fit
    assert ctas_by_smem(layouts["ring_fp64"]) >= 3          # the registers' three fit
    assert ctas_by_smem(layouts["batch_fp32"]) >= 5         # uniform batch body: five by registers
    assert ctas_by_smem(layouts["batch_fp16"]) >= 5
    assert ctas_by_smem(layouts["batch_fp64"]) >= 3
