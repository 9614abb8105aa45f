"""GPU checks of the workload side: the device-side seeded initial state, the
batch with autotuned defaults on an uneven ensemble, and the Poiseuille
channel against its analytic profile.

* sclbm_domain_init_noise writes exactly the state that uploading the host
  generator's populations gives (all three storage forms, porous mask);
* a batch built with the tuned tile shapes (tile_y = NULL, variant 0) advances
  uneven porous domains exactly as stepping each domain alone does;
* the 200 x 50 Poiseuille channel after 10,000 FP64 steps is bit-identical to
  the reference (golden digest) and its centre-line profile matches the
  analytic parabola of half-way bounce-back walls.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
with open(os.path.join(GOLDEN, "golden_digests.json")) as fh:
    DIGESTS = json.load(fh)["cases"]


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).astype("<f8").tobytes()).hexdigest()


@pytest.mark.parametrize("prec_name", ["FP64", "FP32_SHIFTED", "FP16_SHIFTED"])
def test_init_noise_equals_host_upload(sclbm, prec_name):
    from sc_lbm_b200 import workloads as W
    prec = getattr(sclbm, prec_name)
    nx, ny = 150, 70
    m, _, _ = W.disk_mask(nx, ny, 0.7, 3, 6, seed=5, walls="x")
    N = nx * ny
    p = sclbm.make_params(ncomp=2, g_fluid=(0.9, 0.9), g_solid=(0.1, -0.1), rho_ref=(1.1, 0.4))
    host = sclbm.Domain(nx, ny, m, p, prec)
    dev = sclbm.Domain(nx, ny, m, p, prec)
    for comp, (rho0, amp, seed) in enumerate(((1.1, 0.01, 77), (0.4, 0.003, 78))):
        r = rho0 * (1.0 + amp * (2.0 * W.uniform(seed, N) - 1.0))
        host.upload_f(comp, W.populations(r, m))
        dev.init_noise(comp, rho0, amp, seed)
        assert np.array_equal(host.download_f(comp), dev.download_f(comp))
    host.step(5)
    dev.step(5)
    for comp in range(2):
        assert np.array_equal(host.download_f(comp), dev.download_f(comp))


def test_init_noise_matches_spinodal_generator(sclbm):
    from sc_lbm_b200 import workloads as W
    w = W.spinodal(64, 48, seed=101)
    d = sclbm.Domain(64, 48, w["mask"], W.params_of(w, sclbm), sclbm.FP64)
    d.init_noise(0, 1.0, 0.01, 101)
    d.init_noise(1, 1.0, 0.01, 102)
    assert np.array_equal(d.download_f(0), w["f1"])
    assert np.array_equal(d.download_f(1), w["f2"])


@pytest.mark.parametrize("prec_name", ["FP32_SHIFTED", "FP64"])
def test_tuned_batch_equals_individual_domains(sclbm, prec_name):
    from sc_lbm_b200 import workloads as W
    prec = getattr(sclbm, prec_name)
    members = [W.ensemble_member(k, seed=99) for k in range(10)]
    def build():
        doms = []
        for m in members:
            d = sclbm.Domain(m["nx"], m["ny"], m["mask"], W.params_of(m, sclbm), prec)
            d.upload_f(0, m["f1"])
            d.upload_f(1, m["f2"])
            doms.append(d)
        return doms
    batch_doms, solo = build(), build()
    b = sclbm.Batch(batch_doms)  # tuned tile shapes, automatic variant
    b.step(23)
    for d in solo:
        d.step(23)
    for a, c in zip(batch_doms, solo):
        for comp in range(2):
            assert np.array_equal(a.download_f(comp), c.download_f(comp))


def test_poiseuille_10k_reference_and_analytic(sclbm):
    from sc_lbm_b200 import workloads as W
    import gpu_runner
    case = cases.all_cases()["poiseuille_200x50_10k"]
    res = gpu_runner.run_fused(sclbm, case)
    want = DIGESTS["poiseuille_200x50_10k"]
    for k in ("c1_f", "c1_rho_final", "c1_ux_final", "c1_uy_final"):
        assert _digest(res[k]) == want[k][0], k
    w = W.poiseuille()
    nx, ny = w["nx"], w["ny"]
    u = res["c1_ux_final"].reshape(ny, nx)[:, nx // 2]
    nu = (1.0 - 0.5) / 3.0
    h, yc = (ny - 2) / 2.0, (ny - 1) / 2.0
    y = np.arange(1, ny - 1)
    ua = 1e-6 / (2 * nu) * (h * h - (y - yc) ** 2)
    # 10,000 steps are 0.72 viscous times (H^2/nu): the slowest mode has decayed
    # to ~1e-3, and the reference's u = j/rho omits the half-force shift
    assert np.linalg.norm(u[1:-1] - ua) / np.linalg.norm(ua) < 5e-3


def test_laplace_full_size_fp64_matches_reference(sclbm):
    """Configuration 2 at full size (256 x 256, radius 40, 20,000 steps): the
    fused FP64 step on fluid objects and the FP64 domain reproduce the
    compiled reference's populations and final fields bit for bit."""
    import gpu_runner
    name = "laplace_256x256_r40_20k"
    case = cases.long_cases()[name]
    want = DIGESTS[name]
    for res in (gpu_runner.run_fused(sclbm, case), gpu_runner.run_domain(sclbm, case, sclbm.FP64)):
        for k in ("c1_f", "c2_f", "c1_rho_final", "c2_rho_final", "c1_ux_final", "c2_uy_final"):
            assert _digest(res[k]) == want[k][0], k


def test_lattice_beyond_32bit_offsets(sclbm):
    """A lattice whose nine population arrays hold 2^32 elements or more runs
    the 64-bit-offset kernel: 21888^2 FP16 (479 M nodes, 34 GB on the
    device), seeded on the device; two steps conserve each component's mass
    and the periodic lattice stays finite."""
    nx = ny = 21888
    N = nx * ny
    assert 9 * N >= 2 ** 32
    d = sclbm.Domain(nx, ny, np.ones(N, np.int32),
                     sclbm.make_params(ncomp=2, g_fluid=(1.2, 1.2), rho_ref=(1.0, 1.0)),
                     sclbm.FP16_SHIFTED)
    d.init_noise(0, 1.0, 0.01, 5)
    d.init_noise(1, 1.0, 0.01, 6)
    m0 = d.mass_momentum()
    d.step(2)
    m1 = d.mass_momentum()
    assert m1[6] == 0
    for c in (0, 1):
        assert abs(m1[3 * c] - m0[3 * c]) / m0[3 * c] < 1e-3
    del d


@pytest.mark.parametrize("k", [3, 4])
def test_unstable_ensemble_member_blows_up_with_the_reference(sclbm, k):
    """Ensemble members that go non-finite do so at the reference's step: the
    FP64 domain equals the oracle bit for bit one step before (the oracle is
    pinned to the compiled reference at that step, and the reference is shown
    to go non-finite at the next one, tests/test_ensemble_blowup_cpu.py), and
    the monitor reports non-finite populations after the next step."""
    from oracle import pyoracle
    from sc_lbm_b200 import capi, workloads as W
    from test_ensemble_blowup_cpu import BLOWUP, member_case
    s = BLOWUP[k]
    case, m = member_case(k, s - 1)
    want = pyoracle.run_case(case)
    d = sclbm.Domain(m["nx"], m["ny"], m["mask"], W.params_of(m, sclbm), sclbm.FP64)
    d.upload_f(0, m["f1"])
    d.upload_f(1, m["f2"])
    d.step(s - 1)
    for comp, key in ((0, "c1_f"), (1, "c2_f")):
        assert d.download_f(comp).tobytes() == want[key].tobytes(), (k, key)
    d.mass_momentum()  # all finite
    d.step(1)
    with pytest.raises(capi.SclbmNonFinite):
        d.mass_momentum()


def _packing_cases():
    from sc_lbm_b200 import workloads as W
    out = [dict(name="drainage_2048x1024", nx=2048, ny=1024, walls="x",
                disks=dict(porosity=0.6, rmin=8, rmax=20, seed=11, wall_rows=1, max_tries=20000,
                           max_misses=300)),
           dict(name="small_disks_1024", nx=1024, ny=1024, walls=None,
                disks=dict(porosity=0.72, rmin=2, rmax=8, seed=31337, wall_rows=0, max_tries=400000,
                           max_misses=2000))]
    for k in (0, 1, 3, 17, 100, 511):
        e = W.ensemble_draws(k)
        out.append(dict(name=f"ensemble_{k}_{e['nx']}x{e['ny']}", nx=e["nx"], ny=e["ny"], walls=None,
                        disks=e["disks"]))
    return out


@pytest.mark.parametrize("case", _packing_cases(), ids=lambda c: c["name"])
def test_device_packing_equals_host_packer(sclbm, case):
    """Disks placed and rasterised on the device (sclbm_domain_add_random_disks)
    give the host packer's mask node for node (Geometry.add_random_disks, the
    reference's integer circle), the same number of disks, and zero
    populations at the new solid nodes."""
    nx, ny, dk = case["nx"], case["ny"], case["disks"]
    g = sclbm.Geometry(nx, ny)
    if case["walls"]:
        g.add_walls(1, case["walls"])
    base = g.get_geom().copy()
    n_host = g.add_random_disks(**dk)
    want = g.get_geom()
    for prec in (sclbm.FP64, sclbm.FP32_SHIFTED):
        d = sclbm.Domain(nx, ny, base, sclbm.make_params(ncomp=2, g_fluid=(0.9, 0.9)), prec)
        d.init_noise(0, 1.0, 0.01, 5)
        d.init_noise(1, 1.0, 0.01, 6)
        n_dev = d.add_random_disks(**dk)
        assert n_dev == n_host, (case["name"], n_dev, n_host)
        got = d.download_mask()
        assert np.array_equal(got, want), (case["name"], int(np.sum(got != want)))
        solid = want == 0
        for comp in range(2):
            f = d.download_f(comp).reshape(9, -1)
            if prec == sclbm.FP64:
                assert np.all(f[:, solid] == 0.0)
        d.step(3)
        d.mass_momentum()
