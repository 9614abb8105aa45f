"""GPU parity of libsclbm_b200 against the reference (through the C ABI).

FP64 results are compared BIT FOR BIT with the golden digests recorded from
the compiled reference (tests/golden/golden_digests.json) and with the CPU
oracle; the shifted FP32/FP16 storage forms are compared with the FP64 oracle
within the tolerances stated in each test.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import cases
import gpu_runner

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
with open(os.path.join(GOLDEN, "golden_digests.json")) as fh:
    DIGESTS = json.load(fh)["cases"]
ALL = cases.all_cases()
SIM = {k: v for k, v in ALL.items() if v["mode"] != "mask"}
RUNS = {k: v for k, v in SIM.items() if v["mode"] in ("single", "two")}


def digest(a):
    a = np.ascontiguousarray(a)
    a = a.astype("<f8") if a.dtype.kind == "f" else a.astype("<i4")
    return hashlib.sha256(a.tobytes()).hexdigest()


def assert_golden(name, res, keys=None):
    want = DIGESTS[name]
    keys = [k for k in (keys or want) if k in res and k in want]
    assert keys
    bad = []
    for k in keys:
        if digest(res[k]) != want[k][0]:
            bad.append(k)
    assert not bad, f"{name}: differ from the reference: {bad}"


# ------------------------------------------------------------------ per operator
@pytest.mark.parametrize("name", sorted(SIM))
def test_per_operator_bit_exact(sclbm, name):
    """One C-ABI call per reference method: every array the reference exposes
    (f, f_eq, rho, u, u_eq, F_repulsive, F_solid) is bit-identical."""
    res = gpu_runner.run_ops(sclbm, SIM[name])
    assert_golden(name, res)


# ------------------------------------------------------------------ fused FP64
@pytest.mark.parametrize("name", sorted(RUNS))
def test_fused_fp64_bit_exact(sclbm, name):
    """sclbm_lbm_step / sclbm_lbm_step_single: the single-pass fused kernel
    reproduces the reference's populations and final macroscopic fields."""
    res = gpu_runner.run_fused(sclbm, RUNS[name])
    keys = [k for k in res if k.endswith(("_f", "_final"))]
    assert_golden(name, res, keys)


@pytest.mark.parametrize("name", sorted(RUNS))
def test_domain_fp64_bit_exact(sclbm, name):
    res = gpu_runner.run_domain(sclbm, RUNS[name], sclbm.FP64)
    keys = [k for k in res if k.endswith(("_f", "_final"))]
    assert_golden(name, res, keys)


@pytest.mark.parametrize("tx,tile_y,variant", [(64, 3, 2), (128, 8, 2), (128, 1, 2), (128, 5, 1),
                                               (64, 64, 1), (128, 0, 0), (128, 0, 3), (128, 0, 4),
                                               (128, 3, 4), (128, 0, 5), (128, 4, 5),
                                               (128, 0, 7), (128, 0, 8), (128, 3, 8),
                                               (128, 0, 9), (32, 0, 2), (32, 5, 8), (32, 4, 1),
                                               (128, 0, 11), (128, 0, 12), (128, 0, 13), (128, 0, 14)])
def test_domain_fp64_tiling_invariant(sclbm, tx, tile_y, variant):
    """Kernel variant (pipelined persistent, two pass, register tile, register
    tile with L2 prefetch, ring of bulk row copies at three depths) and tile
    shape do not change a single bit."""
    for name in ("porous_96x48", "spinodal_48x40", "channel_80x32", "droplet_solid_flow"):
        res = gpu_runner.run_domain(sclbm, RUNS[name], sclbm.FP64, variant=variant,
                                    tile_y=tile_y, tx=tx)
        assert_golden(name, res, [k for k in res if k.endswith(("_f", "_final"))])
        res["_domain"].mass_momentum()  # raises if a bounded wait ran out


def test_tiny_and_ragged_lattices(sclbm, oracle):
    """Lattices narrower/shorter than a tile, odd sizes, 1-node-wide periodic wraps."""
    for nx, ny, geom in ((1, 1, []), (1, 7, []), (5, 1, []), (3, 3, [("walls", 1, "y")]),
                         (131, 7, [("walls", 1, "x")]), (127, 129, [("circle", 9, 60, 60)])):
        f = np.concatenate([cases.noisy_f_equilibrium(nx + 3 * ny, nx, ny, 1.0, 0.02, 0.03),
                            cases.noisy_f_equilibrium(nx + 5 * ny, nx, ny, 0.4, 0.02, 0.03)])
        case = dict(nx=nx, ny=ny, geom=geom, mode="two", fluid1=(0.9, 1.1, 0.1),
                    fluid2=(1.2, 1.1, -0.1), init=("file", f),
                    force=(3, cases.force_vec(1e-4, "x")), steps=7)
        want = oracle.run_case(case)
        for runner in (gpu_runner.run_fused,
                       lambda s, c: gpu_runner.run_domain(s, c, s.FP64, tile_y=2, tx=64)):
            got = runner(sclbm, case)
            for k in ("c1_f", "c2_f", "c1_rho_final", "c2_ux_final"):
                assert got[k].tobytes() == want[k].tobytes(), (nx, ny, k)


# ------------------------------------------------------------- shifted forms
def density_errors(a, b, mask):
    """(max |a-b| / mean |b|, ||a-b||_2 / ||b||_2) over fluid nodes.  A two-phase
    component has nodes where its density is ~1e-4 of its bulk value, so the
    error is measured against the component's density scale, not per node."""
    m = mask.astype(bool)
    d = a[m] - b[m]
    return float(np.max(np.abs(d)) / np.mean(np.abs(b[m]))), \
        float(np.linalg.norm(d) / np.linalg.norm(b[m]))


# Tolerances: about twice the errors measured on a B200 (rho_ref = the mean
# initial density of each component).  FP32 rounding of the stored deviations
# (~6e-8 |d_i| per step) accumulates over the run; the rest population closes
# each node's mass, so no systematic drift adds to it.  Spinodal decomposition
# at G = 1.2 amplifies a 1-ulp FP64 perturbation 1e4-fold within 100 steps, so
# it is checked early (20 steps), before that growth dominates.  L2 errors are
# bounded by the max/mean errors, so they share the tolerance.
SHIFTED_CASES = [
    # name, steps, precision, max/mean tol (measured)
    ("laplace_64x64", 150, "FP32_SHIFTED", 3e-6),     # 1.4e-6
    ("channel_80x32", 100, "FP32_SHIFTED", 4e-5),     # 2.1e-5
    ("porous_96x48", 120, "FP32_SHIFTED", 1e-5),      # 5.4e-6
    ("spinodal_48x40", 20, "FP32_SHIFTED", 4e-7),     # 1.9e-7
    ("poiseuille_200x50", 100, "FP32_SHIFTED", 1e-7),
    ("laplace_64x64", 150, "FP16_SHIFTED", 3.5e-2),   # 1.6e-2
    ("channel_80x32", 100, "FP16_SHIFTED", 2e-2),     # 9.1e-3
    ("porous_96x48", 120, "FP16_SHIFTED", 3e-2),      # 1.4e-2
    ("spinodal_48x40", 20, "FP16_SHIFTED", 2.5e-3),   # 1.1e-3
    ("poiseuille_200x50", 100, "FP16_SHIFTED", 1e-6),
]


@pytest.mark.parametrize("name,steps,prec,tol_max", SHIFTED_CASES)
def test_shifted_forms_density_error(sclbm, oracle, name, steps, prec, tol_max):
    """Shifted storage (f_i - w_i*rho_ref, rho_ref = mean initial density) with
    FP32 arithmetic stays within the stated density error of the FP64 oracle."""
    case = dict(RUNS[name], steps=steps)
    want = oracle.run_case(case)
    f0 = gpu_runner._init_f(case, want["mask"].astype(np.uint8))
    N = case["nx"] * case["ny"]
    m = want["mask"].astype(bool)
    rr = tuple(float(f.reshape(9, N).sum(0)[m].mean()) for f in f0) + (1.0,)
    got = gpu_runner.run_domain(sclbm, case, getattr(sclbm, prec), rho_ref=rr[:2])
    for c in ("c1_", "c2_") if case["mode"] == "two" else ("c1_",):
        e_max, e_l2 = density_errors(got[c + "rho_final"], want[c + "rho_final"], want["mask"])
        assert e_max <= tol_max and e_l2 <= tol_max, (name, prec, c, e_max, e_l2)


@pytest.mark.parametrize("name,steps", [("laplace_64x64", 150), ("porous_96x48", 120)])
def test_fp32_shifted_within_1e5_on_stable_two_phase(sclbm, oracle, name, steps):
    """The north-star accuracy bar: FP32-shifted densities within 1e-5 of the
    mean density of the FP64 oracle (bit-exact with the reference) on stable
    two-phase states -- a droplet at rest, and two components with wetting
    walls in a porous medium -- with each component's mean initial density as
    rho_ref."""
    case = dict(RUNS[name], steps=steps)
    want = oracle.run_case(case)
    N = case["nx"] * case["ny"]
    m = want["mask"].astype(bool)
    f0 = gpu_runner._init_f(case, want["mask"].astype(np.uint8))
    rr = tuple(float(f.reshape(9, N).sum(0)[m].mean()) for f in f0)
    got = gpu_runner.run_domain(sclbm, case, sclbm.FP32_SHIFTED, rho_ref=rr)
    for c in ("c1_", "c2_"):
        e_max, _ = density_errors(got[c + "rho_final"], want[c + "rho_final"], want["mask"])
        assert e_max <= 1e-5, (name, c, e_max)


def test_shifted_forms_close_each_nodes_mass(sclbm):
    """The rest population closes every node's mass, so the shifted forms keep
    the total mass of a droplet at rest (no systematic drift from the
    float-rounded weights, whose sum is 1 + 7.5e-9: 2,000 steps of that bias
    drifted ~1e-5 of the mass)."""
    case = dict(RUNS["laplace_64x64"], steps=0)
    for prec, tol in ((sclbm.FP32_SHIFTED, 1e-7), (sclbm.FP16_SHIFTED, 1e-2)):
        d = gpu_runner.make_domain(sclbm, case, prec, rho_ref=(0.4, 1.1))
        m0 = d.mass_momentum()
        d.step(2000)
        m1 = d.mass_momentum()
        for k in range(2):
            assert abs(m1[3 * k] - m0[3 * k]) <= tol * abs(m0[3 * k]), (prec, k, m1[3 * k] / m0[3 * k] - 1)


@pytest.mark.parametrize("variant,tile_y,tx", [(1, 4, 128), (4, 0, 128), (4, 7, 128), (3, 0, 128),
                                               (5, 0, 128), (5, 7, 128), (5, 1, 128), (5, 2, 128),
                                               (6, 0, 128), (6, 1, 128), (6, 5, 128), (6, 64, 128),
                                               (7, 0, 128), (7, 3, 128), (8, 0, 128), (8, 5, 128),
                                               (9, 0, 128), (0, 0, 32), (2, 3, 32), (8, 7, 32),
                                               (11, 0, 128), (12, 0, 128), (13, 0, 128), (14, 0, 128),
                                               (14, 5, 128)])
def test_shifted_variants_match_register_tile(sclbm, variant, tile_y, tx):
    """The shifted forms give the same bytes with every kernel variant and
    tile width."""
    for prec in (sclbm.FP32_SHIFTED, sclbm.FP16_SHIFTED):
        if variant == 3 and prec == sclbm.FP16_SHIFTED:
            continue
        a = gpu_runner.run_domain(sclbm, RUNS["porous_96x48"], prec, rho_ref=(0.5, 1.5))
        b = gpu_runner.run_domain(sclbm, RUNS["porous_96x48"], prec, rho_ref=(0.5, 1.5),
                                  variant=variant, tile_y=tile_y, tx=tx)
        assert a["c1_f"].tobytes() == b["c1_f"].tobytes()
        assert a["c2_f"].tobytes() == b["c2_f"].tobytes()
        b["_domain"].mass_momentum()


# lattices for the ring kernel: partial last strips, strips narrower than the
# 16-byte copy window, single rows, and widths whose rows are not 16-byte
# aligned in some storage forms (those domains take the register tile)
RING_LATTICES = [(8, 3, []), (136, 20, [("walls", 1, "x")]), (264, 9, [("circle", 5, 130, 4)]),
                 (16, 1, []), (4, 7, [("walls", 1, "y")]), (130, 6, [("walls", 1, "x")]),
                 (256, 33, [("circle", 9, 200, 16), ("walls", 1, "x")])]


@pytest.mark.parametrize("variant", [11, 14])
@pytest.mark.parametrize("nx,ny,geom", RING_LATTICES)
def test_ring_kernel_ragged_lattices(sclbm, oracle, nx, ny, geom, variant):
    """Ring kernel on awkward shapes, with halo boxes in its stages (variant
    11) and with the lattice-edge columns copied from global memory (variant
    14, FP32): FP64 bit for bit with the oracle, FP32/FP16 byte for byte with
    the register tile."""
    f = np.concatenate([cases.noisy_f_equilibrium(nx + 3 * ny, nx, ny, 1.0, 0.02, 0.03),
                        cases.noisy_f_equilibrium(nx + 5 * ny, nx, ny, 0.4, 0.02, 0.03)])
    case = dict(nx=nx, ny=ny, geom=geom, mode="two", fluid1=(0.9, 1.1, 0.1),
                fluid2=(1.2, 1.1, -0.1), init=("file", f),
                force=(3, cases.force_vec(1e-4, "x")), steps=9)
    want = oracle.run_case(case)
    got = gpu_runner.run_domain(sclbm, case, sclbm.FP64, variant=variant)
    for k in ("c1_f", "c2_f", "c1_rho_final", "c2_ux_final"):
        assert got[k].tobytes() == want[k].tobytes(), (nx, ny, k)
    got["_domain"].mass_momentum()
    for prec in (sclbm.FP32_SHIFTED, sclbm.FP16_SHIFTED):
        a = gpu_runner.run_domain(sclbm, case, prec, rho_ref=(1.0, 0.4))
        b = gpu_runner.run_domain(sclbm, case, prec, rho_ref=(1.0, 0.4), variant=variant)
        assert a["c1_f"].tobytes() == b["c1_f"].tobytes(), (nx, ny, prec)
        assert a["c2_f"].tobytes() == b["c2_f"].tobytes(), (nx, ny, prec)
        b["_domain"].mass_momentum()


@pytest.mark.parametrize("prec_name,ny,porous,variant", [
    ("FP64", 1024, False, 0), ("FP32_SHIFTED", 1536, False, 0), ("FP32_SHIFTED", 1536, True, 0),
    ("FP16_SHIFTED", 2048, False, 0), ("FP32_SHIFTED", 1536, False, 14), ("FP32_SHIFTED", 1536, True, 14)])
def test_default_kernel_on_lattices_that_fill_the_gpu(sclbm, prec_name, ny, porous, variant):
    """Lattices large enough for the default kernel choice to take the ring
    (4096 wide, 2048 bands of the precision's default height: 16 rows FP64, 24
    FP32, 32 FP16) give the register tile's populations byte for byte after
    three steps, all-fluid and porous with a volume force; so does the FP32
    ring without halo boxes (variant 14), five CTAs per SM."""
    from sc_lbm_b200 import workloads as W
    prec = getattr(sclbm, prec_name)
    nx = 4096
    if porous:
        mask, _, _ = W.disk_mask(nx, ny, 0.7, 4, 12, 17, walls="x")
    else:
        mask = np.ones(nx * ny, np.int32)
    params = sclbm.make_params(ncomp=2, tau=(0.9, 1.1), g_fluid=(1.2, 1.2), g_solid=(-0.2, 0.2),
                               rho_ref=(1.0, 1.0), force=(cases.force_vec(1e-5, "x") if porous else None, None))
    digests = []
    for v in (variant, 2):
        d = sclbm.Domain(nx, ny, mask, params, prec)
        d.set_kernel(v, 0)
        d.init_noise(0, 1.0, 0.02, 5)
        d.init_noise(1, 1.0, 0.02, 6)
        d.step(3)
        d.mass_momentum()  # finite, no bounded wait ran out
        digests.append([hashlib.sha256(d.download_f(k).tobytes()).hexdigest() for k in range(2)])
        del d
    assert digests[0] == digests[1], (prec_name, ny, porous)


# ------------------------------------------------------------------- monitors
def test_mass_momentum_monitor(sclbm):
    for prec in (sclbm.FP64, sclbm.FP32_SHIFTED, sclbm.FP16_SHIFTED):
        res = gpu_runner.run_domain(sclbm, RUNS["channel_80x32"], prec, rho_ref=(0.6, 1.4))
        d = res["_domain"]
        mm = d.mass_momentum()
        mask = np.asarray(gpu_runner._geometry(sclbm, RUNS["channel_80x32"])[1], bool)
        for k in range(2):
            f = d.download_f(k).reshape(9, -1)[:, mask]
            assert np.isclose(mm[3 * k], f.sum(), rtol=1e-12)
            assert np.isclose(mm[3 * k + 1], (cases.CX[:, None] * f).sum(), rtol=1e-9, atol=1e-9)
            assert np.isclose(mm[3 * k + 2], (cases.CY[:, None] * f).sum(), rtol=1e-9, atol=1e-9)
        assert mm[6] == 0


def test_mass_conserved_in_periodic_domain(sclbm):
    case = dict(RUNS["spinodal_48x40"], steps=0)
    # FP32: no systematic drift (the rest population closes each node's mass)
    for prec, tol in ((sclbm.FP64, 1e-13), (sclbm.FP32_SHIFTED, 1e-7)):
        d = gpu_runner.make_domain(sclbm, case, prec)
        m0 = d.mass_momentum()
        d.step(500)
        m1 = d.mass_momentum()
        for k in range(2):
            assert abs(m1[3 * k] - m0[3 * k]) <= tol * abs(m0[3 * k]), (prec, k)


def test_monitor_reports_non_finite(sclbm):
    case = dict(RUNS["spinodal_48x40"], steps=0)
    d = gpu_runner.make_domain(sclbm, case, sclbm.FP64)
    f = d.download_f(0)
    f[5] = np.nan
    d.upload_f(0, f)
    from sc_lbm_b200.capi import SclbmNonFinite
    with pytest.raises(SclbmNonFinite):
        d.mass_momentum()


# ---------------------------------------------------------------------- batch
def test_batch_matches_individual_domains(sclbm):
    names = ["porous_96x48", "spinodal_48x40", "channel_80x32", "laplace_64x64",
             "droplet_solid_flow", "absent_24x16"]
    for prec, graph, kernel in ((sclbm.FP64, True, 0), (sclbm.FP32_SHIFTED, True, 0),
                                (sclbm.FP32_SHIFTED, False, 3), (sclbm.FP64, False, 2),
                                (sclbm.FP16_SHIFTED, False, 0), (sclbm.FP32_SHIFTED, True, 5),
                                (sclbm.FP16_SHIFTED, False, 5), (sclbm.FP32_SHIFTED, True, 6),
                                (sclbm.FP16_SHIFTED, False, 6), (sclbm.FP32_SHIFTED, True, 8),
                                (sclbm.FP16_SHIFTED, True, 8), (sclbm.FP32_SHIFTED, True, 9),
                                (sclbm.FP16_SHIFTED, False, 9), (sclbm.FP32_SHIFTED, True, 10),
                                (sclbm.FP16_SHIFTED, False, 10), (sclbm.FP32_SHIFTED, True, 11),
                                (sclbm.FP16_SHIFTED, True, 11), (sclbm.FP64, True, 11),
                                (sclbm.FP32_SHIFTED, False, 11), (sclbm.FP32_SHIFTED, True, 12),
                                (sclbm.FP16_SHIFTED, True, 12), (sclbm.FP64, False, 12)):
        rr = (0.8, 1.2)
        solo = [gpu_runner.run_domain(sclbm, dict(RUNS[n], steps=45), prec, rho_ref=rr) for n in names]
        doms = [gpu_runner.make_domain(sclbm, RUNS[n], prec, rho_ref=rr) for n in names]
        b = sclbm.Batch(doms, tile_y=[3, 16, 8, 5, 12, 2])
        b.set_kernel(kernel)
        b.step(45, use_graph=graph)
        for s, d, n in zip(solo, doms, names):
            for k in range(2):
                assert d.download_f(k).tobytes() == s[f"c{k + 1}_f"].tobytes(), (prec, n, k)


@pytest.mark.parametrize("kernel", [0, 11, 12])
def test_batch_fp64_matches_reference(sclbm, kernel):
    names = ["porous_96x48", "spinodal_48x40", "laplace_64x64"]
    doms = [gpu_runner.make_domain(sclbm, RUNS[n], sclbm.FP64) for n in names]
    steps = {RUNS[n]["steps"] for n in names}
    doms_by = {}
    for n, d in zip(names, doms):
        doms_by.setdefault(RUNS[n]["steps"], []).append((n, d))
    for st, group in doms_by.items():
        b = sclbm.Batch([d for _, d in group])
        b.set_kernel(kernel)
        b.step(st, use_graph=True)
        for n, d in group:
            res = {"c1_f": d.download_f(0), "c2_f": d.download_f(1)}
            assert_golden(n, res, ["c1_f", "c2_f"])
            d.mass_momentum()  # raises if a bounded wait ran out
    assert steps


def test_batch_ring_needs_aligned_rows(sclbm):
    """The ring body copies rows that start on 16-byte boundaries: a batch
    holding a domain 130 wide refuses it in FP32 (130 is not a multiple of 4)
    and keeps its other bodies."""
    f = cases.noisy_f_equilibrium(3, 130, 6, 1.0, 0.02, 0.03)
    case = dict(nx=130, ny=6, geom=[], mode="two", fluid1=(1.0, 1.0, 0.0), fluid2=(1.0, 1.0, 0.0),
                init=("file", np.concatenate([f, f])), steps=3)
    d = gpu_runner.make_domain(sclbm, case, sclbm.FP32_SHIFTED)
    b = sclbm.Batch([d, gpu_runner.make_domain(sclbm, RUNS["spinodal_48x40"], sclbm.FP32_SHIFTED)])
    with pytest.raises(ValueError):
        b.set_kernel(11)
    b.set_kernel(2)
    b.step(3)


# ----------------------------------------------------------------- error paths
def test_reference_error_behaviour(sclbm):
    g = sclbm.Geometry(10, 8)
    a, b = sclbm.Fluid(g), sclbm.Fluid(g)
    lbm = sclbm.LBM(g)
    # compute_equilibrium_velocities before the solid force exists: out_of_range
    with pytest.raises(IndexError):
        lbm.compute_equilibrium_velocities(g, a, b)
    with pytest.raises(IndexError):
        lbm.add_volume_force(g, a, [0.0] * 8)
    g2 = sclbm.Geometry(11, 8)
    with pytest.raises(ValueError):
        lbm.stream(g2, sclbm.Fluid(g2))
    bad = g.get_geom()
    bad[3] = 2
    with pytest.raises(ValueError):
        sclbm.Domain(10, 8, bad, sclbm.make_params())
    with pytest.raises(ValueError):
        sclbm.Domain(10, 8, g.get_geom(), sclbm.make_params(tau=(0.0, 1.0)))
    with pytest.raises(IndexError):
        lbm.initialize_fluid_rectangle(g, a, b, 2.0, 2.0, 0.1, 0.1, 9.0, 6.0, 5.0, 3.0)
