"""GPU checks of the on-device measurements against the reference's
post-processing done in numpy on the downloaded fields.

* Laplace law (compute_surface_tension.py:55-73): pressure jump between two
  nodes and the radius from the interface band's extent -- identical in FP64;
* spurious currents (vel_mag / ave of scripts/benchmark_utils.py): the
  largest |u| identical, the mean of the nonzero |u| to summation order;
* the channel profile (row means of u_x) against numpy and, after 10,000
  steps of the 200 x 50 Poiseuille channel, against the analytic parabola of
  scripts/benchmark_utils.py:8-52;
* the contact angle (compute_contact_angles.py:45-106) against the numpy
  restatement in oracle/post.py and the angles the reference's script printed
  on the same fields.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _laplace_domain(sclbm, prec, steps):
    from sc_lbm_b200 import workloads as W
    w = W.laplace(12.0, nx=64, ny=64)
    rr = tuple(float(w[k].reshape(9, -1).sum(0).mean()) for k in ("f1", "f2"))
    d = sclbm.Domain(64, 64, w["mask"], W.params_of(w, sclbm, rho_ref=rr), prec)
    d.upload_f(0, w["f1"])   # component 0: the droplet (rho 2.0 inside)
    d.upload_f(1, w["f2"])   # component 1: the bulk
    d.step(steps)
    return d, w


def _numpy_laplace(rb, rd, G, rho_bulk, rho_disp, p_in, p_out, nx, ny):
    rb, rd = rb.reshape(ny, nx), rd.reshape(ny, nx)
    p = 1.0 / 3.0 * (rb + rd) + G / 3.0 * rb * rd
    dp = p[p_in[1], p_in[0]] - p[p_out[1], p_out[0]]
    sel = np.where((rd - rb < 0) & (rb <= rho_bulk) & (rb > rho_disp))
    Rr = (np.amax(sel[0]) - np.amin(sel[0])) / 2.0
    Rc = (np.amax(sel[1]) - np.amin(sel[1])) / 2.0
    return dp, 0.5 * (Rr + Rc), len(sel[0])


@pytest.mark.parametrize("prec_name", ["FP64", "FP32_SHIFTED"])
def test_laplace_measure(sclbm, prec_name):
    d, w = _laplace_domain(sclbm, getattr(sclbm, prec_name), 400)
    got = d.laplace_measure(bulk=1, G=0.9, rho_bulk=1.9, rho_disp=0.06, p_in=(32, 32), p_out=(2, 2))
    dp, R, band = _numpy_laplace(d.download_rho(1), d.download_rho(0), 0.9, 1.9, 0.06,
                                 (32, 32), (2, 2), 64, 64)
    if prec_name == "FP64":
        assert got["dp"] == dp and got["R"] == R and got["band_nodes"] == band
    else:
        assert got["dp"] == pytest.approx(dp, rel=1e-9, abs=1e-15)
        assert abs(got["R"] - R) <= 0.5
    assert 8.0 < got["R"] < 16.0 and got["dp"] > 0


@pytest.mark.parametrize("prec_name", ["FP64", "FP32_SHIFTED", "FP16_SHIFTED"])
def test_velocity_stats_and_profile(sclbm, prec_name):
    import cases
    import gpu_runner
    case = cases.all_cases()["porous_96x48"]
    d = gpu_runner.make_domain(sclbm, case, getattr(sclbm, prec_name), rho_ref=(0.5, 1.5))
    d.step(30)
    fluid = (gpu_runner._geometry(sclbm, case)[1].ravel() != 0)
    for comp in (0, 1):
        ux, uy = d.download_velocity(comp)
        m = np.sqrt(ux * ux + uy * uy)[fluid]
        st = d.velocity_stats(comp)
        if prec_name == "FP64":
            assert st["max_u"] == m.max()
        else:
            assert st["max_u"] == pytest.approx(m.max(), rel=1e-12)
        nz = m[m != 0]
        assert st["nonzero"] == nz.size
        assert st["mean_nonzero_u"] == pytest.approx(nz.mean(), rel=1e-12)
        prof = d.profile(comp, 0)
        u2 = ux.reshape(d.ny, d.nx)
        f2 = fluid.reshape(d.ny, d.nx)
        want = np.array([u2[y][f2[y]].mean() if f2[y].any() else 0.0 for y in range(d.ny)])
        np.testing.assert_allclose(prof, want, rtol=1e-12, atol=1e-300)


def test_poiseuille_profile_against_analytic(sclbm):
    from sc_lbm_b200 import workloads as W
    w = W.poiseuille()
    p = sclbm.make_params(ncomp=1, tau=(1.0, 1.0), force=(w["force"], None))
    d = sclbm.Domain(w["nx"], w["ny"], w["mask"], p, sclbm.FP64)
    d.upload_f(0, w["f"])
    d.step(10000)
    prof = d.profile(0, 0)
    # benchmark_utils.channel_flow_analytical: wall thickness 1, half width
    # (ny - 2)/2, u = u_max (1 - (y/h)^2) at the fluid rows' centres
    h = (w["ny"] - 2) / 2.0
    lat = np.arange(-h, h) + 0.5
    mu = (1.0 - 0.5) / 3.0
    ua = w["g"] * h * h / (2 * mu) * (1 - (lat / h) ** 2)
    assert np.linalg.norm(prof[1:-1] - ua) / np.linalg.norm(ua) < 5e-3
    assert prof[0] == 0.0 and prof[-1] == 0.0


def _contact_golden():
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "contact_angle_golden.json")) as fh:
        return json.load(fh)["theta_deg"]


@pytest.mark.parametrize("prec_name", ["FP64", "FP32_SHIFTED", "FP16_SHIFTED"])
def test_contact_angle_against_reference_script(sclbm, prec_name):
    """The device measurement on the synthetic fields the reference's own
    script was run on (contact_angle_golden.json): every quantity equal to
    the numpy restatement on the downloaded densities, and the angle equal to
    the one the script printed."""
    import contact_fields
    from oracle import post
    from sc_lbm_b200 import workloads as W
    golden = _contact_golden()
    for key in contact_fields.CASES:
        rb, rd = contact_fields.fields(key)
        ny, nx = rb.shape
        mask = ((rb != 0) | (rd != 0)).astype(np.int32).ravel()
        rr = (float(rb[rb > 0].mean()), float(rd[rd > 0].mean()))
        d = sclbm.Domain(nx, ny, mask, sclbm.make_params(ncomp=2, rho_ref=rr),
                         getattr(sclbm, prec_name))
        d.upload_f(0, W.populations(rb.ravel(), mask))
        d.upload_f(1, W.populations(rd.ravel(), mask))
        got = d.contact_angle(0, rho_bulk=2.0, rho_disp=0.06)
        want = post.contact_angle(d.download_rho(0), d.download_rho(1), nx, ny, 2.0, 0.06)
        # the shifted forms' densities carry their storage rounding (core nodes
        # at rho_b = 0.06 may join the band); the band's ends and rows do not move
        keys = ("L", "H", "R", "xL", "xR", "y_min", "y_max")
        for k in keys + (("band_nodes",) if prec_name == "FP64" else ()):
            assert got[k] == want[k], (key, k)
        assert got["theta"] == pytest.approx(want["theta"], rel=1e-14, abs=1e-12)
        assert got["theta"] == pytest.approx(golden[key], rel=1e-14, abs=1e-12), key


def test_contact_angle_reduced_benchmark(sclbm):
    """A droplet on a shelf after 2,000 FP64 steps (the reduced contact-angle
    case, bit-identical to the compiled reference): the device measurement
    equals the restatement on the reference's own final densities."""
    import cases
    import gpu_runner
    from oracle import post
    case = cases.all_cases()["contact_120x90"]
    d = gpu_runner.make_domain(sclbm, case, sclbm.FP64)
    d.step(case["steps"])
    got = d.contact_angle(0, rho_bulk=2.0, rho_disp=0.06)
    want = post.contact_angle(d.download_rho(0), d.download_rho(1), 120, 90, 2.0, 0.06)
    for k in ("L", "H", "R", "xL", "xR", "y_min", "y_max", "band_nodes"):
        assert got[k] == want[k], k
    assert got["theta"] == pytest.approx(want["theta"], rel=1e-14)
    assert 30.0 < got["theta"] < 90.0   # the droplet's solid parameter -0.2 wets the shelf


def test_contact_angle_errors(sclbm):
    nx, ny = 32, 24
    d = sclbm.Domain(nx, ny, np.ones(nx * ny, np.int32),
                     sclbm.make_params(ncomp=2, rho_ref=(1.0, 1.0)), sclbm.FP64)
    from sc_lbm_b200 import workloads as W
    d.upload_f(0, W.populations(np.full(nx * ny, 2.0)))
    d.upload_f(1, W.populations(np.full(nx * ny, 0.06)))
    with pytest.raises(IndexError):
        d.contact_angle(0)          # no droplet: empty band
    rb = np.full((ny, nx), 2.0)
    rd = np.full((ny, nx), 0.06)
    rb[12, 5:20], rd[12, 5:20] = 0.7, 1.3   # a band of one row
    d.upload_f(0, W.populations(rb.ravel()))
    d.upload_f(1, W.populations(rd.ravel()))
    with pytest.raises(IndexError):
        d.contact_angle(0)
    with pytest.raises(ValueError):
        d.contact_angle(2)
