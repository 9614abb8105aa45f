"""Full-size runs of the sc_lbm configurations on one B200 (physics and
throughput checks beyond the benchmark line).

    python -m sc_lbm_b200.validation [poiseuille laplace drainage ensemble spinodal contact]
                                     [--out results.json] [--quick]

Each run prints one JSON object; ``--out`` collects them.  The FP64 GPU form is
bit-exact with the reference (the parity tests prove it on the shared cases),
so at sizes the serial reference cannot reach it is the yardstick of the
shifted forms.  Inputs are seeded (sc_lbm_b200/workloads.py).

* poiseuille -- 200 x 50, FP64, 10,000 steps: velocity profile against the
  analytic parabola (laminar_flow_x_dir.cpp with the reference's post-processing
  formula, scripts/benchmark_utils.py:8-52).
* laplace    -- 256 x 256, radii 20..40 in one batch, FP64 and FP32-shifted,
  20,000 steps: pressure jump against 1/R (the Laplace law, surface tension as
  the slope; pressure p = (rho1+rho2)/3 + G rho1 rho2 / 3 as in
  compute_surface_tension.py:65) and the largest spurious velocity.
* drainage   -- 2048 x 1024 porous medium, FP64 / FP32 / FP16, 50,000 steps:
  density error against FP64 over time, saturation, mass drift, MLUPS.
* ensemble   -- 512 domains in one batch (tuned tiles, CUDA graph), FP32,
  10,000 steps: MLUPS against one large domain, mass drift per domain.
* spinodal   -- 16384 x 8192 periodic, FP64 / FP32 / FP16, 5,000 steps:
  MLUPS, fraction of the measured HBM bandwidth, density error and mass drift
  against FP64.
* contact    -- the reference's contact-angle benchmark: 400 x 306, a droplet
  on a solid shelf for eight solid interaction parameters in one batch, FP64
  and FP32-shifted, 30,000 steps: the angle measured on the device
  (compute_contact_angles.py's construction) against the parameter.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)

B_LU = {"fp64": 289, "fp64_1ulp_twin": 289, "fp32s": 145, "fp16s": 73}


def _env():
    import torch
    import sc_lbm_b200 as sc
    from sc_lbm_b200 import workloads as W
    stream = torch.cuda.Stream()
    sc.set_stream(stream.cuda_stream)
    return torch, sc, W, stream


def _timed(torch, stream, fn):
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def _peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            return float(json.load(fh)["hbm_gbs"])
    return 6650.0


def _errors(a, b, fluid=None):
    if fluid is not None:
        a, b = a[fluid], b[fluid]
    d = a - b
    return {"max_over_mean": float(np.max(np.abs(d)) / np.mean(np.abs(b))),
            "rms_over_mean": float(np.sqrt(np.mean(d * d)) / np.mean(np.abs(b)))}


# --------------------------------------------------------------- error reports
# Every shifted-form result states, per component, its density and velocity
# error against the FP64 form (bit-exact with the reference) and its mass
# drift.  The FP64 1-ulp twin starts with component 1's density one ulp
# higher at every fluid node and is compared the same way: its error is what
# the dynamics make of a rounding-sized difference, so a shifted form whose
# error stays far above the twin's owes it to its storage, and one whose error
# tracks the twin's amplification owes it to the physics.
def twin_populations(f, mask=None):
    """Populations whose node density is one ulp higher at fluid nodes: one
    ulp of the density is added to the rest population (perturbing every f_i
    by one ulp instead is lost in the density sum at tau = 1, where the
    collision keeps nothing of f but its moments)."""
    f = np.asarray(f, dtype=np.float64)
    N = f.size // 9
    g = f.copy()
    rho = f.reshape(9, N).sum(axis=0)
    bump = np.spacing(np.abs(rho))
    if mask is not None:
        bump = np.where(np.asarray(mask).ravel() != 0, bump, 0.0)
    g[:N] += bump
    return g


def component_fields(d, c):
    """Density and velocity of component c (u = sum_i f_i c_i / rho on fluid
    nodes, Fluid::compute_velocities, src/fluid.cpp:186-200)."""
    ux, uy = d.download_velocity(c)
    return d.download_rho(c), ux, uy


def field_errors(got, ref, fluid=None):
    """Per component: max and RMS |drho| over the mean density, max |du| over
    max |u_ref| and RMS |du| over RMS |u_ref| (|du| the vector difference)."""
    r, ux, uy = got
    r0, ux0, uy0 = ref
    if fluid is not None:
        r, ux, uy, r0, ux0, uy0 = (a[fluid] for a in (r, ux, uy, r0, ux0, uy0))
    e = _errors(r, r0)
    du = np.hypot(ux - ux0, uy - uy0)
    u0 = np.hypot(ux0, uy0)
    umax, urms = float(np.max(u0)), float(np.sqrt(np.mean(u0 * u0)))
    return {"rho_max": e["max_over_mean"], "rho_rms": e["rms_over_mean"],
            "u_max": float(np.max(du)) / umax if umax > 0 else float(np.max(du)),
            "u_rms": float(np.sqrt(np.mean(du * du))) / urms if urms > 0 else
            float(np.sqrt(np.mean(du * du))), "u_ref_max": umax}


def compare_domains(doms, ref="fp64", fluid=None, ncomp=2):
    """field_errors of every domain but the reference, component by component
    (one component's fields on the host at a time)."""
    out = {k: [] for k in doms if k != ref}
    for c in range(ncomp):
        base = component_fields(doms[ref], c)
        for k, d in doms.items():
            if k != ref:
                out[k].append(field_errors(component_fields(d, c), base, fluid))
    return out


def mass_drift(d, m0, ncomp=2):
    m1 = d.mass_momentum()
    return [float((m1[3 * c] - m0[3 * c]) / m0[3 * c]) for c in range(ncomp)]


# ----------------------------------------------------------------------------- configs
PRECS = (("fp64", "FP64"), ("fp64_1ulp_twin", "FP64"), ("fp32s", "FP32_SHIFTED"),
         ("fp16s", "FP16_SHIFTED"))


def poiseuille(args):
    torch, sc, W, stream = _env()
    w = W.poiseuille()
    nx, ny = w["nx"], w["ny"]
    steps = 2000 if args.quick else 10000
    p = sc.make_params(ncomp=1, tau=(w["tau"], 1.0), rho_ref=(w["rho0"], 0.0),
                       force=(w["force"], None))
    doms, ms = {}, {}
    for name, prec in PRECS:
        d = sc.Domain(nx, ny, w["mask"], p, getattr(sc, prec))
        d.upload_f(0, twin_populations(w["f"], w["mask"]) if "twin" in name else w["f"])
        doms[name] = d
    m0 = {k: d.mass_momentum() for k, d in doms.items()}
    for k, d in doms.items():
        ms[k] = _timed(torch, stream, lambda: d.step(steps))
    ux, _ = doms["fp64"].download_velocity(0)
    rho = doms["fp64"].download_rho(0)
    u = (ux.reshape(ny, nx))[:, nx // 2]
    # half-way bounce-back: walls midway between rows 0|1 and ny-2|ny-1
    nu = (w["tau"] - 0.5) / 3.0
    h = (ny - 2) / 2.0
    yc = (ny - 1) / 2.0
    y = np.arange(ny)
    ua = w["g"] / (2 * nu * w["rho0"]) * (h * h - (y - yc) ** 2)
    fl = slice(1, ny - 1)
    err = float(np.linalg.norm(u[fl] - ua[fl]) / np.linalg.norm(ua[fl]))
    fluid = np.asarray(w["mask"]).ravel() != 0
    return {"config": "poiseuille 200x50 FP64 (shifted forms and twin alongside)", "steps": steps,
            "ms": {k: round(v, 2) for k, v in ms.items()},
            "u_max": float(u.max()), "u_max_analytic": float(ua.max()),
            "l2_rel_error_vs_analytic": err, "mean_rho": float(rho.reshape(ny, nx)[fl].mean()),
            "errors_vs_fp64": compare_domains(doms, fluid=fluid, ncomp=1),
            "mass_drift": {k: mass_drift(d, m0[k], 1) for k, d in doms.items()}}


def _laplace_stats(rho1, rho2, nx, ny, G):
    r1, r2 = rho1.reshape(ny, nx), rho2.reshape(ny, nx)
    p = (r1 + r2) / 3.0 + G * r1 * r2 / 3.0
    thr = 0.5 * (r1.max() + r1.min())
    area = float((r1 > thr).sum())
    R = np.sqrt(area / np.pi)
    yy, xx = np.mgrid[0:ny, 0:nx]
    dist = np.hypot(xx - nx / 2, yy - ny / 2)
    p_in = float(p[dist < 0.5 * R].mean())
    p_out = float(p[dist > R + 0.3 * (min(nx, ny) / 2 - R)].mean())
    return R, p_in - p_out


def laplace(args):
    torch, sc, W, stream = _env()
    radii = [20, 25, 30, 35, 40]
    steps = 4000 if args.quick else 20000
    out = {"config": "laplace 256x256, G=0.9, radii 20-40, one batch per precision",
           "steps": steps}
    ws = [W.laplace(r) for r in radii]
    sets = {}
    for name, prec in PRECS:
        doms = []
        for w in ws:
            rr = tuple(float(w[k].reshape(9, -1).sum(0).mean()) for k in ("f1", "f2"))
            d = sc.Domain(w["nx"], w["ny"], w["mask"], W.params_of(w, sc, rho_ref=rr),
                          getattr(sc, prec))
            d.upload_f(0, twin_populations(w["f1"]) if "twin" in name else w["f1"])
            d.upload_f(1, w["f2"])
            doms.append(d)
        m0 = [d.mass_momentum() for d in doms]
        b = sc.Batch(doms)
        ms = _timed(torch, stream, lambda: b.step(steps))
        del b
        sets[name] = doms
        rows = []
        for w, d, a in zip(ws, doms, m0):
            r1, r2 = d.download_rho(0), d.download_rho(1)
            (u1x, u1y), (u2x, u2y) = d.download_velocity(0), d.download_velocity(1)
            jx, jy = r1 * u1x + r2 * u2x, r1 * u1y + r2 * u2y
            umax = float(np.max(np.hypot(jx, jy) / (r1 + r2)))
            R, dp = _laplace_stats(r1, r2, w["nx"], w["ny"], w["G"])
            rows.append({"R0": w["radius"], "R": R, "dp": dp, "max_spurious_u": umax,
                         "mass_drift": mass_drift(d, a)})
        inv = np.array([1.0 / r["R"] for r in rows])
        dps = np.array([r["dp"] for r in rows])
        A = np.vstack([inv, np.ones_like(inv)]).T
        (sigma, c0), *_ = np.linalg.lstsq(A, dps, rcond=None)
        pred = A @ np.array([sigma, c0])
        r2 = 1.0 - float(np.sum((dps - pred) ** 2) / np.sum((dps - dps.mean()) ** 2))
        out[name] = {"droplets": rows, "surface_tension": float(sigma), "intercept": float(c0),
                     "fit_r2": r2, "ms": round(ms, 2),
                     "mlups": round(sum(d.N for d in doms) * steps / (ms * 1e-3) / 1e6, 1)}
    # field errors of every droplet against its FP64 run
    for name in ("fp64_1ulp_twin", "fp32s", "fp16s"):
        per = [compare_domains({"fp64": sets["fp64"][i], name: sets[name][i]})[name]
               for i in range(len(ws))]
        out[name]["errors_vs_fp64"] = per
        out[name]["worst_vs_fp64"] = {q: max(c[q] for p_ in per for c in p_)
                                      for q in ("rho_max", "rho_rms", "u_max", "u_rms")}
        out[name]["surface_tension_rel_diff"] = abs(out[name]["surface_tension"] /
                                                    out["fp64"]["surface_tension"] - 1)
    return out


def drainage(args):
    torch, sc, W, stream = _env()
    w = W.drainage()
    nx, ny, N = w["nx"], w["ny"], w["nx"] * w["ny"]
    fluid = w["mask"] != 0
    total = 10000 if args.quick else 50000
    checkpoints = [c for c in (100, 1000, 10000, 50000) if c <= total]
    doms = {}
    for name, prec in PRECS:
        rr = (float(w["f1"].reshape(9, -1).sum(0)[fluid].mean()),
              float(w["f2"].reshape(9, -1).sum(0)[fluid].mean()))
        d = sc.Domain(nx, ny, w["mask"], W.params_of(w, sc, rho_ref=rr), getattr(sc, prec))
        d.upload_f(0, twin_populations(w["f1"], w["mask"]) if "twin" in name else w["f1"])
        d.upload_f(1, w["f2"])
        doms[name] = d
    m0 = {k: d.mass_momentum() for k, d in doms.items()}
    out = {"config": f"drainage {nx}x{ny}, porosity {w['porosity']:.3f}, {w['disks']} disks",
           "steps": total, "checkpoints": {}}
    ms_tot = {k: 0.0 for k in doms}
    done = 0
    for cp in checkpoints:
        for k, d in doms.items():
            ms_tot[k] += _timed(torch, stream, lambda: d.step(cp - done))
        done = cp
        row = {"errors_vs_fp64": compare_domains(doms, fluid=fluid),
               "mass_drift": {k: mass_drift(d, m0[k]) for k, d in doms.items()}}
        for k, d in doms.items():
            r0, r1 = d.download_rho(0), d.download_rho(1)
            row[k + "_saturation1"] = float(np.mean(r0[fluid] > r1[fluid]))
        out["checkpoints"][str(cp)] = row
    out["mass_drift"] = {k: mass_drift(d, m0[k]) for k, d in doms.items()}
    out["mlups"] = {k: round(N * total / (ms * 1e-3) / 1e6, 1) for k, ms in ms_tot.items()}
    return out


def _porous_single(sc, W, nx, ny, porosity, prec):
    """One large seeded porous domain shaped like the ensemble members (disks
    of radius 2-8, per-node noise), for the batch-efficiency comparison."""
    m, _, phi = W.disk_mask(nx, ny, porosity, 2, 8, 31337, max_tries=400000, max_misses=2000)
    d = sc.Domain(nx, ny, m, sc.make_params(ncomp=2, tau=(1.0, 1.0), g_fluid=(1.0, 1.0),
                                            g_solid=(0.1, -0.1), rho_ref=(1.0, 1.0)), prec)
    d.init_noise(0, 1.0, 0.01, 101)
    d.init_noise(1, 1.0, 0.01, 102)
    return d, phi


def ensemble(args):
    torch, sc, W, stream = _env()
    n = 128 if args.quick else 512
    steps = 1000 if args.quick else 10000
    t0 = time.time()
    members = W.ensemble(n)
    gen_s = time.time() - t0
    out = {"config": f"ensemble of {n} seeded porous domains, one batch per precision",
           "steps": steps, "porosity_mean": float(np.mean([m["porosity"] for m in members])),
           "generation_s": round(gen_s, 1)}
    finite, sets = {}, {}
    for name, prec in (("fp32s", "FP32_SHIFTED"), ("fp64", "FP64"), ("fp64_1ulp_twin", "FP64"),
                       ("fp16s", "FP16_SHIFTED")):
        doms = []
        for m in members:
            d = sc.Domain(m["nx"], m["ny"], m["mask"], W.params_of(m, sc), getattr(sc, prec))
            d.upload_f(0, twin_populations(m["f1"], m["mask"]) if "twin" in name else m["f1"])
            d.upload_f(1, m["f2"])
            doms.append(d)
        nodes = sum(d.N for d in doms)
        m0 = [d.mass_momentum() for d in doms]
        b = sc.Batch(doms)  # tuned tile shapes per size class
        ntiles, grid = b.info()
        b.step(20)
        ms = _timed(torch, stream, lambda: b.step(steps))
        drift, ok = [], []
        for d, a in zip(doms, m0):
            try:
                m1 = d.mass_momentum()
                drift.append(max(abs((m1[3 * c] - a[3 * c]) / a[3 * c]) for c in range(2)))
                ok.append(True)
            except sc.capi.SclbmNonFinite:
                ok.append(False)
        finite[name] = ok
        sets[name] = doms
        out[name] = {"mlups": round(nodes * steps / (ms * 1e-3) / 1e6, 1), "tiles": ntiles,
                     "ctas": grid, "nodes": nodes, "non_finite_domains": int(len(ok) - sum(ok)),
                     "max_mass_drift_finite": float(max(drift)) if drift else None}
        del b
    bad = [k for k in range(n) if not finite["fp32s"][k] or not finite["fp64"][k]]
    out["non_finite_params"] = [
        {"k": k, "nx": members[k]["nx"], "ny": members[k]["ny"], "tau": members[k]["tau"][0],
         "G": members[k]["G"], "Gs": members[k]["Gs"][0], "porosity": members[k]["porosity"],
         "fp32s_finite": finite["fp32s"][k], "fp64_finite": finite["fp64"][k]} for k in bad[:20]]
    # field errors over the members that stay finite in every form (the
    # others go non-finite in FP64 too, at the reference's own step)
    stable = [k for k in range(n) if all(finite[x][k] for x in finite)]
    out["stable_members"] = len(stable)
    for name in ("fp64_1ulp_twin", "fp32s", "fp16s"):
        per = []
        for k in stable:
            fl = np.asarray(members[k]["mask"]).ravel() != 0
            e = compare_domains({"fp64": sets["fp64"][k], name: sets[name][k]}, fluid=fl)[name]
            per.append({q: max(c[q] for c in e) for q in ("rho_max", "rho_rms", "u_max", "u_rms")})
        out[name]["errors_vs_fp64_stable_members"] = {
            q: {"median": float(np.median([p_[q] for p_ in per])),
                "p90": float(np.percentile([p_[q] for p_ in per], 90)),
                "max": float(np.max([p_[q] for p_ in per]))}
            for q in ("rho_max", "rho_rms", "u_max", "u_rms")} if per else None
    del sets
    # single large domains of the same storage for the efficiency ratio
    D = sc.Domain(4096, 4096, np.ones(4096 * 4096, np.int32),
                  sc.make_params(ncomp=2, g_fluid=(1.2, 1.2), rho_ref=(1.0, 1.0)), sc.FP32_SHIFTED)
    D.init_noise(0, 1.0, 0.01, 101)
    D.init_noise(1, 1.0, 0.01, 102)
    D.step(20)
    ms_big = _timed(torch, stream, lambda: D.step(200)) / 200
    del D
    P, phi = _porous_single(sc, W, 4096, 4096, out["porosity_mean"], sc.FP32_SHIFTED)
    P.step(20)
    ms_por = _timed(torch, stream, lambda: P.step(200)) / 200
    del P
    out["single_4096_all_fluid_mlups"] = round(4096 * 4096 / (ms_big * 1e-3) / 1e6, 1)
    out["single_4096_porous_mlups"] = round(4096 * 4096 / (ms_por * 1e-3) / 1e6, 1)
    out["single_4096_porosity"] = phi
    out["efficiency_vs_single_all_fluid"] = round(out["fp32s"]["mlups"] /
                                                  out["single_4096_all_fluid_mlups"], 4)
    out["efficiency_vs_single_porous"] = round(out["fp32s"]["mlups"] /
                                               out["single_4096_porous_mlups"], 4)
    return out


def spinodal(args):
    torch, sc, W, stream = _env()
    nx, ny = (8192, 4096) if args.quick else (16384, 8192)
    N = nx * ny
    steps = 1000 if args.quick else 5000
    peak = _peak()
    doms = {}
    for name, prec in PRECS:
        d = sc.Domain(nx, ny, np.ones(N, np.int32),
                      sc.make_params(ncomp=2, g_fluid=(1.2, 1.2), rho_ref=(1.0, 1.0)),
                      getattr(sc, prec))
        d.init_noise(0, 1.0, 0.01, 101)
        d.init_noise(1, 1.0, 0.01, 102)
        if "twin" in name:
            d.upload_f(0, twin_populations(d.download_f(0)))
        doms[name] = d
    m0 = {k: d.mass_momentum() for k, d in doms.items()}
    out = {"config": f"spinodal {nx}x{ny} periodic, G=1.2, rho=1+-1%", "steps": steps,
           "device_gb": {k: round(d.device_bytes() / 1e9, 2) for k, d in doms.items()}}
    ms, done, acc = {k: 0.0 for k in doms}, 0, {}
    for cp in (20, steps):
        for k, d in doms.items():
            ms[k] += _timed(torch, stream, lambda: d.step(cp - done))
        done = cp
        acc[str(cp)] = compare_domains(doms)
    out["errors_vs_fp64"] = acc
    out["mass_drift"] = {k: mass_drift(d, m0[k]) for k, d in doms.items()}
    out["mlups"] = {k: round(N * steps / (t * 1e-3) / 1e6, 1) for k, t in ms.items()}
    out["hbm_frac"] = {k: round(B_LU[k] * N * steps / (t * 1e-3) / 1e9 / peak, 4)
                       for k, t in ms.items()}
    return out


def contact(args):
    """The reference's contact-angle benchmark (contact_angles.cpp): one
    400 x 306 domain per solid interaction parameter, all in one batch, and
    the angle measured on the device as compute_contact_angles.py measures it
    from the density files."""
    torch, sc, W, stream = _env()
    gs_values = [-0.4, -0.3, -0.2, -0.1, 0.1, 0.2, 0.3, 0.4]
    steps = 5000 if args.quick else 30000
    out = {"config": "contact angles 400x306, droplet on a 341x20 shelf, G=0.9, "
                     "Gs_droplet -0.4..0.4, one batch per precision", "steps": steps}
    ws = [W.contact_angle(g) for g in gs_values]
    sets = {}
    for name, prec in PRECS:
        doms = []
        for w in ws:
            fl = np.asarray(w["mask"]).ravel() != 0
            rr = tuple(float(w[k].reshape(9, -1).sum(0)[fl].mean()) for k in ("f1", "f2"))
            d = sc.Domain(w["nx"], w["ny"], w["mask"], W.params_of(w, sc, rho_ref=rr),
                          getattr(sc, prec))
            d.upload_f(0, twin_populations(w["f1"], w["mask"]) if "twin" in name else w["f1"])
            d.upload_f(1, w["f2"])
            doms.append(d)
        m0 = [d.mass_momentum() for d in doms]
        b = sc.Batch(doms)
        ms = _timed(torch, stream, lambda: b.step(steps))
        rows = []
        for g, d, a in zip(gs_values, doms, m0):
            row = {"gs_droplet": g}
            try:
                row.update(d.contact_angle(0, rho_bulk=2.0, rho_disp=0.06))
            except IndexError as e:
                row["error"] = str(e)
            m1 = d.mass_momentum()
            row["mass_drift"] = [float((m1[3 * c] - a[3 * c]) / a[3 * c]) for c in range(2)]
            rows.append(row)
        th = [r.get("theta") for r in rows]
        out[name] = {"angles": rows, "theta_deg": th,
                     "monotonic_in_gs": all(x is not None for x in th) and
                     all(th[i] < th[i + 1] for i in range(len(th) - 1)),
                     "ms": round(ms, 2),
                     "mlups": round(sum(d.N for d in doms) * steps / (ms * 1e-3) / 1e6, 1)}
        del b
        sets[name] = doms
    for name in ("fp64_1ulp_twin", "fp32s", "fp16s"):
        a, b_ = out["fp64"]["theta_deg"], out[name]["theta_deg"]
        out[name]["max_abs_theta_diff_deg"] = max(
            (abs(x - y) for x, y in zip(a, b_) if x is not None and y is not None), default=None)
        per = [compare_domains({"fp64": sets["fp64"][i], name: sets[name][i]},
                               fluid=np.asarray(ws[i]["mask"]).ravel() != 0)[name]
               for i in range(len(ws))]
        out[name]["errors_vs_fp64"] = per
        out[name]["worst_vs_fp64"] = {q: max(c[q] for p_ in per for c in p_)
                                      for q in ("rho_max", "rho_rms", "u_max", "u_rms")}
    return out


RUNS = {"poiseuille": poiseuille, "laplace": laplace, "drainage": drainage,
        "ensemble": ensemble, "spinodal": spinodal, "contact": contact}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("runs", nargs="*", default=list(RUNS))
    ap.add_argument("--out", default=None)
    ap.add_argument("--quick", action="store_true", help="shorter runs (smoke)")
    args = ap.parse_args()
    results = {}
    for name in args.runs:
        t0 = time.time()
        r = RUNS[name](args)
        r["wall_s"] = round(time.time() - t0, 1)
        results[name] = r
        print(json.dumps({name: r}), flush=True)
        import gc
        gc.collect()
    if args.out:
        with open(args.out, "w") as fh:
            json.dump(results, fh, indent=1)


if __name__ == "__main__":
    main()
