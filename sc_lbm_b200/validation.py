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

B_LU = {"fp64": 289, "fp32s": 145, "fp16s": 73}


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


# ----------------------------------------------------------------------------- configs
def poiseuille(args):
    torch, sc, W, stream = _env()
    w = W.poiseuille()
    nx, ny = w["nx"], w["ny"]
    steps = 2000 if args.quick else 10000
    p = sc.make_params(ncomp=1, tau=(w["tau"], 1.0), force=(w["force"], None))
    d = sc.Domain(nx, ny, w["mask"], p, sc.FP64)
    d.upload_f(0, w["f"])
    ms = _timed(torch, stream, lambda: d.step(steps))
    ux, _ = d.download_velocity(0)
    rho = d.download_rho(0)
    u = (ux.reshape(ny, nx))[:, nx // 2]
    # half-way bounce-back: walls midway between rows 0|1 and ny-2|ny-1
    nu = (w["tau"] - 0.5) / 3.0
    h = (ny - 2) / 2.0
    yc = (ny - 1) / 2.0
    y = np.arange(ny)
    ua = w["g"] / (2 * nu * w["rho0"]) * (h * h - (y - yc) ** 2)
    fl = slice(1, ny - 1)
    err = float(np.linalg.norm(u[fl] - ua[fl]) / np.linalg.norm(ua[fl]))
    return {"config": "poiseuille 200x50 FP64", "steps": steps, "ms": round(ms, 2),
            "u_max": float(u.max()), "u_max_analytic": float(ua.max()),
            "l2_rel_error_vs_analytic": err, "mean_rho": float(rho.reshape(ny, nx)[fl].mean())}


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
    for prec, name in ((sc.FP64, "fp64"), (sc.FP32_SHIFTED, "fp32s")):
        ws = [W.laplace(r) for r in radii]
        doms = []
        for w in ws:
            rr = tuple(float(w[k].reshape(9, -1).sum(0).mean()) for k in ("f1", "f2"))
            d = sc.Domain(w["nx"], w["ny"], w["mask"], W.params_of(w, sc, rho_ref=rr), prec)
            d.upload_f(0, w["f1"])
            d.upload_f(1, w["f2"])
            doms.append(d)
        b = sc.Batch(doms)
        ms = _timed(torch, stream, lambda: b.step(steps))
        rows = []
        for w, d in zip(ws, doms):
            r1, r2 = d.download_rho(0), d.download_rho(1)
            (u1x, u1y), (u2x, u2y) = d.download_velocity(0), d.download_velocity(1)
            jx, jy = r1 * u1x + r2 * u2x, r1 * u1y + r2 * u2y
            umax = float(np.max(np.hypot(jx, jy) / (r1 + r2)))
            R, dp = _laplace_stats(r1, r2, w["nx"], w["ny"], w["G"])
            rows.append({"R0": w["radius"], "R": R, "dp": dp, "max_spurious_u": umax})
        inv = np.array([1.0 / r["R"] for r in rows])
        dps = np.array([r["dp"] for r in rows])
        A = np.vstack([inv, np.ones_like(inv)]).T
        (sigma, c0), *_ = np.linalg.lstsq(A, dps, rcond=None)
        pred = A @ np.array([sigma, c0])
        r2 = 1.0 - float(np.sum((dps - pred) ** 2) / np.sum((dps - dps.mean()) ** 2))
        out[name] = {"droplets": rows, "surface_tension": float(sigma), "intercept": float(c0),
                     "fit_r2": r2, "ms": round(ms, 2),
                     "mlups": round(sum(d.N for d in doms) * steps / (ms * 1e-3) / 1e6, 1)}
        del b, doms
    out["surface_tension_rel_diff_fp32s"] = abs(out["fp32s"]["surface_tension"] /
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
    for prec, name in ((sc.FP64, "fp64"), (sc.FP32_SHIFTED, "fp32s"), (sc.FP16_SHIFTED, "fp16s")):
        rr = (float(w["f1"].reshape(9, -1).sum(0)[fluid].mean()),
              float(w["f2"].reshape(9, -1).sum(0)[fluid].mean()))
        d = sc.Domain(nx, ny, w["mask"], W.params_of(w, sc, rho_ref=rr), prec)
        d.upload_f(0, w["f1"])
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
        ref = [doms["fp64"].download_rho(c) for c in range(2)]
        row = {}
        for k in ("fp32s", "fp16s"):
            rho = [doms[k].download_rho(c) for c in range(2)]
            row[k] = [_errors(rho[c], ref[c], fluid) for c in range(2)]
            row[k + "_saturation1"] = float(np.mean(rho[0][fluid] > rho[1][fluid]))
        row["fp64_saturation1"] = float(np.mean(ref[0][fluid] > ref[1][fluid]))
        out["checkpoints"][str(cp)] = row
    out["mass_drift"] = {k: [float((d.mass_momentum()[3 * c] - m0[k][3 * c]) / m0[k][3 * c])
                             for c in range(2)] for k, d in doms.items()}
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
    rho, finite = {}, {}
    for prec, name in ((sc.FP32_SHIFTED, "fp32s"), (sc.FP64, "fp64")):
        doms = []
        for m in members:
            d = sc.Domain(m["nx"], m["ny"], m["mask"], W.params_of(m, sc), prec)
            d.upload_f(0, m["f1"])
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
        rho[name] = [d.download_rho(0) if good else None for d, good in zip(doms, ok)]
        out[name] = {"mlups": round(nodes * steps / (ms * 1e-3) / 1e6, 1), "tiles": ntiles,
                     "ctas": grid, "nodes": nodes, "non_finite_domains": int(len(ok) - sum(ok)),
                     "max_mass_drift_finite": float(max(drift)) if drift else None}
        del b, doms
    bad = [k for k in range(n) if not finite["fp32s"][k] or not finite["fp64"][k]]
    out["non_finite_params"] = [
        {"k": k, "nx": members[k]["nx"], "ny": members[k]["ny"], "tau": members[k]["tau"][0],
         "G": members[k]["G"], "Gs": members[k]["Gs"][0], "porosity": members[k]["porosity"],
         "fp32s_finite": finite["fp32s"][k], "fp64_finite": finite["fp64"][k]} for k in bad[:20]]
    errs = []
    for k in range(n):
        if finite["fp32s"][k] and finite["fp64"][k]:
            fl = np.asarray(members[k]["mask"]).ravel() != 0
            a, b_ = rho["fp32s"][k][fl], rho["fp64"][k][fl]
            errs.append(float(np.max(np.abs(a - b_)) / np.mean(np.abs(b_))))
    out["fp32s_rho1_max_over_mean_vs_fp64"] = {
        "median": float(np.median(errs)), "max": float(np.max(errs))} if errs else None
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
    for prec, name in ((sc.FP64, "fp64"), (sc.FP32_SHIFTED, "fp32s"), (sc.FP16_SHIFTED, "fp16s")):
        d = sc.Domain(nx, ny, np.ones(N, np.int32),
                      sc.make_params(ncomp=2, g_fluid=(1.2, 1.2), rho_ref=(1.0, 1.0)), prec)
        d.init_noise(0, 1.0, 0.01, 101)
        d.init_noise(1, 1.0, 0.01, 102)
        doms[name] = d
    m0 = {k: d.mass_momentum() for k, d in doms.items()}
    out = {"config": f"spinodal {nx}x{ny} periodic, G=1.2, rho=1+-1%", "steps": steps,
           "device_gb": {k: round(d.device_bytes() / 1e9, 2) for k, d in doms.items()}}
    ms, done, acc = {k: 0.0 for k in doms}, 0, {}
    for cp in (20, steps):
        for k, d in doms.items():
            ms[k] += _timed(torch, stream, lambda: d.step(cp - done))
        done = cp
        ref = [doms["fp64"].download_rho(c) for c in range(2)]
        acc[str(cp)] = {k: [_errors(doms[k].download_rho(c), ref[c]) for c in range(2)]
                        for k in ("fp32s", "fp16s")}
    out["accuracy_vs_fp64"] = acc
    out["mass_drift"] = {k: [float((d.mass_momentum()[3 * c] - m0[k][3 * c]) / m0[k][3 * c])
                             for c in range(2)] for k, d in doms.items()}
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
    for prec, name in ((sc.FP64, "fp64"), (sc.FP32_SHIFTED, "fp32s")):
        ws = [W.contact_angle(g) for g in gs_values]
        doms = []
        for w in ws:
            fl = np.asarray(w["mask"]).ravel() != 0
            rr = tuple(float(w[k].reshape(9, -1).sum(0)[fl].mean()) for k in ("f1", "f2"))
            d = sc.Domain(w["nx"], w["ny"], w["mask"], W.params_of(w, sc, rho_ref=rr), prec)
            d.upload_f(0, w["f1"])
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
        del b, doms
    a, b_ = out["fp64"]["theta_deg"], out["fp32s"]["theta_deg"]
    out["max_abs_theta_diff_fp32s_deg"] = max(
        (abs(x - y) for x, y in zip(a, b_) if x is not None and y is not None), default=None)
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
