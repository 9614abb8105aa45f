"""Autotuner of the batched two-component step (run on a B200).

    python -m sc_lbm_b200.autotune [--out sc_lbm_b200/tuning/b200.json] [--steps 200]

For every domain size class of the ensemble workload (Nx in 64..512, Ny in
64..256) it builds a batch of seeded porous domains of the class's
representative size and times one persistent launch per step (CUDA graph)
over the candidate shapes of each storage precision:

* tile list (variant 2) with tile_y = 4, 8, 16, 32, 64 rows per tile -- the
  nodes each thread advances per tile (one column per thread, 128 threads);
* strips x bands (variant 3, pipelined body; FP64 and FP32 storage).

It then runs one member of the class in FP64 and in the shifted forms for
`--accuracy-steps` steps and records max|drho|/mean(rho) against FP64; the
recommended storage of the class is the fastest whose error stays within
`--tolerance` (1e-5).

Finally it times what a batch actually runs on the benchmark's mixed workload:
the whole seeded 512-domain ensemble (sizes, porosities and parameters mixed
as the configuration draws them) in one batch, for every batch body -- the
ring bodies (variants 11 and 12: 128- and 64-column strips) at several rows
per unit, the tile lists (2 register tile, 8 uniform solid form, 9 half
tiles, 10 one-warp tiles) at several rows per tile, and the strips x bands
body (3) -- per storage precision.  The fastest becomes the `batch_default`
of that precision, the body every batch with solid nodes starts with.  The
JSON it writes is compiled into the library by build.py (sclbm_tuned_config,
the size-class tile heights and the batch defaults).
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

NX_EDGES = (64, 160, 320, 513)
NY_EDGES = (64, 128, 257)
TILE_Y = (4, 8, 16, 32, 64)
PREC_NAMES = ("fp64", "fp32s", "fp16s")


def representative(lo, hi):
    """multiple of 16 near the geometric middle of [lo, hi)"""
    return int(16 * round(np.sqrt(lo * (hi - 1)) / 16))


def make_domains(sc, W, nx, ny, prec, count, distinct=8, seed=4242):
    members = [W.ensemble_member(k, seed, size=(nx, ny)) for k in range(distinct)]
    doms = []
    for k in range(count):
        m = members[k % distinct]
        d = sc.Domain(nx, ny, m["mask"], W.params_of(m, sc), prec)
        d.upload_f(0, m["f1"])
        d.upload_f(1, m["f2"])
        doms.append(d)
    return doms, members


def time_batch(torch, sc, stream, doms, variant, tile_y, steps, warmup):
    b = sc.Batch(doms, tile_y=[tile_y] * len(doms))
    b.set_kernel(variant)
    b.step(max(warmup, 20))  # builds the 20-step CUDA graph outside the timed steps
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.step(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    nodes = sum(d.N for d in doms)
    del b
    return nodes / (ms * 1e-3) / 1e6, ms


def accuracy(sc, W, member, steps):
    """max|drho|/mean(rho) of the shifted forms against FP64 after `steps`."""
    nx, ny = member["nx"], member["ny"]
    fluid = np.asarray(member["mask"]).ravel() != 0
    out, rho64 = {}, None
    for prec, name in ((sc.FP64, "fp64"), (sc.FP32_SHIFTED, "fp32s"), (sc.FP16_SHIFTED, "fp16s")):
        d = sc.Domain(nx, ny, member["mask"], W.params_of(member, sc), prec)
        d.upload_f(0, member["f1"])
        d.upload_f(1, member["f2"])
        d.step(steps)
        rho = [d.download_rho(k)[fluid] for k in range(2)]
        if rho64 is None:
            rho64 = rho
            continue
        out[name] = max(float(np.max(np.abs(rho[k] - rho64[k])) / np.mean(np.abs(rho64[k])))
                        for k in range(2))
    out["fp64"] = 0.0
    return out


# candidates of the mixed-ensemble sweep: (variant, rows per unit / tile)
ENSEMBLE_CANDIDATES = {
    "fp64": [(11, 16), (11, 24), (11, 32), (11, 48), (11, 64), (12, 32), (2, 16), (2, 32), (3, 0)],
    "fp32s": [(11, 16), (11, 24), (11, 32), (11, 48), (11, 64), (12, 32), (2, 16), (8, 16), (8, 32),
              (9, 16), (10, 16), (10, 32), (3, 0)],
    "fp16s": [(11, 16), (11, 32), (11, 64), (12, 32), (2, 32), (8, 16), (8, 32), (10, 16), (10, 32)],
}


def ensemble_sweep(torch, sc, W, stream, steps, warmup, n=512):
    """Mixed-ensemble timings per precision and the fastest body of each."""
    members = W.ensemble(n)
    sweep, best = {}, {}
    for prec, pname in ((sc.FP64, "fp64"), (sc.FP32_SHIFTED, "fp32s"), (sc.FP16_SHIFTED, "fp16s")):
        doms = []
        for m in members:
            d = sc.Domain(m["nx"], m["ny"], m["mask"], W.params_of(m, sc), prec)
            d.upload_f(0, m["f1"])
            d.upload_f(1, m["f2"])
            doms.append(d)
        res = []
        for variant, rows in ENSEMBLE_CANDIDATES[pname]:
            mlups, ms = time_batch(torch, sc, stream, doms, variant, rows or 16, steps, warmup)
            res.append({"variant": variant, "rows": rows, "mlups": round(mlups, 1),
                        "ms_per_step": round(ms, 5)})
            print(json.dumps({"ensemble": pname, **res[-1]}), flush=True)
        sweep[pname] = res
        top = max(res, key=lambda r: r["mlups"])
        best[pname] = {"variant": top["variant"], "rows": top["rows"], "mlups": top["mlups"]}
        del doms
    return sweep, best


def select(results, margin):
    """The shape to use from one precision's sweep: among the candidates within
    `margin` (relative) of the fastest, the tile list with the most rows per
    tile (fewest halo rows, which a mixed batch of small domains pays for more
    than the homogeneous batch timed here), else the fastest."""
    top = max(r["mlups"] for r in results)
    near = [r for r in results if r["mlups"] >= (1.0 - margin) * top]
    lists = [r for r in near if r["variant"] == 2]
    pick = max(lists, key=lambda r: r["tile_y"]) if lists else max(near, key=lambda r: r["mlups"])
    return {"variant": pick["variant"], "tile_y": pick["tile_y"], "mlups": pick["mlups"]}


def reselect(path, margin):
    """Re-apply the selection rule to a committed sweep (no GPU needed)."""
    with open(path) as fh:
        d = json.load(fh)
    for c in d["classes"]:
        for p in PREC_NAMES:
            c["shapes"][p] = select(c["sweep"][p], margin)
    d["margin"] = margin
    with open(path, "w") as fh:
        json.dump(d, fh, indent=1)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "tuning", "b200.json"))
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=40)
    ap.add_argument("--nodes", type=float, default=4e6, help="lattice nodes per timed batch")
    ap.add_argument("--accuracy-steps", type=int, default=100)
    ap.add_argument("--tolerance", type=float, default=1e-5)
    ap.add_argument("--margin", type=float, default=0.03,
                    help="shapes within this fraction of the fastest count as equal")
    ap.add_argument("--reselect", action="store_true",
                    help="re-apply the selection rule to the sweep in --out and exit")
    ap.add_argument("--ensemble-only", action="store_true",
                    help="only the mixed-ensemble sweep, merged into the existing --out")
    args = ap.parse_args()
    if args.reselect:
        reselect(args.out, args.margin)
        print(f"re-selected {args.out}")
        return

    import torch
    import sc_lbm_b200 as sc
    from sc_lbm_b200 import workloads as W

    stream = torch.cuda.Stream()
    sc.set_stream(stream.cuda_stream)
    props = torch.cuda.get_device_properties(0)
    t_start = time.time()
    if args.ensemble_only:
        with open(args.out) as fh:
            out = json.load(fh)
        out["ensemble_sweep"], out["batch_default"] = ensemble_sweep(torch, sc, W, stream, args.steps,
                                                                     args.warmup)
        out["ensemble_command"] = "python -m sc_lbm_b200.autotune " + " ".join(sys.argv[1:])
        with open(args.out, "w") as fh:
            json.dump(out, fh, indent=1)
        print(f"wrote {args.out}")
        return
    classes = []
    for i in range(len(NX_EDGES) - 1):
        for j in range(len(NY_EDGES) - 1):
            nx = representative(NX_EDGES[i], NX_EDGES[i + 1])
            ny = representative(NY_EDGES[j], NY_EDGES[j + 1])
            count = int(max(32, min(512, args.nodes // (nx * ny))))
            sweep, shapes = {}, {}
            members = None
            for prec, pname in ((sc.FP64, "fp64"), (sc.FP32_SHIFTED, "fp32s"),
                                (sc.FP16_SHIFTED, "fp16s")):
                doms, members = make_domains(sc, W, nx, ny, prec, count)
                cands = [(2, ty) for ty in TILE_Y] + ([(3, 0)] if pname != "fp16s" else [])
                res = []
                for variant, ty in cands:
                    mlups, ms = time_batch(torch, sc, stream, doms, variant, ty or 16,
                                           args.steps, args.warmup)
                    res.append({"variant": variant, "tile_y": ty or 16, "mlups": round(mlups, 1),
                                "ms_per_step": round(ms, 5)})
                sweep[pname] = res
                shapes[pname] = select(res, args.margin)
                del doms
            err = accuracy(sc, W, members[0], args.accuracy_steps)
            ok = [p for p in PREC_NAMES if err[p] <= args.tolerance]
            rec = max(ok, key=lambda p: shapes[p]["mlups"])
            c = {"nx": [NX_EDGES[i], NX_EDGES[i + 1]], "ny": [NY_EDGES[j], NY_EDGES[j + 1]],
                 "representative": [nx, ny], "domains": count, "precision": rec,
                 "shapes": shapes, "error_vs_fp64": err, "sweep": sweep}
            classes.append(c)
            print(json.dumps({k: c[k] for k in ("nx", "ny", "representative", "domains",
                                                  "precision", "shapes", "error_vs_fp64")}),
                  flush=True)
    out = {"device": props.name, "sm_count": props.multi_processor_count,
           "command": "python -m sc_lbm_b200.autotune " + " ".join(sys.argv[1:]),
           "steps": args.steps, "warmup": args.warmup, "accuracy_steps": args.accuracy_steps,
           "tolerance": args.tolerance, "margin": args.margin,
           "seconds": round(time.time() - t_start, 1),
           "note": "tile_y = rows (nodes per thread) per tile of the tile-list kernel; "
                   "variant 2 = tile list, 3 = strips x bands; mlups of a batch of "
                   "`domains` seeded porous domains of the representative size",
           "classes": classes}
    out["ensemble_sweep"], out["batch_default"] = ensemble_sweep(torch, sc, W, stream, args.steps,
                                                                 args.warmup)
    out["seconds"] = round(time.time() - t_start, 1)
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    with open(args.out, "w") as fh:
        json.dump(out, fh, indent=1)
    print(f"wrote {args.out}")


if __name__ == "__main__":
    main()
