"""Run a few fused steps on one domain -- the command the committed ncu
summaries under profiles/ were captured with.

    python -m sc_lbm_b200.profile_case --nx 2048 --ny 2048 --precision fp32 --steps 3

Two-component periodic spinodal lattice (tau = 1, G12 = 1.2, rho = 1 +- 1%),
`--warmup` untimed steps then `--steps` steps; prints the CUDA-event time per
step.  Sized by the caller so an ncu capture stays small.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=2048)
    ap.add_argument("--ny", type=int, default=2048)
    ap.add_argument("--precision", default="fp32", choices=["fp64", "fp32", "fp16"])
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--variant", type=int, default=0)
    ap.add_argument("--tile-y", type=int, default=0)
    ap.add_argument("--threads", type=int, default=128)
    ap.add_argument("--porosity", type=float, default=1.0,
                    help="< 1: seeded disks of radius 8-20 and walls top and bottom")
    ap.add_argument("--force", action="store_true", help="body force 1e-5 along x on component 1")
    ap.add_argument("--disks", type=int, nargs=2, default=[8, 20], metavar=("RMIN", "RMAX"),
                    help="disk radii of --porosity (2 8: the ensemble's geometry, no walls)")
    ap.add_argument("--ensemble", type=int, default=0,
                    help="> 0: time a batch of that many seeded ensemble domains instead")
    args = ap.parse_args()

    import torch
    import sc_lbm_b200 as sc
    from sc_lbm_b200 import workloads as W

    prec = {"fp64": sc.FP64, "fp32": sc.FP32_SHIFTED, "fp16": sc.FP16_SHIFTED}[args.precision]
    stream = torch.cuda.Stream()
    sc.set_stream(stream.cuda_stream)
    if args.ensemble > 0:
        members = W.ensemble(args.ensemble)
        doms = []
        for m in members:
            dm = sc.Domain(m["nx"], m["ny"], m["mask"], W.params_of(m, sc), prec)
            dm.upload_f(0, m["f1"])
            dm.upload_f(1, m["f2"])
            doms.append(dm)
        N = sum(dm.N for dm in doms)
        d = sc.Batch(doms)
        if args.variant:
            d.set_kernel(args.variant)
    else:
        N = args.nx * args.ny
        if args.porosity < 1.0:
            if args.disks == [8, 20]:
                mask, _, _ = W.disk_mask(args.nx, args.ny, args.porosity, 8, 20, 11, walls="x")
            else:
                mask, _, _ = W.disk_mask(args.nx, args.ny, args.porosity, args.disks[0], args.disks[1],
                                         31337, max_tries=400000, max_misses=2000)
        else:
            mask = np.ones(N, np.int32)
        rng = np.random.default_rng(1)
        f = [W.populations(1.0 + 0.02 * (rng.random(N) - 0.5), mask) for _ in range(2)]
        d = sc.Domain(args.nx, args.ny, mask,
                      sc.make_params(ncomp=2, g_fluid=(1.2, 1.2), g_solid=(-0.2, 0.2),
                                     rho_ref=(1.0, 1.0),
                                     force=(W.force_vec(1e-5) if args.force else None, None)),
                      prec)
        d.set_kernel(args.variant, args.tile_y)
        d.set_threads(args.threads)
        d.upload_f(0, f[0])
        d.upload_f(1, f[1])
    d.step(args.warmup)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    d.step(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(args.steps, 1)
    print(json.dumps({"nx": args.nx, "ny": args.ny, "precision": args.precision,
                      "variant": args.variant, "porosity": args.porosity, "force": args.force,
                      "ensemble": args.ensemble, "nodes": N, "ms_per_step": ms,
                      "mlups": N / (ms * 1e-3) / 1e6}))


if __name__ == "__main__":
    main()
