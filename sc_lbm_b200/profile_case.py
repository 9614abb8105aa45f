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
    args = ap.parse_args()

    import torch
    import sc_lbm_b200 as sc

    prec = {"fp64": sc.FP64, "fp32": sc.FP32_SHIFTED, "fp16": sc.FP16_SHIFTED}[args.precision]
    N = args.nx * args.ny
    rng = np.random.default_rng(1)
    f = [np.tile((1.0 + 0.02 * (rng.random(N) - 0.5)) / 9.0, 9) for _ in range(2)]
    stream = torch.cuda.Stream()
    sc.set_stream(stream.cuda_stream)
    d = sc.Domain(args.nx, args.ny, np.ones(N, np.int32),
                  sc.make_params(ncomp=2, g_fluid=(1.2, 1.2), rho_ref=(1.0, 1.0)), prec)
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
                      "variant": args.variant, "ms_per_step": ms,
                      "mlups": N / (ms * 1e-3) / 1e6}))


if __name__ == "__main__":
    main()
