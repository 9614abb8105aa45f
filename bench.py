"""Benchmark of the sc_lbm D2Q9 Shan-Chen step on B200.

Workload (the north-star headline): a 4096x4096 fully periodic two-component
spinodal decomposition (tau = 1, G12 = 1.2, rho1 = rho2 = 1 +- 1% seeded
noise), stored in the FP32-shifted form (f_i - w_i*rho_ref in float, float
arithmetic); the plain FP64 GPU form is timed on the same lattice for the
>= 2x comparison and the density error of FP32 against FP64 is reported.
Inputs are generated from a seeded splitmix64 stream ("data": "synthetic").

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line is printed by rank 0.  Under torchrun each rank advances its own
independent replica (weak scaling, no collective on the data path); the time
is the max over ranks.  Without torchrun, `--gpus N` (N > 1) starts the N rank
processes itself (RANK / LOCAL_RANK / WORLD_SIZE / MASTER_* set per process).
`--impl reference` times the reference's own serial CPU step (oracle/_ref, the
unmodified library compiled from its sources; or, when that was not built,
the C restatement in oracle/) on the same 4096x4096 lattice, pinned to one
core; it stops after a bounded time (at least three timed steps) and says how
many steps it timed.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX = NY = 4096
G12 = 1.2
B_LU = {"fp64": 36 * 8 + 1, "fp32s": 36 * 4 + 1, "fp16s": 36 * 2 + 1}  # bytes / lattice update
E2E_STEPS = 100  # LBM steps per end-to-end call
REF_BUDGET_S = 240.0  # reference arm: stop timing after this long (>= 3 timed steps)
CPU_LEG_STEPS = (1, 3)  # our arm's CPU-baseline leg: warm-up and timed steps


def env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), \
        int(os.environ.get("LOCAL_RANK", "0"))


class Ranks:
    """One process per GPU under torchrun: the barrier and the max over ranks
    of device-timed values (NCCL on GPUs; gloo with device "cpu" in the CPU
    tests).  World size 1 needs no process group."""

    def __init__(self, backend="nccl", device="cuda"):
        import datetime
        import torch
        import torch.distributed as dist
        self.torch, self.dist, self.device = torch, dist, device
        self.rank, self.world, self.local = env_rank()
        self.owns_group = False
        if self.world > 1 and not dist.is_initialized():
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
            self.owns_group = True

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()
        if self.device == "cuda":
            self.torch.cuda.synchronize()

    def max(self, x: float) -> float:
        if self.world == 1:
            return x
        t = self.torch.tensor([float(x)], dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def whole_job_mlups(self, nodes_per_rank: int, steps: int, ms_max: float) -> float:
        """Lattice updates of all ranks over the slowest rank's time."""
        return self.world * nodes_per_rank * steps / (ms_max * 1e-3) / 1e6

    def close(self):
        if self.owns_group:
            self.dist.destroy_process_group()
            self.owns_group = False


def seeded_populations(nx, ny, seed):
    """f_i = rho/9 with rho = 1 +- 1% (the reference initialisers' rho/9 shape)."""
    from sc_lbm_b200.workloads import uniform
    N = nx * ny
    r = 1.0 + 0.01 * (2.0 * uniform(seed, N) - 1.0)
    return np.tile(r / 9.0, 9)


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kernel_key):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) from
    the committed ncu summaries: a line `traffic_per_launch[<key>] = <bytes>`."""
    import glob
    import re
    pat = re.compile(r"^traffic_per_launch\[(\w+)\]\s*=\s*(\d+)\s*$", re.M)
    for p in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        with open(p) as fh:
            for key, val in pat.findall(fh.read()):
                if key == kernel_key:
                    return int(val)
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            time.sleep(0.3)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------
def reference_steps(nx, ny, warmup, steps, budget_s):
    """Per-step seconds of the reference's serial step on an nx x ny lattice,
    pinned to one core: the compiled reference (oracle/_ref) when it was
    built, else the C restatement.  Timing stops after budget_s seconds once
    three steps past the warm-up have run.  Returns (seconds, kind, info)."""
    from oracle import pyoracle
    info = pyoracle.cpu_info()
    if pyoracle.have_ref():
        r = pyoracle.ref_bench(nx, ny, warmup + steps, core=info["pin_core"],
                               max_seconds=budget_s, min_steps=warmup + min(3, steps))
        return r["step_seconds"][warmup:], "reference", info
    return cpu_port_steps(nx, ny, warmup + steps, info["pin_core"], budget_s,
                          warmup + min(3, steps))[warmup:], "port", info


def run_reference(args):
    rank, world, _ = env_rank()
    check_world(args, world)
    if rank != 0:
        return
    from oracle import pyoracle
    nx, ny = args.lattice
    warm = min(args.warmup, 3)
    per, kind, info = reference_steps(nx, ny, warm, args.steps, REF_BUDGET_S)
    t = sum(per)
    mlups = nx * ny * len(per) / t / 1e6
    # The reference is serial: one lattice runs on one core, which is the
    # headline reference value.  For context, the whole host's throughput on
    # independent lattices (one serial run per core, 512 x 512, 10 steps).
    all_cores = None
    if kind == "reference":
        cores = max(1, min(info["usable"], 64))
        par = pyoracle.ref_bench_parallel(512, 512, 10, cores)
        all_cores = {"instances": cores, "value": round(par["mlups"], 3), "unit": "MLUPS",
                     "sample": "independent 512x512 lattices, 10 steps each, one serial "
                               "reference run per core at once"}
    same = (nx, ny) == (NX, NY)
    line = {
        "metric": "two-component D2Q9 Shan-Chen step throughput", "value": round(mlups, 4),
        "unit": "MLUPS", "impl": "reference", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1e3 * t / len(per), 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"spinodal two-component {nx}x{ny} periodic, tau=1, G12={G12}, "
                               "rho=1+-1% seeded" + ("" if same else " (reduced lattice)"),
                   "lattice": [nx, ny], "precision": "fp64 (reference serial C++)",
                   "timed_steps": len(per), "warmup_steps_run": warm,
                   "time_budget_s": REF_BUDGET_S},
        "cpu_baseline": {"value": round(mlups, 4), "unit": "MLUPS", "cores": 1, "kind": kind,
                         "sample": f"{len(per)} steps of the {nx}x{ny} two-component periodic "
                                   "lattice after " + f"{warm} warm-up steps, reference call "
                                   "sequence laplace_law.cpp:123-133",
                         "cpu_model": info["model"], "nproc": info["nproc"],
                         "pinned_core": info["pin_core"], "all_cores": all_cores},
        "e2e": {"value": round(mlups, 4), "unit": "MLUPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "gpu_launches": 0,
    }
    print(json.dumps(line), flush=True)


def cpu_config_runs(sample_steps=10, members=8, member_steps=200):
    """The reference's serial code on every configuration, pinned to one core:
    full runs of the Poiseuille channel (200x50, 10,000 steps) and the Laplace
    droplet (256x256, radius 40, 20,000 steps); `sample_steps` steady steps of
    the 2048x1024 drainage lattice; `member_steps` steps of each of the first
    `members` ensemble domains (the ensemble's serial time is estimated from
    their aggregate rate); and the 4096x4096 two-component lattice, the
    stand-in for the 16384x8192 spinodal lattice (about 80 GB of host memory
    in the reference's layout), whose per-node work it shares."""
    from oracle import pyoracle
    from sc_lbm_b200 import workloads as W
    info = pyoracle.cpu_info()
    core = info["pin_core"]

    def two(w, steps, fl1, fl2, force=(0, [0.0] * 9)):
        nx, ny = w["nx"], w["ny"]
        m = np.asarray(w["mask"]).reshape(ny, nx)
        ys, xs = np.nonzero(m == 0)
        return dict(nx=nx, ny=ny, geom=[("solid_node", int(x), int(y)) for y, x in zip(ys, xs)],
                    mode="two", fluid1=fl1, fluid2=fl2,
                    init=("file", np.concatenate([w["f1"], w["f2"]])), force=force, steps=steps)

    def timed(label, case, full):
        r = pyoracle.run_ref(case, core=core, timing=True)
        t = float(r["loop_seconds"][0])
        n = case["nx"] * case["ny"]
        return {"config": label, "lattice": [case["nx"], case["ny"]], "steps": case["steps"],
                "full_run": full, "loop_seconds": round(t, 3),
                "mlups": round(n * case["steps"] / t / 1e6, 4)}

    out = []
    w = W.poiseuille()
    out.append(timed("1 poiseuille 200x50 FP64", dict(
        nx=200, ny=50, geom=[("walls", 1, "x")], mode="single", fluid1=(1.0, 0, 0),
        init=("simple", 1.0), force=(1, list(w["force"])), steps=10000), True))
    w = W.laplace(40)
    out.append(timed("2 laplace 256x256 radius 40", two(w, 20000, (1.0, 0.9, 0.0), (1.0, 0.9, 0.0)),
                     True))
    w = W.drainage()
    out.append(timed("3 drainage 2048x1024 porous (sampled steps)",
                     two(w, sample_steps, (1.0, 0.9, -0.2), (1.0, 0.9, 0.2),
                         (1, list(w["force1"]))), False))
    nodes = t = 0.0
    sizes = []
    for k in range(members):
        m = W.ensemble_member(k)
        r = timed(f"member {k}", two(m, member_steps, (m["tau"][0], m["G"], m["Gs"][0]),
                                     (m["tau"][1], m["G"], m["Gs"][1])), False)
        nodes += m["nx"] * m["ny"] * member_steps
        t += r["loop_seconds"]
        sizes.append([m["nx"], m["ny"]])
    ens = W.ensemble(512)
    total = sum(m["nx"] * m["ny"] for m in ens)
    out.append({"config": "4 ensemble of 512 (sampled members, serial)", "members_timed": sizes,
                "steps": member_steps, "full_run": False, "mlups": round(nodes / t / 1e6, 4),
                "estimated_serial_seconds_10000_steps": round(total * 10000 / (nodes / t), 1)})
    r = pyoracle.ref_bench(4096, 4096, 4, core=core, max_seconds=120.0, min_steps=2)
    per = r["step_seconds"][1:]
    out.append({"config": "5 spinodal (4096x4096 stand-in for 16384x8192, sampled steps)",
                "lattice": [4096, 4096], "steps": len(per), "full_run": False,
                "mlups": round(4096 * 4096 * len(per) / sum(per) / 1e6, 4)})
    return {"cores": 1, "pinned_core": core, "cpu_model": info["model"], "nproc": info["nproc"],
            "kind": "reference", "runs": out}


def cpu_port_steps(nx, ny, steps, core=None, budget_s=0.0, min_steps=1):
    """Per-step seconds of the C restatement (oracle/) -- the fallback CPU arm
    (this process pinned to `core` while it runs)."""
    import ctypes as C
    from oracle import pyoracle
    old_aff = None
    if core is not None and hasattr(os, "sched_setaffinity"):
        old_aff = os.sched_getaffinity(0)
        os.sched_setaffinity(0, {core})
    L = pyoracle.lib()
    N = nx * ny
    g = np.ones(N, np.uint8)
    f = seeded_populations(nx, ny, 7)
    comps = []
    keep = []
    zero = np.zeros(N)
    for k in range(2):
        arr = dict(f=f.copy(), feq=np.zeros(9 * N), rho=np.zeros(N), ux=np.zeros(N),
                   uy=np.zeros(N), uex=np.zeros(N), uey=np.zeros(N), frx=np.zeros(N),
                   fry=np.zeros(N))
        keep.append(arr)
        c = pyoracle._Comp(*[pyoracle._p(arr[n]) for n in ("f", "feq", "rho", "ux", "uy", "uex",
                                                          "uey", "frx", "fry")],
                           pyoracle._p(zero), pyoracle._p(zero), 1.0, G12)
        comps.append(c)
    tmp = np.zeros(9 * N)
    out = []
    start = time.perf_counter()
    for k in range(steps):
        t0 = time.perf_counter()
        L.orc_run_two(nx, ny, pyoracle._p(g), C.byref(comps[0]), C.byref(comps[1]), None, 0, 1,
                      pyoracle._p(tmp))
        out.append(time.perf_counter() - t0)
        if budget_s > 0 and k + 1 >= min_steps and time.perf_counter() - start > budget_s:
            break
    if old_aff is not None:
        os.sched_setaffinity(0, old_aff)
    return out


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def accuracy_report(sc, mask, params, f1, f2, checkpoints=(20, 200)):
    """Shifted forms against the FP64 GPU form (itself bit-exact with the
    reference) from the same start, plus an FP64 twin whose component-1
    populations start one ulp away: the twin's divergence is the amplification
    the spinodal dynamics applies to any rounding difference.  Per component:
    density error max and RMS over the mean density, velocity (u = j / rho)
    error max over max |u| and RMS over RMS |u|; mass drift per component."""
    from sc_lbm_b200.validation import compare_domains, mass_drift, twin_populations
    NXY = mask.size
    doms = {"fp64": sc.Domain(NX, NY, mask, params, sc.FP64),
            "fp64_1ulp_twin": sc.Domain(NX, NY, mask, params, sc.FP64),
            "fp32s": sc.Domain(NX, NY, mask, params, sc.FP32_SHIFTED),
            "fp16s": sc.Domain(NX, NY, mask, params, sc.FP16_SHIFTED)}
    for name, d in doms.items():
        d.upload_f(0, twin_populations(f1) if name == "fp64_1ulp_twin" else f1)
        d.upload_f(1, f2)
    m0 = {k: d.mass_momentum() for k, d in doms.items()}
    rep, done = {"metric": "per component: rho_max / rho_rms = max / RMS |drho| over mean rho; "
                           "u_max = max |du| / max |u|, u_rms = RMS |du| / RMS |u|; vs FP64"}, 0
    for cp in checkpoints:
        for d in doms.values():
            d.step(cp - done)
        done = cp
        rep[f"step_{cp}"] = compare_domains(doms)
    rep["mass_drift"] = {k: mass_drift(d, m0[k]) for k, d in doms.items()}
    rep["nodes"] = NXY
    del doms
    return rep


def time_domain(torch, sc, dom, stream, steps, warmup):
    """Device time of `steps` fused steps, CUDA events on the launching stream."""
    dom.step(warmup)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    dom.step(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def run_ensemble(torch, sc, stream, steps, warmup, single_mlups, ranks, n=512):
    """The uneven ensemble (512 seeded porous two-component domains, Nx in
    64..512, Ny in 64..256, per-domain G, Gs, tau) advanced by one batch:
    one persistent launch per step from a CUDA graph, tuned tile shapes.
    Each rank advances its own ensemble (weak scaling); times are the max over
    ranks and the MLUPS count every rank's nodes."""
    from sc_lbm_b200 import workloads as W
    t0 = time.time()
    members = W.ensemble(n, seed=2024 + ranks.rank)
    doms = []
    for m in members:
        d = sc.Domain(m["nx"], m["ny"], m["mask"], W.params_of(m, sc), sc.FP32_SHIFTED)
        d.upload_f(0, m["f1"])
        d.upload_f(1, m["f2"])
        doms.append(d)
    setup_s = time.time() - t0
    nodes = sum(d.N for d in doms)
    b = sc.Batch(doms)
    ntiles, grid = b.info()
    # the first 20 steps capture and instantiate the batch's CUDA graph: keep
    # that out of the timed region
    b.step(20)
    b.step(warmup)
    ranks.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.step(steps)
    e1.record(stream)
    ranks.barrier()
    ms = ranks.max(e0.elapsed_time(e1)) / steps
    mlups = ranks.whole_job_mlups(nodes, 1, ms)
    fluid = sum(int(np.count_nonzero(m["mask"])) for m in members)
    del b, doms
    # one large porous domain of the same geometry class (disks of radius 2-8 at
    # the ensemble's mean fluid fraction), same storage, same timing
    from sc_lbm_b200.validation import _porous_single
    P, phi = _porous_single(sc, W, 4096, 4096, fluid / nodes, sc.FP32_SHIFTED)
    P.step(warmup)
    ranks.barrier()
    e0.record(stream)
    P.step(steps)
    e1.record(stream)
    ranks.barrier()
    porous_mlups = ranks.whole_job_mlups(4096 * 4096, 1, ranks.max(e0.elapsed_time(e1)) / steps)
    del P
    return {"value": round(mlups, 2), "unit": "MLUPS", "ms_per_step": round(ms, 5),
            "domains": n, "nodes": nodes, "fluid_fraction": round(fluid / nodes, 4),
            "efficiency_vs_single_4096": round(mlups / single_mlups, 4),
            "single_porous_4096_mlups": round(porous_mlups, 2),
            "single_porous_fluid_fraction": round(phi, 4),
            "efficiency_vs_single_porous_4096": round(mlups / porous_mlups, 4),
            "tiles": ntiles, "ctas": grid, "precision": "fp32_shifted", "setup_s": round(setup_s, 1),
            "workload": f"{n} seeded porous two-component domains, Nx 64..512 x Ny 64..256 "
                        "(multiples of 16), porosity 0.5-0.9, G 0.8-1.2, Gs -0.3..0.3, "
                        "tau 0.6-1.5; one launch per step (CUDA graph), tuned tiles"}


def run_ours(args):
    import torch
    import sc_lbm_b200 as sc

    rank, world, local = env_rank()
    check_world(args, world)
    torch.cuda.set_device(local)
    ranks = Ranks("nccl", "cuda")
    stream = torch.cuda.Stream()
    sc.set_stream(stream.cuda_stream)

    N = NX * NY
    mask = np.ones(N, np.int32)
    f1 = seeded_populations(NX, NY, 101 + 2 * rank)
    f2 = seeded_populations(NX, NY, 102 + 2 * rank)
    params = sc.make_params(ncomp=2, tau=(1.0, 1.0), g_fluid=(G12, G12), g_solid=(0.0, 0.0),
                            rho_ref=(1.0, 1.0))

    barrier, max_over_ranks = ranks.barrier, ranks.max

    # --- FP32-shifted headline -------------------------------------------------
    d32 = sc.Domain(NX, NY, mask, params, sc.FP32_SHIFTED)
    d32.upload_f(0, f1)
    d32.upload_f(1, f2)
    barrier()
    with ClockSampler(local) as clk:
        barrier()
        ms = time_domain(torch, sc, d32, stream, args.steps, args.warmup)
        barrier()
    ms = max_over_ranks(ms)
    clocks = clk.summary()
    ms_step = ms / args.steps
    mlups32 = world * N / (ms_step * 1e-3) / 1e6

    # --- FP64 GPU form (same lattice, same start) ---------------------------
    d64 = sc.Domain(NX, NY, mask, params, sc.FP64)
    d64.upload_f(0, f1)
    d64.upload_f(1, f2)
    k64 = max(10, args.steps // 2)
    ms64 = max_over_ranks(time_domain(torch, sc, d64, stream, k64, args.warmup)) / k64
    mlups64 = world * N / (ms64 * 1e-3) / 1e6

    # --- FP16-shifted timing (same lattice, same start) ----------------------
    d16 = sc.Domain(NX, NY, mask, params, sc.FP16_SHIFTED)
    d16.upload_f(0, f1)
    d16.upload_f(1, f2)
    ms16 = max_over_ranks(time_domain(torch, sc, d16, stream, args.steps, args.warmup)) / args.steps
    del d16

    ensemble = None if args.no_batch else run_ensemble(torch, sc, stream, args.steps, args.warmup,
                                                       mlups32, ranks)

    accuracy = accuracy_report(sc, mask, params, f1, f2) if rank == 0 else None

    # --- end to end through the C ABI with pinned host buffers ----------------
    f1p = torch.empty(9 * N, dtype=torch.float64, pin_memory=True).numpy()
    f2p = torch.empty(9 * N, dtype=torch.float64, pin_memory=True).numpy()
    f1p[:] = f1
    f2p[:] = f2
    r1p = torch.empty(N, dtype=torch.float64, pin_memory=True).numpy()
    r2p = torch.empty(N, dtype=torch.float64, pin_memory=True).numpy()
    d32.run(f1p, f2p, 2, r1p, r2p)  # warm
    e2e_calls = 3
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_calls):
        d32.run(f1p, f2p, E2E_STEPS, r1p, r2p)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0) / e2e_calls
    e2e_mlups = world * N * E2E_STEPS / e2e_s / 1e6

    # --- CPU baseline (reference serial code, same lattice, a few steps) -------
    cpu = None
    if rank == 0 and not args.no_cpu:
        w, k = CPU_LEG_STEPS
        per, kind, info = reference_steps(NX, NY, w, k, 60.0)
        cpu = {"value": round(NX * NY * len(per) / sum(per) / 1e6, 4), "unit": "MLUPS",
               "cores": 1, "kind": kind,
               "sample": f"{len(per)} steps of the {NX}x{NY} two-component periodic lattice "
                         f"after {w} warm-up step (reference call sequence "
                         "laplace_law.cpp:123-133), one pinned core",
               "cpu_model": info["model"], "nproc": info["nproc"], "pinned_core": info["pin_core"]}

    peak, peak_kind = measured_peak_hbm()
    achieved = B_LU["fp32s"] * N / (ms_step * 1e-3) / 1e9
    line = {
        "metric": "two-component D2Q9 Shan-Chen step throughput", "value": round(mlups32, 2),
        "unit": "MLUPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms_step, 5), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"spinodal two-component {NX}x{NY} periodic, tau=1, G12={G12}, "
                               "rho=1+-1% seeded, FP32-shifted storage",
                   "lattice": [NX, NY], "precision": "fp32_shifted",
                   "kernel": "fused single pass, TMA row ring (4 stages, 24-row bands; density recomputed per band)",
                   "l2": "inputs larger than L2 (2 x 1.2 GB population buffers)",
                   "parallelism": f"replicas{world}"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "traffic": ncu_traffic("ring_fp32s_4096"),
                     "bytes_per_update": B_LU["fp32s"], "peak_source": peak_kind},
        "fp64": {"value": round(mlups64, 2), "unit": "MLUPS", "ms_per_step": round(ms64, 5),
                 "frac": round(B_LU["fp64"] * N / (ms64 * 1e-3) / 1e9 / peak, 4),
                 "traffic": ncu_traffic("ring_fp64_4096"),
                 "speedup_fp32s_over_fp64": round(mlups32 / mlups64, 3)},
        "fp16": {"value": round(world * N / (ms16 * 1e-3) / 1e6, 2), "unit": "MLUPS",
                 "ms_per_step": round(ms16, 5),
                 "frac": round(B_LU["fp16s"] * N / (ms16 * 1e-3) / 1e9 / peak, 4),
                 "traffic": ncu_traffic("ring_fp16s_4096")},
        "ensemble": ensemble,
        "accuracy": accuracy,
        "e2e": {"value": round(e2e_mlups, 2), "unit": "MLUPS",
                "h2d_bytes_per_step": 2 * 9 * N * 8, "d2h_bytes_per_step": 2 * N * 8,
                "lbm_steps_per_step": E2E_STEPS,
                "call": "sclbm_domain_run (upload FP64 populations, 100 steps, download rho)"},
        "clocks": clocks,
        "gpu_launches": args.steps,
        "cpu_baseline": cpu,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    ranks.close()


def check_world(args, world):
    if world != args.gpus:
        raise SystemExit(f"bench.py --gpus {args.gpus} but {world} rank process(es) are running")


def self_launch(argv, n):
    """Start the n rank processes of `bench.py --gpus n` when no launcher did:
    one process per GPU with RANK / LOCAL_RANK / WORLD_SIZE / MASTER_ADDR /
    MASTER_PORT set, rank 0's output passed through; exit status = the worst."""
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    procs = []
    for r in range(n):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(n),
                   LOCAL_WORLD_SIZE=str(n), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, os.path.abspath(__file__)] + argv, env=env))
    rcs = [p.wait() for p in procs]
    return max(abs(rc) for rc in rcs)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-batch", action="store_true", help="skip the 512-domain ensemble leg")
    ap.add_argument("--cpu-configs", action="store_true",
                    help="time the reference's serial code on every configuration (CPU only)")
    ap.add_argument("--out", default=None, help="--cpu-configs: write the results here")
    ap.add_argument("--lattice", type=int, nargs=2, default=[NX, NY], metavar=("NX", "NY"),
                    help="reference arm only: a smaller lattice for quick checks (labelled)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(self_launch(sys.argv[1:], args.gpus))
    if args.cpu_configs:
        res = cpu_config_runs()
        print(json.dumps(res), flush=True)
        if args.out:
            with open(args.out, "w") as fh:
                json.dump(res, fh, indent=1)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
