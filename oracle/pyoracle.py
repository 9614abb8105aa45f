"""numpy front-end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loads ``oracle/libsclbm_oracle.so`` (the plain-C restatement of the sc_lbm
step, built by ``oracle/Makefile``) and, when it has been built here,
``oracle/_ref/sclbm_ref_runner`` (the unmodified reference compiled from its
own sources).  Only the tests, ``__graft_entry__.smoke()`` and bench.py's
CPU-baseline / reference legs import this module, and only as the checker.

A *case* is a plain dict shared by the oracle, the reference runner and the
GPU library tests::

    dict(nx=.., ny=.., geom=[("walls", 1, "x"), ("circle", 11, 30, 20), ...],
         mode="two" | "single" | "ops1" | "ops2" | "mask",
         fluid1=(tau, G, Gs), fluid2=(tau, G, Gs),
         init=("file", f) | ("droplet", 7 args) | ("rectangle", 8 args) | ("simple", rho0),
         force=(mode, [9 doubles]), steps=N)

``force`` mode: 0 none, 1 single-fluid overload on component 1, 2 on
component 2, 3 the two-fluid overload (src/lbm.cpp:315-340).
"""
from __future__ import annotations

import ctypes as C
import os
import struct
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsclbm_oracle.so")
REF_RUNNER = os.path.join(HERE, "_ref", "sclbm_ref_runner")

ERR_NAMES = {0: "ok", 1: "invalid_argument", 2: "runtime_error", 3: "out_of_range", 4: "domain_error"}

_lib = None


def build(ref: bool = True) -> None:
    """Compile the oracle (and the reference runner when its sources exist)."""
    targets = ["oracle"] + (["ref"] if ref else [])
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build(ref=False)
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


def have_ref() -> bool:
    return os.path.exists(REF_RUNNER)


_D = C.POINTER(C.c_double)
_U8 = C.POINTER(C.c_uint8)
_SZ = C.c_size_t


class _Comp(C.Structure):
    _fields_ = [(n, _D) for n in ("f", "feq", "rho", "ux", "uy", "uex", "uey", "frx", "fry",
                                   "fsx", "fsy")] + [("omega", C.c_double), ("G", C.c_double)]


def _declare(L):
    L.orc_geom_add_walls.argtypes = [_U8, _SZ, _SZ, _SZ, C.c_char_p]
    for n in ("orc_geom_add_rectangle", "orc_geom_add_ellipse"):
        getattr(L, n).argtypes = [_U8, _SZ, _SZ, _SZ, _SZ, _SZ, _SZ]
    for n in ("orc_geom_add_square", "orc_geom_add_circle"):
        getattr(L, n).argtypes = [_U8, _SZ, _SZ, _SZ, _SZ, _SZ]
    L.orc_geom_add_array.argtypes = [_U8, _SZ, _SZ, C.c_char_p, C.POINTER(_SZ), _SZ,
                                     C.POINTER(_SZ), _SZ, _SZ, C.c_int]
    L.orc_compute_density.argtypes = [_SZ, _D, _D]
    L.orc_compute_velocities.argtypes = [_SZ, _U8, _D, _D, _D, _D]
    L.orc_feq_single.argtypes = [_SZ, _U8, _D, _D, _D, _D, _D]
    L.orc_feq_multi.argtypes = [_SZ, _D, _D, _D, _D]
    L.orc_init_droplet.argtypes = [_SZ, _SZ, _U8, _D, _D] + [C.c_double] * 7
    L.orc_init_rectangle.argtypes = [_SZ, _SZ, _U8, _D, _D] + [C.c_double] * 8
    L.orc_simple_ini.argtypes = [_SZ, _U8, _D, C.c_double]
    L.orc_solid_sum.argtypes = [_SZ, _SZ, _U8, _D, _D]
    L.orc_surface_force.argtypes = [_SZ, C.c_double, _D, _D, _D, _D]
    L.orc_repulsive.argtypes = [_SZ, _SZ, _U8, _D, _D, C.c_double, C.c_double, _D, _D, _D, _D]
    L.orc_eqvel.argtypes = [_SZ, _SZ, _U8, C.c_double, C.c_double] + [_D] * 20
    L.orc_collide.argtypes = [_SZ, C.c_double, _D, _D]
    L.orc_volume_force.argtypes = [_SZ, _U8, _D, _D]
    L.orc_stream.argtypes = [_SZ, _SZ, _U8, _D, _D]
    L.orc_run_two.argtypes = [_SZ, _SZ, _U8, C.POINTER(_Comp), C.POINTER(_Comp), _D, C.c_int,
                              C.c_int, _D]
    L.orc_run_single.argtypes = [_SZ, _SZ, _U8, C.c_double, _D, _D, _D, _D, _D, _D, C.c_int, _D]


def _p(a: np.ndarray):
    if a.dtype == np.float64:
        return a.ctypes.data_as(_D)
    if a.dtype == np.uint8:
        return a.ctypes.data_as(_U8)
    raise TypeError(a.dtype)


# ----------------------------------------------------------------------------
# geometry
# ----------------------------------------------------------------------------

def build_mask(nx: int, ny: int, geom_cmds) -> tuple[np.ndarray, int]:
    """Apply geometry commands like the reference Geometry; returns (mask, err)."""
    L = lib()
    g = np.ones(nx * ny, dtype=np.uint8)
    for cmd in geom_cmds:
        k = cmd[0]
        if k == "walls":
            rc = L.orc_geom_add_walls(_p(g), nx, ny, cmd[1], cmd[2].encode())
        elif k == "rectangle":
            rc = L.orc_geom_add_rectangle(_p(g), nx, ny, *cmd[1:5])
        elif k == "square":
            rc = L.orc_geom_add_square(_p(g), nx, ny, *cmd[1:4])
        elif k == "ellipse":
            rc = L.orc_geom_add_ellipse(_p(g), nx, ny, *cmd[1:5])
        elif k == "circle":
            rc = L.orc_geom_add_circle(_p(g), nx, ny, *cmd[1:4])
        elif k in ("array_n", "array_d"):
            _, typ, props, bounds, a, b = cmd
            P = (_SZ * len(props))(*props)
            B = (_SZ * 4)(*bounds)
            rc = L.orc_geom_add_array(_p(g), nx, ny, typ.encode(), P, len(props), B, a, b,
                                      1 if k == "array_n" else 0)
        elif k == "fluid_node":
            g[cmd[2] * nx + cmd[1]] = 1
            rc = 0
        elif k == "solid_node":
            g[cmd[2] * nx + cmd[1]] = 0
            rc = 0
        else:
            raise ValueError(k)
        if rc:
            return g, rc
    return g, 0


# ----------------------------------------------------------------------------
# oracle runs of a case
# ----------------------------------------------------------------------------

def _init_two(case, g):
    nx, ny = case["nx"], case["ny"]
    N = nx * ny
    L = lib()
    f1 = np.zeros(9 * N)
    f2 = np.zeros(9 * N)
    kind, *args = case["init"]
    if kind == "droplet":
        L.orc_init_droplet(nx, ny, _p(g), _p(f1), _p(f2), *map(float, args[:7]))
    elif kind == "rectangle":
        rc = L.orc_init_rectangle(nx, ny, _p(g), _p(f1), _p(f2), *map(float, args[:8]))
        if rc:
            raise IndexError("initialize_fluid_rectangle out of range")
    elif kind == "file":
        f = np.asarray(args[0], dtype=np.float64).ravel()
        f1[:] = f[:9 * N]
        f2[:] = f[9 * N:]
    else:
        raise ValueError(kind)
    return f1, f2


def _new_comp(N, f, tau, G, gs, ssx, ssy):
    L = lib()
    arr = dict(f=f, feq=np.zeros(9 * N), rho=np.zeros(N), ux=np.zeros(N), uy=np.zeros(N),
               uex=np.zeros(N), uey=np.zeros(N), frx=np.zeros(N), fry=np.zeros(N),
               fsx=np.zeros(N), fsy=np.zeros(N))
    L.orc_surface_force(N, float(gs), _p(ssx), _p(ssy), _p(arr["fsx"]), _p(arr["fsy"]))
    c = _Comp(*[_p(arr[n]) for n in ("f", "feq", "rho", "ux", "uy", "uex", "uey", "frx", "fry",
                                      "fsx", "fsy")], 1.0 / float(tau), float(G))
    return arr, c


def run_case(case) -> dict:
    """Run a case through the oracle; returns arrays named like the reference runner."""
    L = lib()
    nx, ny = case["nx"], case["ny"]
    N = nx * ny
    g, err = build_mask(nx, ny, case.get("geom", []))
    out = {"mask": g.astype(np.int32), "error": np.array([err], dtype=np.int32)}
    mode = case.get("mode", "mask")
    if mode == "mask" or err:
        return out
    fmode, fvec = case.get("force", (0, [0.0] * 9))
    force = np.asarray(fvec, dtype=np.float64)
    tmp = np.zeros(9 * N)
    if mode in ("single", "ops1"):
        tau = case.get("fluid1", (1.0, 0, 0))[0]
        omega = 1.0 / float(tau)
        kind, *args = case["init"]
        f = np.zeros(9 * N)
        if kind == "simple":
            L.orc_simple_ini(N, _p(g), _p(f), float(args[0]))
        else:
            f[:] = np.asarray(args[0], dtype=np.float64).ravel()
        feq, rho, ux, uy = np.zeros(9 * N), np.zeros(N), np.zeros(N), np.zeros(N)
        if mode == "ops1":
            L.orc_feq_single(N, _p(g), _p(f), _p(rho), _p(ux), _p(uy), _p(feq))
            L.orc_collide(N, omega, _p(f), _p(feq))
            out.update(collide_f=f.copy(), collide_feq=feq.copy(), collide_rho=rho.copy(),
                       collide_ux=ux.copy(), collide_uy=uy.copy())
            L.orc_volume_force(N, _p(g), _p(f), _p(force))
            out["force_f"] = f.copy()
            L.orc_stream(nx, ny, _p(g), _p(f), _p(tmp))
            out["stream_f"] = f.copy()
            return out
        L.orc_run_single(nx, ny, _p(g), omega, _p(f), _p(feq), _p(rho), _p(ux), _p(uy),
                         _p(force) if fmode else None, int(case.get("steps", 0)), _p(tmp))
        out.update(c1_f=f, c1_feq=feq, c1_rho=rho, c1_ux=ux, c1_uy=uy)
        r2, u2x, u2y = np.zeros(N), np.zeros(N), np.zeros(N)
        L.orc_compute_density(N, _p(f), _p(r2))
        L.orc_compute_velocities(N, _p(g), _p(f), _p(r2), _p(u2x), _p(u2y))
        out.update(c1_rho_final=r2, c1_ux_final=u2x, c1_uy_final=u2y)
        return out

    f1, f2 = _init_two(case, g)
    ssx, ssy = np.zeros(N), np.zeros(N)
    L.orc_solid_sum(nx, ny, _p(g), _p(ssx), _p(ssy))
    t1, G1, gs1 = case.get("fluid1", (1.0, 0.0, 0.0))
    t2, G2, gs2 = case.get("fluid2", (1.0, 0.0, 0.0))
    a1, c1 = _new_comp(N, f1, t1, G1, gs1, ssx, ssy)
    a2, c2 = _new_comp(N, f2, t2, G2, gs2, ssx, ssy)
    if mode == "ops2":
        L.orc_compute_density(N, _p(f1), _p(a1["rho"]))
        L.orc_compute_density(N, _p(f2), _p(a2["rho"]))
        out.update(density_c1_rho=a1["rho"].copy(), density_c2_rho=a2["rho"].copy())
        L.orc_repulsive(nx, ny, _p(g), _p(a1["rho"]), _p(a2["rho"]), float(G1), float(G2),
                        _p(a1["frx"]), _p(a1["fry"]), _p(a2["frx"]), _p(a2["fry"]))
        out.update(rep_c1_frx=a1["frx"].copy(), rep_c1_fry=a1["fry"].copy(),
                   rep_c2_frx=a2["frx"].copy(), rep_c2_fry=a2["fry"].copy())
        L.orc_eqvel(nx, ny, _p(g), c1.omega, c2.omega, _p(f1), _p(f2), _p(a1["rho"]),
                    _p(a2["rho"]), *[_p(a[k]) for a in (a1, a2) for k in ("frx", "fry")],
                    *[_p(a[k]) for a in (a1, a2) for k in ("fsx", "fsy")],
                    *[_p(a[k]) for a in (a1, a2) for k in ("ux", "uy")],
                    *[_p(a[k]) for a in (a1, a2) for k in ("uex", "uey")])
        for c, a in (("c1", a1), ("c2", a2)):
            for k in ("ux", "uy", "uex", "uey"):
                out[f"eqv_{c}_{k}"] = a[k].copy()
        for a, c in ((a1, c1), (a2, c2)):
            L.orc_feq_multi(N, _p(a["rho"]), _p(a["uex"]), _p(a["uey"]), _p(a["feq"]))
            L.orc_collide(N, c.omega, _p(a["f"]), _p(a["feq"]))
        out.update(collide_c1_f=f1.copy(), collide_c2_f=f2.copy(),
                   collide_c1_feq=a1["feq"].copy(), collide_c2_feq=a2["feq"].copy())
        L.orc_volume_force(N, _p(g), _p(f1), _p(force))
        L.orc_volume_force(N, _p(g), _p(f2), _p(force))
        out.update(force_c1_f=f1.copy(), force_c2_f=f2.copy())
        L.orc_stream(nx, ny, _p(g), _p(f1), _p(tmp))
        L.orc_stream(nx, ny, _p(g), _p(f2), _p(tmp))
        out.update(stream_c1_f=f1.copy(), stream_c2_f=f2.copy())
        return out
    L.orc_run_two(nx, ny, _p(g), C.byref(c1), C.byref(c2), _p(force) if fmode else None,
                  int(fmode), int(case.get("steps", 0)), _p(tmp))
    for c, a in (("c1", a1), ("c2", a2)):
        for k in ("f", "feq", "rho", "ux", "uy", "uex", "uey", "frx", "fry", "fsx", "fsy"):
            out[f"{c}_{k}"] = a[k]
        r, ux, uy = np.zeros(N), np.zeros(N), np.zeros(N)
        L.orc_compute_density(N, _p(a["f"]), _p(r))
        L.orc_compute_velocities(N, _p(g), _p(a["f"]), _p(r), _p(ux), _p(uy))
        out.update({f"{c}_rho_final": r, f"{c}_ux_final": ux, f"{c}_uy_final": uy})
    return out


# ----------------------------------------------------------------------------
# reference runner (oracle/_ref) -- only where the reference was compiled here
# ----------------------------------------------------------------------------

def _spec_text(case, init_path, out_path) -> str:
    L = [f"size {case['nx']} {case['ny']}", f"mode {case.get('mode', 'mask')}", f"out {out_path}"]
    for cmd in case.get("geom", []):
        k = cmd[0]
        if k in ("array_n", "array_d"):
            _, typ, props, bounds, a, b = cmd
            L.append(f"{k} {typ} {len(props)} " + " ".join(map(str, props)) + " "
                     + " ".join(map(str, bounds)) + f" {a} {b}")
        else:
            L.append(" ".join(map(str, cmd)))
    for i in (1, 2):
        if f"fluid{i}" in case:
            L.append(f"fluid{i} " + " ".join(repr(float(v)) for v in case[f"fluid{i}"]))
    if "init" in case:
        kind, *args = case["init"]
        if kind == "file":
            L.append(f"init file {init_path}")
        else:
            L.append(f"init {kind} " + " ".join(repr(float(v)) for v in args))
    fmode, fvec = case.get("force", (0, [0.0] * 9))
    L.append(f"force {int(fmode)} " + " ".join(repr(float(v)) for v in fvec))
    L.append(f"steps {int(case.get('steps', 0))}")
    return "\n".join(L) + "\n"


def read_ref_output(path: str) -> dict:
    out = {}
    with open(path, "rb") as fh:
        data = fh.read()
    assert data[:8] == b"SCLBMREF", "bad reference output"
    off = 8
    while off < len(data):
        name = data[off:off + 48].split(b"\0", 1)[0].decode()
        dt, n = struct.unpack_from("<iq", data, off + 48)
        off += 60
        if dt == 0:
            out[name] = np.frombuffer(data, dtype="<f8", count=n, offset=off).copy()
            off += 8 * n
        else:
            out[name] = np.frombuffer(data, dtype="<i4", count=n, offset=off).copy()
            off += 4 * n
    return out


def run_ref(case, runner: str | None = None, core=None, timing: bool = False) -> dict:
    """Run a case through the compiled reference (oracle/_ref), or through
    ``runner``: the same driver source (ref_runner.cpp) built against another
    implementation of the reference's Geometry / Fluid / LBM classes.  `core`
    pins the run to one CPU; with `timing`, ``loop_seconds`` (the main loop's
    time) is returned with the arrays."""
    if runner is None:
        if not have_ref():
            raise FileNotFoundError("oracle/_ref/sclbm_ref_runner was not built")
        runner = REF_RUNNER
    with tempfile.TemporaryDirectory() as td:
        init_path = os.path.join(td, "init.bin")
        out_path = os.path.join(td, "out.bin")
        spec = os.path.join(td, "case.txt")
        if case.get("init", ("",))[0] == "file":
            np.asarray(case["init"][1], dtype="<f8").tofile(init_path)
        with open(spec, "w") as fh:
            fh.write(_spec_text(case, init_path, out_path))
        cmd, pre = _pinned([runner, "case", spec], core)
        subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL, preexec_fn=pre)
        res = read_ref_output(out_path)
        if not timing:
            res.pop("loop_seconds", None)
        return res


def ref_bench_parallel(nx: int, ny: int, steps: int, instances: int) -> dict:
    """`instances` independent serial reference runs at once, one per core
    (the reference code itself is single-threaded): aggregate lattice updates
    per second over the wall time from the first start to the last finish."""
    import json
    import time
    t0 = time.perf_counter()
    procs = [subprocess.Popen([REF_RUNNER, "bench", str(nx), str(ny), str(steps), str(1 + k)],
                              stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
             for k in range(instances)]
    outs = [p.communicate()[0] for p in procs]
    wall = time.perf_counter() - t0
    if any(p.returncode for p in procs):
        raise RuntimeError("reference bench run failed")
    runs = [json.loads(o.strip().splitlines()[-1]) for o in outs]
    return {"instances": instances, "wall_seconds": wall,
            "mlups": instances * nx * ny * steps / wall / 1e6,
            "per_instance_mlups": [r["mlups"] for r in runs]}


def cpu_info() -> dict:
    """The host's CPU model string, its logical CPU count and the CPUs this
    process may run on (the first of them is the one serial runs pin to)."""
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as fh:
            for ln in fh:
                if ln.startswith("model name"):
                    model = ln.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    usable = sorted(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else \
        list(range(os.cpu_count() or 1))
    return {"model": model, "nproc": os.cpu_count(), "usable": len(usable), "pin_core": usable[-1]}


def _pinned(cmd, core):
    """`cmd` pinned to one core: taskset -c <core> when present, else the
    scheduler affinity set in the child before exec."""
    import shutil
    if core is None:
        return cmd, None
    if shutil.which("taskset"):
        return ["taskset", "-c", str(core)] + cmd, None
    return cmd, (lambda: os.sched_setaffinity(0, {core}))


def ref_bench(nx: int, ny: int, steps: int, seed: int = 1, core=None, max_seconds: float = 0.0,
              min_steps: int = 1) -> dict:
    """Time the reference's serial two-component step on one core (`core`
    pins it).  With max_seconds > 0 the run stops once that much time has
    passed and at least min_steps steps are done; `step_seconds` lists the
    steps that ran."""
    import json
    cmd, pre = _pinned([REF_RUNNER, "bench", str(nx), str(ny), str(steps), str(seed),
                        repr(float(max_seconds)), str(int(min_steps))], core)
    r = subprocess.run(cmd, check=True, capture_output=True, text=True, preexec_fn=pre)
    out = json.loads(r.stdout.strip().splitlines()[-1])
    out["pinned_core"] = core
    return out
