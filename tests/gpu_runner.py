"""Run a parity case (tests/golden/cases.py format) through libsclbm_b200 on the
GPU, via the C ABI, returning arrays named like the oracle / reference runner.

* ``run_ops``  : the reference driver sequence, one C-ABI call per reference
                 method (per-operator kernels);
* ``run_fused``: the fused FP64 step on fluid objects (sclbm_lbm_step /
                 sclbm_lbm_step_single);
* ``run_domain``: the production domain (FP64 / FP32 / FP16 storage).
"""
from __future__ import annotations

import numpy as np

from oracle import pyoracle


def _geometry(sc, case):
    mask, err = pyoracle.build_mask(case["nx"], case["ny"], case.get("geom", []))
    assert err == 0
    return sc.Geometry.from_mask(case["nx"], case["ny"], mask.astype(np.int32)), mask


def _init_f(case, mask):
    """Initial populations exactly as the reference initialisers produce them."""
    nx, ny = case["nx"], case["ny"]
    N = nx * ny
    kind, *args = case["init"]
    if case["mode"] in ("single", "ops1"):
        if kind == "simple":
            f = np.zeros(9 * N)
            pyoracle.lib().orc_simple_ini(N, pyoracle._p(mask), pyoracle._p(f), float(args[0]))
            return [f]
        return [np.asarray(args[0], dtype=np.float64).ravel().copy()]
    f1, f2 = pyoracle._init_two(case, mask)
    return [f1, f2]


def _force(case):
    fmode, fvec = case.get("force", (0, [0.0] * 9))
    return int(fmode), np.asarray(fvec, dtype=np.float64)


def _final_macros(out, prefix, fl, geom):
    fl.compute_density()
    fl.compute_velocities(geom)
    out[prefix + "rho_final"] = fl.get("rho")
    out[prefix + "ux_final"] = fl.get("ux")
    out[prefix + "uy_final"] = fl.get("uy")


def _two_fluids(sc, case, geom, lbm, init_via_api=True):
    t1, G1, gs1 = case.get("fluid1", (1.0, 0.0, 0.0))
    t2, G2, gs2 = case.get("fluid2", (1.0, 0.0, 0.0))
    a, b = sc.Fluid(geom, t1), sc.Fluid(geom, t2)
    a.initialize_interactions(gs1, G1)
    b.initialize_interactions(gs2, G2)
    kind, *args = case["init"]
    if init_via_api and kind == "droplet":
        lbm.initialize_droplet(geom, a, b, *args[:7])
    elif init_via_api and kind == "rectangle":
        lbm.initialize_fluid_rectangle(geom, a, b, *args[:8])
    else:
        f = np.asarray(args[0], dtype=np.float64).ravel()
        N = case["nx"] * case["ny"]
        a.set("f", f[:9 * N])
        b.set("f", f[9 * N:])
    lbm.compute_solid_surface_force(geom, a, b, gs1, gs2)
    return a, b


def run_ops(sc, case) -> dict:
    geom, mask = _geometry(sc, case)
    out = {"mask": mask.astype(np.int32), "error": np.array([0], np.int32)}
    lbm = sc.LBM(geom)
    fmode, force = _force(case)
    if case["mode"] in ("single", "ops1"):
        fl = sc.Fluid(geom, case.get("fluid1", (1.0,))[0])
        kind, *args = case["init"]
        if kind == "simple":
            fl.simple_ini(geom, args[0])
        else:
            fl.set("f", np.asarray(args[0], dtype=np.float64).ravel())
        if case["mode"] == "ops1":
            lbm.collide(geom, fl)
            for k in ("f", "feq", "rho", "ux", "uy"):
                out["collide_" + k] = fl.get(k)
            lbm.add_volume_force(geom, fl, force)
            out["force_f"] = fl.get("f")
            lbm.stream(geom, fl)
            out["stream_f"] = fl.get("f")
            return out
        for _ in range(int(case.get("steps", 0))):
            lbm.collide(geom, fl)
            if fmode:
                lbm.add_volume_force(geom, fl, force)
            lbm.stream(geom, fl)
        for k in ("f", "feq", "rho", "ux", "uy"):
            out["c1_" + k] = fl.get(k)
        _final_macros(out, "c1_", fl, geom)
        return out
    a, b = _two_fluids(sc, case, geom, lbm)
    if case["mode"] == "ops2":
        a.compute_density()
        b.compute_density()
        out.update(density_c1_rho=a.get("rho"), density_c2_rho=b.get("rho"))
        lbm.compute_fluid_repulsive_interactions(geom, a, b)
        for c, fl in (("c1", a), ("c2", b)):
            out[f"rep_{c}_frx"], out[f"rep_{c}_fry"] = fl.get("frx"), fl.get("fry")
        lbm.compute_equilibrium_velocities(geom, a, b)
        for c, fl in (("c1", a), ("c2", b)):
            for k in ("ux", "uy", "uex", "uey"):
                out[f"eqv_{c}_{k}"] = fl.get(k)
        lbm.collide(a, b)
        for c, fl in (("c1", a), ("c2", b)):
            out[f"collide_{c}_f"], out[f"collide_{c}_feq"] = fl.get("f"), fl.get("feq")
        lbm.add_volume_force(geom, a, b, force)
        out.update(force_c1_f=a.get("f"), force_c2_f=b.get("f"))
        lbm.stream(geom, a, b)
        out.update(stream_c1_f=a.get("f"), stream_c2_f=b.get("f"))
        return out
    for _ in range(int(case.get("steps", 0))):
        a.compute_density()
        b.compute_density()
        lbm.compute_fluid_repulsive_interactions(geom, a, b)
        lbm.compute_equilibrium_velocities(geom, a, b)
        lbm.collide(a, b)
        if fmode == 3:
            lbm.add_volume_force(geom, a, b, force)
        elif fmode == 1:
            lbm.add_volume_force(geom, a, force)
        elif fmode == 2:
            lbm.add_volume_force(geom, b, force)
        lbm.stream(geom, a, b)
    for c, fl in (("c1", a), ("c2", b)):
        for k in ("f", "feq", "rho", "ux", "uy", "uex", "uey", "frx", "fry", "fsx", "fsy"):
            out[f"{c}_{k}"] = fl.get(k)
    for c, fl in (("c1", a), ("c2", b)):
        _final_macros(out, c + "_", fl, geom)
    return out


def run_fused(sc, case) -> dict:
    """Fused FP64 steps; returns the populations and final macroscopic fields."""
    geom, mask = _geometry(sc, case)
    out = {}
    lbm = sc.LBM(geom)
    fmode, force = _force(case)
    steps = int(case.get("steps", 0))
    if case["mode"] == "single":
        fl = sc.Fluid(geom, case.get("fluid1", (1.0,))[0])
        kind, *args = case["init"]
        if kind == "simple":
            fl.simple_ini(geom, args[0])
        else:
            fl.set("f", np.asarray(args[0], dtype=np.float64).ravel())
        lbm.step_single(geom, fl, steps, force if fmode else None)
        out["c1_f"] = fl.get("f")
        _final_macros(out, "c1_", fl, geom)
        return out
    a, b = _two_fluids(sc, case, geom, lbm)
    f1 = force if fmode in (1, 3) else None
    f2 = force if fmode in (2, 3) else None
    lbm.step(geom, a, b, steps, f1, f2)
    for c, fl in (("c1", a), ("c2", b)):
        out[c + "_f"] = fl.get("f")
        _final_macros(out, c + "_", fl, geom)
    return out


def domain_params(sc, case, rho_ref=(1.0, 1.0)):
    fmode, force = _force(case)
    if case["mode"] == "single":
        t1 = case.get("fluid1", (1.0, 0, 0))
        return sc.make_params(ncomp=1, tau=(t1[0], 1.0), rho_ref=rho_ref,
                              force=(force if fmode else None, None))
    t1, G1, gs1 = case.get("fluid1", (1.0, 0.0, 0.0))
    t2, G2, gs2 = case.get("fluid2", (1.0, 0.0, 0.0))
    return sc.make_params(ncomp=2, tau=(t1, t2), g_fluid=(G1, G2), g_solid=(gs1, gs2),
                          rho_ref=rho_ref,
                          force=(force if fmode in (1, 3) else None,
                                 force if fmode in (2, 3) else None))


def make_domain(sc, case, precision, rho_ref=(1.0, 1.0)):
    geom, mask = _geometry(sc, case)
    d = sc.Domain(case["nx"], case["ny"], mask.astype(np.int32),
                  domain_params(sc, case, rho_ref), precision)
    for k, f in enumerate(_init_f(case, mask)):
        d.upload_f(k, f)
    return d


def run_domain(sc, case, precision, rho_ref=(1.0, 1.0), variant=0, tile_y=0, tx=128,
               steps=None) -> dict:
    d = make_domain(sc, case, precision, rho_ref)
    d.set_kernel(variant, tile_y)
    d.set_threads(tx)
    d.step(int(case.get("steps", 0)) if steps is None else steps)
    out = {}
    for k in range(d.ncomp):
        c = f"c{k + 1}_"
        out[c + "f"] = d.download_f(k)
        out[c + "rho_final"] = d.download_rho(k)
        out[c + "ux_final"], out[c + "uy_final"] = d.download_velocity(k)
    out["_domain"] = d
    return out
