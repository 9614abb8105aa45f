"""Python mirror of the reference's Geometry / Fluid / LBM classes over the
C ABI of libsclbm_b200.so (include/sclbm.h).

Method names, argument order and error behaviour follow the reference
(include/geometry.h, include/fluid.h, include/lbm.h); arrays are numpy float64
in the reference layout.  ``Domain`` is the production path: one device
domain in FP64 or a shifted FP32/FP16 storage form, advanced by the fused
kernel.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi
from .capi import call, lib

_D = C.POINTER(C.c_double)


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


class _Handle:
    _destroy = ""

    def __init__(self):
        self._h = C.c_void_p()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and h.value and capi._lib is not None:
            getattr(capi._lib, self._destroy)(h)
            self._h = C.c_void_p()

    @property
    def handle(self):
        return self._h


class Geometry(_Handle):
    """Geometry(Nx, Ny): all-fluid mask (include/geometry.h:58-59)."""
    _destroy = "sclbm_geometry_destroy"

    def __init__(self, nx: int, ny: int):
        super().__init__()
        call("sclbm_geometry_create", nx, ny, C.byref(self._h))

    def Nx(self) -> int:
        a, b = C.c_size_t(), C.c_size_t()
        call("sclbm_geometry_dims", self._h, C.byref(a), C.byref(b))
        return a.value

    def Ny(self) -> int:
        a, b = C.c_size_t(), C.c_size_t()
        call("sclbm_geometry_dims", self._h, C.byref(a), C.byref(b))
        return b.value

    def add_walls(self, dH: int = 1, where: str = "y"):
        call("sclbm_geometry_add_walls", self._h, dH, where.encode())

    def add_rectangle(self, Lx, Ly, xc, yc):
        call("sclbm_geometry_add_rectangle", self._h, Lx, Ly, xc, yc)

    def add_square(self, Ls, xc, yc):
        call("sclbm_geometry_add_square", self._h, Ls, xc, yc)

    def add_ellipse(self, Lx, Ly, xc, yc):
        call("sclbm_geometry_add_ellipse", self._h, Lx, Ly, xc, yc)

    def add_circle(self, D, xc, yc):
        call("sclbm_geometry_add_circle", self._h, D, xc, yc)

    def add_array(self, props, bounds, a, b=None, object_type="ellipse"):
        """add_array(props, [[x0,x1],[y0,y1]], [nx,ny], type) or
        add_array(props, bounds, dx, dy, type) like the two reference overloads."""
        P = (C.c_size_t * len(props))(*props)
        B = (C.c_size_t * 4)(bounds[0][0], bounds[0][1], bounds[1][0], bounds[1][1])
        if isinstance(a, (list, tuple)):
            if b is not None:
                object_type = b
            call("sclbm_geometry_add_array_numbers", self._h, P, len(props), B, a[0], a[1],
                 object_type.encode())
        else:
            call("sclbm_geometry_add_array_spacing", self._h, P, len(props), B, a, b,
                 object_type.encode())

    def add_random_disks(self, porosity, rmin, rmax, seed, wall_rows=0, max_tries=20000,
                         max_misses=300) -> int:
        """Seeded non-overlapping disks to the given fluid fraction (native)."""
        n = C.c_size_t()
        call("sclbm_geometry_add_random_disks", self._h, float(porosity), int(rmin), int(rmax),
             int(seed), int(wall_rows), int(max_tries), int(max_misses), C.byref(n))
        return n.value

    def set_node_fluid(self, x, y):
        call("sclbm_geometry_set_node", self._h, x, y, 1)

    def set_node_solid(self, x, y):
        call("sclbm_geometry_set_node", self._h, x, y, 0)

    def get_geom(self) -> np.ndarray:
        n = self.Nx() * self.Ny()
        out = np.zeros(n, dtype=np.int32)
        call("sclbm_geometry_get_mask", self._h, out.ctypes.data_as(C.POINTER(C.c_int32)), n)
        return out

    def set_geom(self, nx, ny, mask):
        m = np.ascontiguousarray(mask, dtype=np.int32).ravel()
        call("sclbm_geometry_set_mask", self._h, nx, ny, m.ctypes.data_as(C.POINTER(C.c_int32)))

    @classmethod
    def from_mask(cls, nx, ny, mask) -> "Geometry":
        g = cls(nx, ny)
        g.set_geom(nx, ny, mask)
        return g


class Fluid(_Handle):
    """Fluid(name, cs2, tau) + zero_density_ini(geom) (include/fluid.h:60-70)."""
    _destroy = "sclbm_fluid_destroy"

    def __init__(self, geom: Geometry, tau: float = 1.0):
        super().__init__()
        self.nx, self.ny = geom.Nx(), geom.Ny()
        self.N = self.nx * self.ny
        call("sclbm_fluid_create", self.nx, self.ny, float(tau), C.byref(self._h))

    def initialize_interactions(self, Gs: float, Gf: float):
        call("sclbm_fluid_set_interactions", self._h, float(Gs), float(Gf))

    def _size(self, name):
        return 9 * self.N if name in ("f", "feq") else self.N

    def get(self, name: str) -> np.ndarray:
        out = np.empty(self._size(name))
        call("sclbm_fluid_read", self._h, capi.FIELDS[name], _dp(out), out.size)
        return out

    def set(self, name: str, values) -> None:
        v = np.ascontiguousarray(values, dtype=np.float64).ravel()
        call("sclbm_fluid_write", self._h, capi.FIELDS[name], _dp(v), v.size)

    def compute_density(self):
        call("sclbm_fluid_compute_density", self._h)

    def compute_velocities(self, geom):
        call("sclbm_fluid_compute_velocities", self._h, geom.handle)

    def compute_f_equilibrium(self, geom=None):
        if geom is None:
            call("sclbm_fluid_compute_f_equilibrium", self._h)
        else:
            call("sclbm_fluid_compute_f_equilibrium_geom", self._h, geom.handle)

    def simple_ini(self, geom, rho0):
        call("sclbm_fluid_simple_ini", self._h, geom.handle, float(rho0))


class LBM(_Handle):
    """LBM(geom): the step operators (include/lbm.h:23-135)."""
    _destroy = "sclbm_lbm_destroy"

    def __init__(self, geom: Geometry):
        super().__init__()
        call("sclbm_lbm_create", geom.handle, C.byref(self._h))

    def initialize_droplet(self, geom, bulk, droplet, *args):
        call("sclbm_lbm_initialize_droplet", self._h, geom.handle, bulk.handle, droplet.handle,
             *map(float, args))

    def initialize_fluid_rectangle(self, geom, bulk, droplet, *args):
        call("sclbm_lbm_initialize_fluid_rectangle", self._h, geom.handle, bulk.handle,
             droplet.handle, *map(float, args))

    def solid_surface_sums(self, geom):
        n = geom.Nx() * geom.Ny()
        sx, sy = np.empty(n), np.empty(n)
        call("sclbm_lbm_solid_surface_sums", self._h, geom.handle, _dp(sx), _dp(sy), n)
        return sx, sy

    def compute_solid_surface_force(self, geom, f1, f2, gs1, gs2):
        """LBM::compute_solid_surface_force + Fluid::add_surface_forces (first call)."""
        sx, sy = self.solid_surface_sums(geom)
        for fl, gs in ((f1, gs1), (f2, gs2)):
            fl.set("fsx", (-1.0 * gs) * sx)
            fl.set("fsy", (-1.0 * gs) * sy)

    def compute_fluid_repulsive_interactions(self, geom, f1, f2):
        call("sclbm_lbm_fluid_repulsive_interactions", self._h, geom.handle, f1.handle, f2.handle)

    def compute_equilibrium_velocities(self, geom, f1, f2):
        call("sclbm_lbm_equilibrium_velocities", self._h, geom.handle, f1.handle, f2.handle)

    def collide(self, a, b):
        """collide(geom, fluid) or collide(fluid1, fluid2), like the overloads."""
        if isinstance(a, Geometry):
            call("sclbm_lbm_collide_single", self._h, a.handle, b.handle)
        else:
            call("sclbm_lbm_collide", self._h, a.handle, b.handle)

    def add_volume_force(self, geom, f1, f2_or_force, force=None):
        if force is None:
            F = np.ascontiguousarray(f2_or_force, dtype=np.float64)
            call("sclbm_lbm_add_volume_force_single", self._h, geom.handle, f1.handle, _dp(F),
                 F.size)
        else:
            F = np.ascontiguousarray(force, dtype=np.float64)
            call("sclbm_lbm_add_volume_force", self._h, geom.handle, f1.handle,
                 f2_or_force.handle, _dp(F), F.size)

    def stream(self, geom, f1, f2=None):
        if f2 is None:
            call("sclbm_lbm_stream_single", self._h, geom.handle, f1.handle)
        else:
            call("sclbm_lbm_stream", self._h, geom.handle, f1.handle, f2.handle)

    def step(self, geom, f1, f2, nsteps, force1=None, force2=None):
        F1 = None if force1 is None else np.ascontiguousarray(force1, dtype=np.float64)
        F2 = None if force2 is None else np.ascontiguousarray(force2, dtype=np.float64)
        call("sclbm_lbm_step", self._h, geom.handle, f1.handle, f2.handle,
             None if F1 is None else _dp(F1), None if F2 is None else _dp(F2), int(nsteps))

    def step_single(self, geom, f, nsteps, force=None):
        F = None if force is None else np.ascontiguousarray(force, dtype=np.float64)
        call("sclbm_lbm_step_single", self._h, geom.handle, f.handle,
             None if F is None else _dp(F), int(nsteps))


def make_params(ncomp=2, tau=(1.0, 1.0), g_fluid=(0.0, 0.0), g_solid=(0.0, 0.0),
                rho_ref=(1.0, 1.0), force=(None, None)) -> capi.Params:
    p = capi.Params()
    p.ncomp = ncomp
    for k in range(2):
        p.tau[k] = float(tau[k])
        p.g_fluid[k] = float(g_fluid[k])
        p.g_solid[k] = float(g_solid[k])
        p.rho_ref[k] = float(rho_ref[k])
        p.force_on[k] = 0 if force[k] is None else 1
        for i in range(9):
            p.force[k][i] = 0.0 if force[k] is None else float(force[k][i])
    return p


class Domain(_Handle):
    """Device domain advanced by the fused kernel (FP64 / FP32 / FP16 storage)."""
    _destroy = "sclbm_domain_destroy"

    def __init__(self, nx, ny, mask, params: capi.Params, precision: int = capi.FP64):
        super().__init__()
        self.nx, self.ny, self.N = nx, ny, nx * ny
        self.ncomp = params.ncomp
        m = np.ascontiguousarray(mask, dtype=np.int32).ravel()
        call("sclbm_domain_create", nx, ny, m.ctypes.data_as(C.POINTER(C.c_int32)),
             C.byref(params), int(precision), C.byref(self._h))

    def upload_f(self, comp, f):
        v = np.ascontiguousarray(f, dtype=np.float64).ravel()
        call("sclbm_domain_upload_f", self._h, comp, _dp(v), v.size)

    def add_random_disks(self, porosity, rmin, rmax, seed, wall_rows=0, max_tries=20000,
                         max_misses=300) -> int:
        """Seeded non-overlapping disks to the given fluid fraction, placed and
        rasterised on the device; the same disks as Geometry.add_random_disks
        with the same arguments on the same mask.  Returns the disks placed."""
        n = C.c_size_t()
        call("sclbm_domain_add_random_disks", self._h, float(porosity), int(rmin), int(rmax),
             int(seed), int(wall_rows), int(max_tries), int(max_misses), C.byref(n))
        return n.value

    def download_mask(self) -> np.ndarray:
        """The device mask (int32, 1 fluid, 0 solid)."""
        m = np.zeros(self.N, np.int32)
        call("sclbm_domain_download_mask", self._h, m.ctypes.data_as(C.POINTER(C.c_int32)), self.N)
        return m

    def init_noise(self, comp, rho0, amp, seed):
        """f_i = rho/9, rho = rho0*(1 + amp*(2u-1)), u = splitmix64(seed, node),
        written on the device (equal to uploading workloads.populations)."""
        call("sclbm_domain_init_noise", self._h, int(comp), float(rho0), float(amp), int(seed))

    def download_f(self, comp) -> np.ndarray:
        out = np.empty(9 * self.N)
        call("sclbm_domain_download_f", self._h, comp, _dp(out), out.size)
        return out

    def download_rho(self, comp) -> np.ndarray:
        out = np.empty(self.N)
        call("sclbm_domain_download_rho", self._h, comp, _dp(out), out.size)
        return out

    def download_velocity(self, comp):
        ux, uy = np.empty(self.N), np.empty(self.N)
        call("sclbm_domain_download_velocity", self._h, comp, _dp(ux), _dp(uy), self.N)
        return ux, uy

    def step(self, n=1):
        call("sclbm_domain_step", self._h, int(n))

    def mass_momentum(self) -> np.ndarray:
        out = np.zeros(7)
        call("sclbm_domain_mass_momentum", self._h, _dp(out))
        return out

    def set_kernel(self, variant=0, tile_y=0):
        call("sclbm_domain_set_kernel", self._h, int(variant), int(tile_y))

    # halo rows of a slab domain (sc_lbm_b200/slabs.py); ptr = device address
    def halo_bytes(self, rows) -> int:
        return int(lib().sclbm_domain_halo_bytes(self._h, int(rows)))

    def halo_pack(self, rows, side, ptr):
        call("sclbm_domain_halo_pack", self._h, int(rows), int(side), C.c_void_p(int(ptr)))

    def halo_unpack(self, rows, side, ptr):
        call("sclbm_domain_halo_unpack", self._h, int(rows), int(side), C.c_void_p(int(ptr)))

    # per-step exchange with one ghost row per side (slab.cu)
    def halo_min_bytes(self) -> int:
        return int(lib().sclbm_domain_halo_min_bytes(self._h))

    def halo_min_pack(self, side, ptr):
        call("sclbm_domain_halo_min_pack", self._h, int(side), C.c_void_p(int(ptr)))

    def halo_min_unpack(self, side, ptr):
        call("sclbm_domain_halo_min_unpack", self._h, int(side), C.c_void_p(int(ptr)))

    def step_rows(self, row0, nrows, finish=False):
        """One step of rows [row0, row0 + nrows); finish ends the step."""
        call("sclbm_domain_step_rows", self._h, int(row0), int(nrows), 1 if finish else 0)

    def set_threads(self, tx):
        call("sclbm_domain_set_threads", self._h, int(tx))

    def device_bytes(self) -> int:
        return int(lib().sclbm_domain_device_bytes(self._h))

    # reference-format text output (density 0, ux 1, uy 2, populations 3)
    def write_text(self, comp, what, path, asynchronous=False):
        call("sclbm_domain_write_text", self._h, int(comp), int(what), str(path).encode(),
             1 if asynchronous else 0)

    def write_density(self, comp, path, asynchronous=False):
        self.write_text(comp, 0, path, asynchronous)

    def save_state(self, comp, frho, fux, fuy, step, asynchronous=False):
        """Fluid::save_state: <frho>_<step>.txt, <fux>_<step>.txt, <fuy>_<step>.txt"""
        for what, name in ((0, frho), (1, fux), (2, fuy)):
            self.write_text(comp, what, f"{name}_{int(step)}.txt", asynchronous)

    def write_f(self, comp, prefix, asynchronous=False):
        self.write_text(comp, 3, prefix, asynchronous)

    def restart_from_file(self, comp, prefix):
        call("sclbm_domain_read_text_f", self._h, int(comp), str(prefix).encode())

    def checkpoint_save(self, path):
        call("sclbm_domain_checkpoint_save", self._h, str(path).encode())

    def checkpoint_load(self, path):
        call("sclbm_domain_checkpoint_load", self._h, str(path).encode())

    # measurements on the device (the reference's post-processing scripts)
    def laplace_measure(self, bulk, G, rho_bulk, rho_disp, p_in, p_out) -> dict:
        out = np.zeros(5)
        call("sclbm_domain_laplace_measure", self._h, int(bulk), float(G), float(rho_bulk),
             float(rho_disp), int(p_in[0]), int(p_in[1]), int(p_out[0]), int(p_out[1]), _dp(out))
        return {"dp": out[0], "R": out[1], "R_rows": out[2], "R_cols": out[3],
                "band_nodes": int(out[4])}

    def velocity_stats(self, comp) -> dict:
        out = np.zeros(3)
        call("sclbm_domain_velocity_stats", self._h, int(comp), _dp(out))
        return {"max_u": out[0], "mean_nonzero_u": out[1], "nonzero": int(out[2])}

    def profile(self, comp, axis=0) -> np.ndarray:
        out = np.zeros(self.ny)
        call("sclbm_domain_profile", self._h, int(comp), int(axis), _dp(out), self.ny)
        return out

    def contact_angle(self, bulk, rho_bulk=2.0, rho_disp=0.06) -> dict:
        """Contact angle of the droplet (the other component) on a flat solid,
        measured as compute_contact_angles.py does (degrees)."""
        out = np.zeros(9)
        call("sclbm_domain_contact_angle", self._h, int(bulk), float(rho_bulk), float(rho_disp),
             _dp(out))
        return {"theta": out[0], "L": out[1], "H": out[2], "R": out[3], "xL": out[4],
                "xR": out[5], "y_min": int(out[6]), "y_max": int(out[7]),
                "band_nodes": int(out[8])}

    def run(self, f1, f2, nsteps, rho1, rho2=None):
        call("sclbm_domain_run", self._h, _dp(f1), None if f2 is None else _dp(f2), int(nsteps),
             _dp(rho1), None if rho2 is None else _dp(rho2))


class Batch(_Handle):
    """Many domains advanced together by one launch per step (CUDA graph)."""
    _destroy = "sclbm_batch_destroy"

    def __init__(self, domains, tile_y=None):
        super().__init__()
        self.domains = list(domains)
        arr = (C.c_void_p * len(self.domains))(*[d.handle.value for d in self.domains])
        ty = None if tile_y is None else (C.c_int * len(self.domains))(*tile_y)
        call("sclbm_batch_create", arr, len(self.domains), ty, C.byref(self._h))

    def step(self, n=1, use_graph=True):
        call("sclbm_batch_step", self._h, int(n), 1 if use_graph else 0)

    def set_kernel(self, variant):
        call("sclbm_batch_set_kernel", self._h, int(variant))

    def info(self):
        a, b = C.c_int(), C.c_int()
        call("sclbm_batch_info", self._h, C.byref(a), C.byref(b))
        return a.value, b.value


def tuned_config(nx: int, ny: int, precision: int | None = None) -> dict:
    """Tuned batch launch shape for an nx x ny domain (host lookup in the
    autotuned table): {"tile_y", "variant", "recommended_precision"}."""
    t, v, r = C.c_int(), C.c_int(), C.c_int()
    call("sclbm_tuned_config", int(nx), int(ny), -1 if precision is None else int(precision),
         C.byref(t), C.byref(v), C.byref(r))
    return {"tile_y": t.value, "variant": v.value, "recommended_precision": r.value}


def io_wait():
    """Join the asynchronous text writers; raises the first failure."""
    call("sclbm_io_wait")


def write_rows(path, values, nx, ny):
    v = np.ascontiguousarray(values, dtype=np.float64).ravel()
    if v.size != nx * ny:
        raise ValueError("values must hold nx*ny entries")
    call("sclbm_write_rows", str(path).encode(), _dp(v), int(nx), int(ny))


def read_rows(path, nx, ny) -> np.ndarray:
    out = np.empty(nx * ny)
    call("sclbm_read_rows", str(path).encode(), _dp(out), int(nx), int(ny))
    return out


def synchronize():
    call("sclbm_synchronize")


def set_stream(ptr):
    call("sclbm_set_stream", C.c_void_p(ptr) if ptr else None)


def version() -> str:
    return lib().sclbm_version().decode()
