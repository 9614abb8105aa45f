"""ctypes binding of libsclbm_b200.so (declarations of include/sclbm.h).

The library is loaded from this package directory; there is no fallback: if
the shared object is missing or no sm_100 device is present the calls raise.
Status codes are mapped to the Python counterparts of the reference's C++
exceptions (invalid_argument -> ValueError, runtime_error -> RuntimeError,
out_of_range -> IndexError).
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsclbm_b200.so")

OK = 0
E_INVALID_ARGUMENT = 1
E_RUNTIME = 2
E_OUT_OF_RANGE = 3
E_DOMAIN = 4
E_CUDA = 5
E_NO_DEVICE = 6
E_NONFINITE = 7
E_ALLOC = 8

FP64, FP32_SHIFTED, FP16_SHIFTED = 0, 1, 2
FIELDS = {"f": 0, "feq": 1, "rho": 2, "ux": 3, "uy": 4, "uex": 5, "uey": 6, "frx": 7, "fry": 8,
          "fsx": 9, "fsy": 10}


class SclbmError(RuntimeError):
    """A failure reported by libsclbm_b200 (CUDA, device, allocation)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[sclbm {code}] {msg}")
        self.code = code


class SclbmNonFinite(SclbmError):
    pass


class SclbmDomainError(ValueError):
    pass


class Params(C.Structure):
    _fields_ = [("ncomp", C.c_int), ("tau", C.c_double * 2), ("g_fluid", C.c_double * 2),
                ("g_solid", C.c_double * 2), ("rho_ref", C.c_double * 2),
                ("force_on", C.c_int * 2), ("force", (C.c_double * 9) * 2)]


_D = C.POINTER(C.c_double)
_I32 = C.POINTER(C.c_int32)
_SZ = C.c_size_t
_VP = C.c_void_p

# name -> (restype, argtypes); every handle is passed as c_void_p
SIGNATURES = {
    "sclbm_last_error": (C.c_int, [C.c_char_p, _SZ]),
    "sclbm_version": (C.c_char_p, []),
    "sclbm_set_stream": (C.c_int, [_VP]),
    "sclbm_get_stream": (_VP, []),
    "sclbm_synchronize": (C.c_int, []),
    "sclbm_geometry_create": (C.c_int, [_SZ, _SZ, C.POINTER(_VP)]),
    "sclbm_geometry_destroy": (None, [_VP]),
    "sclbm_geometry_dims": (C.c_int, [_VP, C.POINTER(_SZ), C.POINTER(_SZ)]),
    "sclbm_geometry_add_walls": (C.c_int, [_VP, _SZ, C.c_char_p]),
    "sclbm_geometry_add_rectangle": (C.c_int, [_VP, _SZ, _SZ, _SZ, _SZ]),
    "sclbm_geometry_add_square": (C.c_int, [_VP, _SZ, _SZ, _SZ]),
    "sclbm_geometry_add_ellipse": (C.c_int, [_VP, _SZ, _SZ, _SZ, _SZ]),
    "sclbm_geometry_add_circle": (C.c_int, [_VP, _SZ, _SZ, _SZ]),
    "sclbm_geometry_add_array_spacing": (C.c_int, [_VP, C.POINTER(_SZ), _SZ, C.POINTER(_SZ), _SZ,
                                                   _SZ, C.c_char_p]),
    "sclbm_geometry_add_array_numbers": (C.c_int, [_VP, C.POINTER(_SZ), _SZ, C.POINTER(_SZ), _SZ,
                                                   _SZ, C.c_char_p]),
    "sclbm_geometry_set_node": (C.c_int, [_VP, _SZ, _SZ, C.c_int]),
    "sclbm_geometry_get_mask": (C.c_int, [_VP, _I32, _SZ]),
    "sclbm_geometry_set_mask": (C.c_int, [_VP, _SZ, _SZ, _I32]),
    "sclbm_fluid_create": (C.c_int, [_SZ, _SZ, C.c_double, C.POINTER(_VP)]),
    "sclbm_fluid_destroy": (None, [_VP]),
    "sclbm_fluid_set_interactions": (C.c_int, [_VP, C.c_double, C.c_double]),
    "sclbm_fluid_get_params": (C.c_int, [_VP, _D, _D, _D]),
    "sclbm_fluid_write": (C.c_int, [_VP, C.c_int, _D, _SZ]),
    "sclbm_fluid_read": (C.c_int, [_VP, C.c_int, _D, _SZ]),
    "sclbm_fluid_compute_density": (C.c_int, [_VP]),
    "sclbm_fluid_compute_velocities": (C.c_int, [_VP, _VP]),
    "sclbm_fluid_compute_f_equilibrium_geom": (C.c_int, [_VP, _VP]),
    "sclbm_fluid_compute_f_equilibrium": (C.c_int, [_VP]),
    "sclbm_fluid_simple_ini": (C.c_int, [_VP, _VP, C.c_double]),
    "sclbm_lbm_create": (C.c_int, [_VP, C.POINTER(_VP)]),
    "sclbm_lbm_destroy": (None, [_VP]),
    "sclbm_lbm_initialize_droplet": (C.c_int, [_VP, _VP, _VP, _VP] + [C.c_double] * 7),
    "sclbm_lbm_initialize_fluid_rectangle": (C.c_int, [_VP, _VP, _VP, _VP] + [C.c_double] * 8),
    "sclbm_lbm_solid_surface_sums": (C.c_int, [_VP, _VP, _D, _D, _SZ]),
    "sclbm_lbm_fluid_repulsive_interactions": (C.c_int, [_VP, _VP, _VP, _VP]),
    "sclbm_lbm_equilibrium_velocities": (C.c_int, [_VP, _VP, _VP, _VP]),
    "sclbm_lbm_collide_single": (C.c_int, [_VP, _VP, _VP]),
    "sclbm_lbm_collide": (C.c_int, [_VP, _VP, _VP]),
    "sclbm_lbm_add_volume_force_single": (C.c_int, [_VP, _VP, _VP, _D, _SZ]),
    "sclbm_lbm_add_volume_force": (C.c_int, [_VP, _VP, _VP, _VP, _D, _SZ]),
    "sclbm_lbm_stream_single": (C.c_int, [_VP, _VP, _VP]),
    "sclbm_lbm_stream": (C.c_int, [_VP, _VP, _VP, _VP]),
    "sclbm_lbm_step": (C.c_int, [_VP, _VP, _VP, _VP, _D, _D, C.c_int]),
    "sclbm_lbm_step_single": (C.c_int, [_VP, _VP, _VP, _D, C.c_int]),
    "sclbm_domain_create": (C.c_int, [_SZ, _SZ, _I32, C.POINTER(Params), C.c_int, C.POINTER(_VP)]),
    "sclbm_domain_destroy": (None, [_VP]),
    "sclbm_domain_upload_f": (C.c_int, [_VP, C.c_int, _D, _SZ]),
    "sclbm_domain_download_f": (C.c_int, [_VP, C.c_int, _D, _SZ]),
    "sclbm_domain_init_noise": (C.c_int, [_VP, C.c_int, C.c_double, C.c_double, C.c_uint64]),
    "sclbm_domain_add_random_disks": (C.c_int, [_VP, C.c_double, C.c_int, C.c_int, C.c_uint64,
                                                C.c_int, C.c_long, C.c_long, C.POINTER(_SZ)]),
    "sclbm_domain_download_mask": (C.c_int, [_VP, C.POINTER(C.c_int32), _SZ]),
    "sclbm_domain_download_rho": (C.c_int, [_VP, C.c_int, _D, _SZ]),
    "sclbm_domain_download_velocity": (C.c_int, [_VP, C.c_int, _D, _D, _SZ]),
    "sclbm_domain_step": (C.c_int, [_VP, C.c_int]),
    "sclbm_domain_mass_momentum": (C.c_int, [_VP, _D]),
    "sclbm_domain_set_kernel": (C.c_int, [_VP, C.c_int, C.c_int]),
    "sclbm_domain_set_threads": (C.c_int, [_VP, C.c_int]),
    "sclbm_domain_device_bytes": (_SZ, [_VP]),
    "sclbm_domain_run": (C.c_int, [_VP, _D, _D, C.c_int, _D, _D]),
    "sclbm_mass_momentum_noalloc": (C.c_int, [_VP, _VP, _VP, _SZ, _SZ, C.c_int, C.c_int, _D, _VP,
                                              _D]),
    "sclbm_batch_create": (C.c_int, [C.POINTER(_VP), C.c_int, C.POINTER(C.c_int), C.POINTER(_VP)]),
    "sclbm_batch_destroy": (None, [_VP]),
    "sclbm_batch_step": (C.c_int, [_VP, C.c_int, C.c_int]),
    "sclbm_batch_set_kernel": (C.c_int, [_VP, C.c_int]),
    "sclbm_batch_info": (C.c_int, [_VP, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "sclbm_domain_write_text": (C.c_int, [_VP, C.c_int, C.c_int, C.c_char_p, C.c_int]),
    "sclbm_io_wait": (C.c_int, []),
    "sclbm_domain_read_text_f": (C.c_int, [_VP, C.c_int, C.c_char_p]),
    "sclbm_write_rows": (C.c_int, [C.c_char_p, _D, _SZ, _SZ]),
    "sclbm_read_rows": (C.c_int, [C.c_char_p, _D, _SZ, _SZ]),
    "sclbm_domain_checkpoint_save": (C.c_int, [_VP, C.c_char_p]),
    "sclbm_domain_checkpoint_load": (C.c_int, [_VP, C.c_char_p]),
    "sclbm_domain_laplace_measure": (C.c_int, [_VP, C.c_int, C.c_double, C.c_double, C.c_double,
                                               _SZ, _SZ, _SZ, _SZ, _D]),
    "sclbm_domain_velocity_stats": (C.c_int, [_VP, C.c_int, _D]),
    "sclbm_domain_profile": (C.c_int, [_VP, C.c_int, C.c_int, _D, _SZ]),
    "sclbm_domain_contact_angle": (C.c_int, [_VP, C.c_int, C.c_double, C.c_double, _D]),
    "sclbm_domain_halo_bytes": (_SZ, [_VP, C.c_int]),
    "sclbm_domain_halo_pack": (C.c_int, [_VP, C.c_int, C.c_int, _VP]),
    "sclbm_domain_halo_unpack": (C.c_int, [_VP, C.c_int, C.c_int, _VP]),
    "sclbm_domain_halo_min_bytes": (_SZ, [_VP]),
    "sclbm_domain_halo_min_pack": (C.c_int, [_VP, C.c_int, _VP]),
    "sclbm_domain_halo_min_unpack": (C.c_int, [_VP, C.c_int, _VP]),
    "sclbm_domain_step_rows": (C.c_int, [_VP, C.c_int, C.c_int, C.c_int]),
    "sclbm_geometry_add_random_disks": (C.c_int, [_VP, C.c_double, C.c_int, C.c_int, C.c_uint64,
                                                  C.c_int, C.c_long, C.c_long,
                                                  C.POINTER(_SZ)]),
    "sclbm_tuned_config": (C.c_int, [_SZ, _SZ, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                     C.POINTER(C.c_int)]),
}

_lib = None


def lib():
    """Load libsclbm_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: build it with `python -m sc_lbm_b200.build` "
                "(or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return list(SIGNATURES)


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    lib().sclbm_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(rc: int) -> None:
    if rc == OK:
        return
    msg = last_error()
    if rc == E_INVALID_ARGUMENT:
        raise ValueError(msg)
    if rc == E_RUNTIME:
        raise RuntimeError(msg)
    if rc == E_OUT_OF_RANGE:
        raise IndexError(msg)
    if rc == E_DOMAIN:
        raise SclbmDomainError(msg)
    if rc == E_NONFINITE:
        raise SclbmNonFinite(rc, msg)
    raise SclbmError(rc, msg)


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args))
