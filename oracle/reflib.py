"""ctypes bindings of the reference's own PBF step, compiled from its sources
by oracle/ref_build/Makefile into oracle/_ref/libpbf_ref*.so.

TEST INFRASTRUCTURE ONLY: the checker the restated oracle and the CUDA path
are pinned against, and the timed CPU baseline / reference arm of bench.py.
This module imports nothing of the product package, so a process that only
drives the reference (bench.py --impl reference) never maps the product's
library.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

ROOT = Path(__file__).resolve().parent
REF_LIB = ROOT / "_ref" / "libpbf_ref.so"
REF_LIB_SERIAL = ROOT / "_ref" / "libpbf_ref_serial.so"
_vp = C.c_void_p


class RefParams(C.Structure):
    """ref_params_t of ref_build/ref_driver.cpp: the fields of the reference's
    Parameters (Common/parameters.h:550-573) that its driver sets before
    derive_from_input (parameters.h:123-148)."""
    _fields_ = [
        ("time_step", C.c_float), ("gravity", C.c_float), ("gamma", C.c_float), ("visc_c", C.c_float),
        ("lambda_epsilon", C.c_float), ("k_stiff", C.c_float), ("vorticity_coef", C.c_float),
        ("smoothing_radius", C.c_float), ("neighbor_bin_spacing", C.c_float), ("rest_spacing", C.c_float),
        ("boundary_min", C.c_float * 3), ("boundary_max", C.c_float * 3),
        ("fluid_min", C.c_float * 3), ("fluid_max", C.c_float * 3), ("mover_center", C.c_float * 3),
        ("solve_steps", C.c_uint64), ("max_particles_local", C.c_uint64), ("global_particle_count", C.c_uint64),
        ("rest_density", C.c_float),
    ]


_ref_libs: dict[str, C.CDLL] = {}


def ref_available(serial: bool = False) -> bool:
    return (REF_LIB_SERIAL if serial else REF_LIB).exists()


def ref_lib(serial: bool = False) -> C.CDLL:
    path = REF_LIB_SERIAL if serial else REF_LIB
    key = str(path)
    if key not in _ref_libs:
        if not path.exists():
            raise RuntimeError(f"{path} missing: it is built from the reference sources by oracle/ref_build/Makefile")
        lib = C.CDLL(key)
        R = C.POINTER(RefParams)
        sig = {
            "ref_last_error": (C.c_char_p, []),
            "ref_set_threads": (None, [C.c_int]),
            "ref_get_threads": (C.c_int, []),
            "ref_derived": (C.c_int, [R, _vp]),
            "ref_derived_from_ini": (C.c_int, [C.c_char_p, _vp, _vp]),
            "ref_create": (_vp, [R]),
            "ref_destroy": (None, [_vp]),
            "ref_set_rest_density": (None, [_vp, C.c_float]),
            "ref_get_param": (C.c_float, [_vp, C.c_int]),
            "ref_construct_fluid": (C.c_int64, [_vp]),
            "ref_construct_fluid_box": (C.c_int64, [_vp, _vp, _vp, _vp]),
            "ref_add": (C.c_int, [_vp, _vp, _vp, C.c_uint64]),
            "ref_count": (C.c_uint64, [_vp]),
            "ref_remove": (C.c_int, [_vp, C.c_uint64]),
            "ref_stage_span": (C.c_int, [_vp, C.c_int, C.c_int, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64]),
            "ref_set_vec": (C.c_int, [_vp, C.c_int, _vp]),
            "ref_get_vec": (C.c_int, [_vp, C.c_int, _vp]),
            "ref_get_scalar": (C.c_int, [_vp, C.c_int, _vp]),
            "ref_set_scalar": (C.c_int, [_vp, C.c_int, _vp]),
            "ref_bin_dims": (None, [_vp, _vp]),
            "ref_bin_id": (C.c_uint64, [_vp, _vp]),
            "ref_get_neighbors": (C.c_int, [_vp, _vp, _vp, C.c_int]),
            "ref_get_bins": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
            "ref_stage": (C.c_int, [_vp, C.c_int, C.c_int]),
            "ref_step": (C.c_int, [_vp, C.c_int]),
            "ref_time_steps": (C.c_double, [_vp, C.c_int]),
        }
        for k, (r, a) in sig.items():
            f = getattr(lib, k)
            f.restype = r
            f.argtypes = a
        _ref_libs[key] = lib
    return _ref_libs[key]


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1
