"""ctypes declarations of the C ABI in include/pbf.h (libpbf_b200.so)."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

PKG_ROOT = Path(__file__).resolve().parent.parent
LIB_PATH = PKG_ROOT / "lib" / "libpbf_b200.so"

PBF_OK = 0
PBF_ERR_ARG = -1
PBF_ERR_CUDA = -2
PBF_ERR_CAPACITY = -3
PBF_ERR_SPAN = -4
PBF_ERR_PARAMS = -5
PBF_ERR_STATE = -6
PBF_ERR_DEVICE = -7
PBF_ERR_IO = -8

PBF_FLAG_KEY_RANGE = 1
PBF_FLAG_NONFINITE = 2
PBF_FLAG_WAIT_TIMEOUT = 4

ARRAY_POSITIONS = 0
ARRAY_POSITION_STARS = 1
ARRAY_VELOCITIES = 2
ARRAY_SCRATCH = 3
ARRAY_DENSITIES = 4
ARRAY_LAMBDAS = 5

MLP_FEATURES = 12
MLP_PARAMS = 5057
MLP_NORM = 25

TUNE_FAMILIES = ("density", "delta_p", "viscosity", "vorticity", "apply_vorticity")
# (lanes per particle, threads per block, staged in shared memory)
TUNE_CANDIDATES = ((4, 128, 0), (4, 256, 0), (8, 128, 0), (8, 256, 0), (2, 128, 0), (2, 256, 0), (4, 128, 1))

NOALLOC_MAX_PARTICLES = 65536
NOALLOC_MAX_BINS = 262144
NOALLOC_SCRATCH_BYTES = 5506560

F3 = C.c_float * 3


class PbfParams(C.Structure):
    _fields_ = [
        ("time_step", C.c_float),
        ("gravity", C.c_float),
        ("gamma", C.c_float),
        ("visc_c", C.c_float),
        ("lambda_epsilon", C.c_float),
        ("vorticity_coef", C.c_float),
        ("smoothing_radius", C.c_float),
        ("neighbor_bin_spacing", C.c_float),
        ("rest_density", C.c_float),
        ("rest_mass", C.c_float),
        ("max_speed", C.c_float),
        ("particle_rest_spacing", C.c_float),
        ("boundary_min", F3),
        ("boundary_max", F3),
        ("mover_center", F3),
        ("mover_radius", C.c_float),
        ("solve_steps", C.c_int32),
        ("neighbor_cap", C.c_int32),
        ("scorr_k", C.c_float),
        ("scorr_n", C.c_float),
        ("scorr_dq", C.c_float),
        ("exact_math", C.c_int32),
        ("solver", C.c_int32),
        ("residual_tol", C.c_float),
        ("max_iterations", C.c_int32),
        ("residual_sample", C.c_int32),
    ]

    def as_dict(self) -> dict:
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if hasattr(v, "__len__") else v
        return out


class PbfStats(C.Structure):
    _fields_ = [
        ("n", C.c_uint64),
        ("mean_density_error", C.c_double),
        ("max_density_error", C.c_double),
        ("kinetic_energy", C.c_double),
        ("center_of_mass", C.c_double * 3),
        ("mean_neighbors", C.c_double),
        ("cap_hits", C.c_uint64),
        ("error_flags", C.c_uint32),
        ("solver_iterations", C.c_uint32),
        ("solver_residual", C.c_double),
        ("tiles", C.c_uint32),
        ("tiles_staged", C.c_uint32),
        ("lists_slot_order", C.c_uint32),
    ]

    def as_dict(self) -> dict:
        return {
            "n": int(self.n),
            "mean_density_error": self.mean_density_error,
            "max_density_error": self.max_density_error,
            "kinetic_energy": self.kinetic_energy,
            "center_of_mass": list(self.center_of_mass),
            "mean_neighbors": self.mean_neighbors,
            "cap_hits": int(self.cap_hits),
            "error_flags": int(self.error_flags),
            "solver_iterations": int(self.solver_iterations),
            "solver_residual": self.solver_residual,
            "tiles": int(self.tiles),
            "tiles_staged": int(self.tiles_staged),
            "lists_slot_order": int(self.lists_slot_order),
        }


class PbfScene(C.Structure):
    _fields_ = [("boundary_min", F3), ("boundary_max", F3), ("count", C.c_size_t)]


class PbfTuning(C.Structure):
    _fields_ = [("lanes", C.c_int * 5), ("block", C.c_int * 5), ("staged", C.c_int * 5)]

    def as_dict(self) -> dict:
        return {f: (int(self.lanes[i]), int(self.block[i]), int(self.staged[i])) for i, f in enumerate(TUNE_FAMILIES)}


_P = C.POINTER
_vp = C.c_void_p
_i = C.c_int
_sz = C.c_size_t
_fp = _P(C.c_float)

# name -> (restype, argtypes); every symbol include/pbf.h declares.
SIGNATURES = {
    "pbf_params_init": (None, [_P(PbfParams)]),
    "pbf_params_derive": (_i, [_P(PbfParams), C.c_float, C.c_float]),
    "pbf_params_from_ini": (_i, [C.c_char_p, _P(PbfParams), _fp, _fp]),
    "pbf_lattice_dims": (_i, [_fp, _fp, C.c_float, _P(C.c_int64)]),
    "pbf_build_lattice": (_i, [_fp, _P(C.c_int64), C.c_float, C.c_float, C.c_uint64, _fp]),
    "pbf_lattice_rest_density": (_i, [_P(PbfParams), C.c_float, _fp]),
    "pbf_grid_dims": (_i, [_P(PbfParams), _P(C.c_int64)]),
    "pbf_create": (_i, [_P(PbfParams), _sz, _P(_vp)]),
    "pbf_destroy": (None, [_vp]),
    "pbf_last_error": (C.c_char_p, [_vp]),
    "pbf_create_error": (C.c_char_p, []),
    "pbf_set_params": (_i, [_vp, _P(PbfParams)]),
    "pbf_get_params": (_i, [_vp, _P(PbfParams)]),
    "pbf_upload": (_i, [_vp, _vp, _vp, _sz]),
    "pbf_download": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "pbf_count": (_sz, [_vp]),
    "pbf_get_array": (_i, [_vp, _i, _vp]),
    "pbf_set_array": (_i, [_vp, _i, _vp]),
    "pbf_apply_external_forces": (_i, [_vp, _sz, _sz]),
    "pbf_predict_positions": (_i, [_vp, _sz, _sz]),
    "pbf_find_neighbors": (_i, [_vp, _sz, _sz, _sz, _sz]),
    "pbf_compute_densities": (_i, [_vp, _sz, _sz]),
    "pbf_compute_pressure_lambdas": (_i, [_vp, _sz, _sz]),
    "pbf_compute_pressure_dps": (_i, [_vp, _sz, _sz, _i]),
    "pbf_update_position_stars": (_i, [_vp, _sz, _sz]),
    "pbf_update_velocities": (_i, [_vp, _sz, _sz]),
    "pbf_apply_surface_tension": (_i, [_vp, _sz, _sz, _sz, _sz]),
    "pbf_apply_viscosity": (_i, [_vp, _sz, _sz]),
    "pbf_compute_vorticity": (_i, [_vp, _sz, _sz]),
    "pbf_apply_vorticity": (_i, [_vp, _sz, _sz]),
    "pbf_update_positions": (_i, [_vp, _sz, _sz]),
    "pbf_step": (_i, [_vp, _i]),
    "pbf_get_neighbors": (_i, [_vp, _vp, _vp]),
    "pbf_get_bins": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "pbf_num_bins": (C.c_int64, [_vp]),
    "pbf_stats": (_i, [_vp, _P(PbfStats)]),
    "pbf_sync": (_i, [_vp]),
    "pbf_get_stream": (_i, [_vp, _P(_vp)]),
    "pbf_set_timing": (_i, [_vp, _i]),
    "pbf_kernel_times": (_i, [_vp, _i, _P(C.c_char_p), _P(C.c_int64), _P(C.c_double), _P(C.c_int)]),
    "pbf_reset_timing": (_i, [_vp]),
    "pbf_launches_per_step": (_i, [_vp, _P(C.c_int64)]),
    "pbf_add_particles": (_i, [_vp, _vp, _vp, _sz]),
    "pbf_construct_fluid": (_i, [_vp, _P(C.c_float), _P(C.c_float), _P(C.c_float), _P(_sz)]),
    "pbf_step_count": (C.c_uint64, [_vp]),
    "pbf_save_state": (_i, [_vp, C.c_char_p]),
    "pbf_load_state": (_i, [_vp, C.c_char_p]),
    "pbf_create_batch": (_i, [_P(PbfParams), _P(PbfScene), _i, _P(_vp)]),
    "pbf_scene_count": (_i, [_vp]),
    "pbf_scene_stats": (_i, [_vp, _i, _P(PbfStats)]),
    "pbf_get_tuning": (_i, [_vp, _P(PbfTuning)]),
    "pbf_set_tuning": (_i, [_vp, _P(PbfTuning)]),
    "pbf_autotune": (_i, [_vp, _i, _P(PbfTuning), _P(C.c_double)]),
    "pbf_find_neighbors_noalloc": (_i, [_P(PbfParams), _vp, _sz, _vp, _vp, _vp, _vp]),
    "pbf_mlp_init": (_i, [_vp, C.c_uint64]),
    "pbf_mlp_get": (_i, [_vp, _vp, _vp]),
    "pbf_mlp_set": (_i, [_vp, _vp, _vp]),
    "pbf_set_recording": (_i, [_vp, _i]),
    "pbf_get_training_data": (_i, [_vp, _vp, _vp]),
    "pbf_mlp_train": (_i, [_vp, _i, _i, C.c_float, C.c_uint64, _P(C.c_float)]),
    "pbf_mlp_gradients": (_i, [_vp, _vp, _vp, _sz, _vp, _P(C.c_float)]),
    "pbf_mlp_predict": (_i, [_vp, _vp, _sz, _vp]),
    "pbf_selftest_mlp_wait_timeout": (_i, [_vp, _vp]),
    "pbf_set_persistent": (_i, [_vp, _i]),
    "pbf_selftest_persistent_wait_timeout": (_i, [_vp, _vp]),
    "pbf_group_create": (_i, [_vp, _i, _P(_vp)]),
    "pbf_group_step": (_i, [_vp, _i]),
    "pbf_group_sync": (_i, [_vp]),
    "pbf_group_get_stream": (_i, [_vp, _P(_vp)]),
    "pbf_group_destroy": (None, [_vp]),
}

_lib = None


def load(path: Path | None = None) -> C.CDLL:
    """Load libpbf_b200.so; raises if it has not been built (there is no fallback)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(
            f"{p} is missing: build it with `python sph-cpp_b200/build.py` (the PBF step has no CPU fallback)")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib
