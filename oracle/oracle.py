"""Python access to the two CPU checkers of the PBF step.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference arm; never by the product package.

  OracleSim  the plain-C restatement of the reference algorithm (oracle/pbf_oracle.c)
  RefSim     the reference's own particles.h/neighbors.h compiled from its
             sources (oracle/ref_build/Makefile -> oracle/_ref/libpbf_ref*.so)

Both take the product's pbf_params block (include/pbf.h) so a scene feeds
the GPU path and both checkers identically.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
ORACLE_LIB = ROOT / "_build" / "libpbf_oracle.so"

# Stage numbering shared by both checkers (and the reference driver).
STAGES = ["apply_external_forces", "predict_positions", "find_neighbors", "compute_densities",
          "compute_pressure_lambdas", "compute_pressure_dps", "update_position_stars", "update_velocities",
          "apply_surface_tension", "apply_viscosity", "compute_vorticity", "apply_vorticity", "update_positions"]

ARRAY_POSITIONS, ARRAY_POSITION_STARS, ARRAY_VELOCITIES, ARRAY_SCRATCH, ARRAY_DENSITIES, ARRAY_LAMBDAS = range(6)


def _params_type():
    import sys
    pkg = ROOT.parent / "sph-cpp_b200"
    if str(pkg) not in sys.path:
        sys.path.insert(0, str(pkg))
    from pbf_b200._abi import PbfParams, PbfStats
    return PbfParams, PbfStats


PbfParams, PbfStats = _params_type()
_vp = C.c_void_p


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


_oracle = None


def oracle_lib() -> C.CDLL:
    global _oracle
    if _oracle is None:
        if not ORACLE_LIB.exists():
            raise RuntimeError(f"{ORACLE_LIB} missing: run `python sph-cpp_b200/build.py`")
        lib = C.CDLL(str(ORACLE_LIB))
        P = C.POINTER(PbfParams)
        sig = {
            "oracle_params_derive": (C.c_int, [P, C.c_float, C.c_float]),
            "oracle_lattice_dims": (C.c_int, [_vp, _vp, C.c_float, _vp]),
            "oracle_build_lattice": (C.c_int, [_vp, _vp, C.c_float, C.c_float, C.c_uint64, _vp]),
            "oracle_grid_dims": (C.c_int, [P, _vp]),
            "oracle_create": (_vp, [P, C.c_size_t]),
            "oracle_destroy": (None, [_vp]),
            "oracle_set_visc_mode": (None, [_vp, C.c_int]),
            "oracle_set_params": (None, [_vp, P]),
            "oracle_set_state": (C.c_int, [_vp, _vp, _vp, C.c_size_t]),
            "oracle_get": (C.c_int, [_vp, C.c_int, _vp]),
            "oracle_set": (C.c_int, [_vp, C.c_int, _vp]),
            "oracle_bin_id": (C.c_uint64, [_vp, _vp]),
            "oracle_stage": (C.c_int, [_vp, C.c_int, C.c_int]),
            "oracle_step": (C.c_int, [_vp, C.c_int]),
            "oracle_get_neighbors": (C.c_int, [_vp, _vp, _vp]),
            "oracle_get_bins": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
            "oracle_num_bins": (C.c_int64, [_vp]),
            "oracle_stats": (C.c_int, [_vp, C.POINTER(PbfStats)]),
            "oracle_poly6": (C.c_float, [C.c_float, C.c_float]),
            "oracle_del_spikey": (None, [C.c_float, _vp, _vp, _vp]),
            "oracle_c_spline": (C.c_float, [C.c_float, C.c_float]),
            "oracle_lattice_rest_density": (C.c_int, [P, C.c_float, C.POINTER(C.c_float)]),
        }
        for k, (r, a) in sig.items():
            f = getattr(lib, k)
            f.restype = r
            f.argtypes = a
        _oracle = lib
    return _oracle


class OracleSim:
    """CPU restatement; visc_mode 0 = Jacobi XSPH (GPU semantics), 1 = the
    reference's in-place single-thread order."""

    def __init__(self, params, capacity: int, visc_mode: int = 0):
        self.lib = oracle_lib()
        self.params = params
        self.h = self.lib.oracle_create(C.byref(params), int(capacity))
        if not self.h:
            raise RuntimeError("oracle_create failed")
        self.cap = params.neighbor_cap
        self.lib.oracle_set_visc_mode(self.h, visc_mode)
        self.n = 0

    def close(self):
        if self.h:
            self.lib.oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def set_state(self, x, v=None):
        x = np.ascontiguousarray(x, np.float32).reshape(-1, 3)
        v = None if v is None else np.ascontiguousarray(v, np.float32).reshape(-1, 3)
        rc = self.lib.oracle_set_state(self.h, _ptr(x), _ptr(v), x.shape[0])
        if rc:
            raise RuntimeError(f"oracle_set_state {rc}")
        self.n = x.shape[0]

    def stage(self, i: int, sub: int = 0):
        rc = self.lib.oracle_stage(self.h, i, sub)
        if rc:
            raise RuntimeError(f"oracle stage {STAGES[i]} failed {rc}")

    def step(self, n: int = 1):
        rc = self.lib.oracle_step(self.h, n)
        if rc:
            raise RuntimeError(f"oracle_step {rc}")

    def get(self, which: int) -> np.ndarray:
        out = np.empty((self.n, 3) if which <= ARRAY_SCRATCH else (self.n,), np.float32)
        self.lib.oracle_get(self.h, which, _ptr(out))
        return out

    def set(self, which: int, a):
        a = np.ascontiguousarray(a, np.float32)
        self.lib.oracle_set(self.h, which, _ptr(a))

    def neighbors(self):
        idx = np.empty((self.n, self.cap), np.int32)
        cnt = np.empty(self.n, np.int32)
        self.lib.oracle_get_neighbors(self.h, _ptr(idx), _ptr(cnt))
        return idx, cnt

    def bins(self):
        B = int(self.lib.oracle_num_bins(self.h))
        keys = np.empty(self.n, np.uint32)
        ids = np.empty(self.n, np.uint32)
        b0 = np.empty(B, np.uint32)
        b1 = np.empty(B, np.uint32)
        self.lib.oracle_get_bins(self.h, _ptr(keys), _ptr(ids), _ptr(b0), _ptr(b1))
        return {"sorted_keys": keys, "sorted_ids": ids, "bin_begin": b0, "bin_end": b1}

    def bin_id(self, p) -> int:
        a = np.ascontiguousarray(p, np.float32)
        return int(self.lib.oracle_bin_id(self.h, _ptr(a)))

    def stats(self) -> dict:
        st = PbfStats()
        rc = self.lib.oracle_stats(self.h, C.byref(st))
        if rc:
            raise RuntimeError(f"oracle_stats {rc}")
        return st.as_dict()


# ---------------------------------------------------------------- reference
# The reference build's bindings live in reflib (no product import there).
from .reflib import REF_LIB, REF_LIB_SERIAL, RefParams, host_cores, ref_available, ref_lib  # noqa: E402,F401


def ref_params_from(p, capacity: int, fluid_min=(0, 0, 0), fluid_max=(0, 0, 0)) -> RefParams:
    r = RefParams()
    r.time_step = p.time_step
    r.gravity = p.gravity
    r.gamma = p.gamma
    r.visc_c = p.visc_c
    r.lambda_epsilon = p.lambda_epsilon
    r.k_stiff = 1.0
    r.vorticity_coef = p.vorticity_coef
    r.smoothing_radius = p.smoothing_radius
    r.neighbor_bin_spacing = p.neighbor_bin_spacing
    r.rest_spacing = p.particle_rest_spacing
    for a in range(3):
        r.boundary_min[a] = p.boundary_min[a]
        r.boundary_max[a] = p.boundary_max[a]
        r.fluid_min[a] = fluid_min[a]
        r.fluid_max[a] = fluid_max[a]
        r.mover_center[a] = p.mover_center[a]
    r.solve_steps = p.solve_steps
    r.max_particles_local = capacity
    r.global_particle_count = capacity
    r.rest_density = p.rest_density
    return r


class RefSim:
    """The reference's own Particles<float,3>, driven over [0, N) as its
    serial tests do (no MPI Distributor)."""

    def __init__(self, params, capacity: int, serial: bool = False, threads: int | None = None):
        if params.neighbor_cap != 60:
            raise ValueError("the reference's neighbor cap is the compile-time MAX_NEIGHBORS = 60")
        if params.scorr_k != 0.0:
            raise ValueError("the reference has no s_corr term")
        self.lib = ref_lib(serial)
        if threads is not None:
            self.lib.ref_set_threads(threads)
        self.rp = ref_params_from(params, capacity)
        self.h = self.lib.ref_create(C.byref(self.rp))
        if not self.h:
            raise RuntimeError("ref_create: " + self.lib.ref_last_error().decode())
        self.cap = 60
        self.n = 0

    def close(self):
        if self.h:
            self.lib.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def set_state(self, x, v=None):
        x = np.ascontiguousarray(x, np.float32).reshape(-1, 3)
        v = np.zeros_like(x) if v is None else np.ascontiguousarray(v, np.float32).reshape(-1, 3)
        if self.lib.ref_add(self.h, _ptr(x), _ptr(v), x.shape[0]):
            raise RuntimeError("ref_add: " + self.lib.ref_last_error().decode())
        self.n = int(self.lib.ref_count(self.h))

    def stage(self, i: int, sub: int = 0):
        if self.lib.ref_stage(self.h, i, sub):
            raise RuntimeError("ref_stage: " + self.lib.ref_last_error().decode())

    def step(self, n: int = 1):
        if self.lib.ref_step(self.h, n):
            raise RuntimeError("ref_step: " + self.lib.ref_last_error().decode())

    def time_steps(self, n: int) -> float:
        t = self.lib.ref_time_steps(self.h, n)
        if t < 0:
            raise RuntimeError("ref_step: " + self.lib.ref_last_error().decode())
        return t

    def get(self, which: int) -> np.ndarray:
        if which <= ARRAY_SCRATCH:
            out = np.empty((self.n, 3), np.float32)
            self.lib.ref_get_vec(self.h, which, _ptr(out))
        else:
            out = np.empty(self.n, np.float32)
            self.lib.ref_get_scalar(self.h, which - ARRAY_DENSITIES, _ptr(out))
        return out

    def set(self, which: int, a):
        a = np.ascontiguousarray(a, np.float32)
        if which <= ARRAY_SCRATCH:
            self.lib.ref_set_vec(self.h, which, _ptr(a))
        else:
            self.lib.ref_set_scalar(self.h, which - ARRAY_DENSITIES, _ptr(a))

    def neighbors(self):
        idx = np.full((self.n, self.cap), -1, np.int32)
        cnt = np.empty(self.n, np.int32)
        self.lib.ref_get_neighbors(self.h, _ptr(idx), _ptr(cnt), self.cap)
        return idx, cnt

    def bin_dims(self):
        d = np.empty(3, np.uint64)
        self.lib.ref_bin_dims(self.h, _ptr(d))
        return tuple(int(v) for v in d)

    def bin_id(self, p) -> int:
        a = np.ascontiguousarray(p, np.float32)
        return int(self.lib.ref_bin_id(self.h, _ptr(a)))

    def bins(self):
        d = self.bin_dims()
        B = d[0] * d[1] * d[2]
        keys = np.empty(self.n, np.uint64)
        ids = np.empty(self.n, np.uint64)
        b0 = np.empty(B, np.uint64)
        b1 = np.empty(B, np.uint64)
        self.lib.ref_get_bins(self.h, _ptr(keys), _ptr(ids), _ptr(b0), _ptr(b1))
        return {"sorted_keys": keys, "sorted_ids": ids, "bin_begin": b0, "bin_end": b1}

    def stats(self, params) -> dict:
        """Residual statistics computed the way pbf_stats does, from the
        reference's own arrays after one more compute_densities pass."""
        self.stage(3)
        rho = self.get(ARRAY_DENSITIES).astype(np.float64)
        x = self.get(ARRAY_POSITIONS).astype(np.float64)
        v = self.get(ARRAY_VELOCITIES).astype(np.float64)
        _, cnt = self.neighbors()
        err = np.maximum(rho / float(params.rest_density) - 1.0, 0.0)
        return {
            "n": self.n,
            "mean_density_error": float(err.mean()),
            "max_density_error": float(err.max()),
            "kinetic_energy": float(0.5 * float(params.rest_mass) * (v * v).sum()),
            "center_of_mass": [float(c) for c in x.mean(axis=0)],
            "mean_neighbors": float(cnt.mean()),
            "cap_hits": int((cnt >= self.cap).sum()),
            "error_flags": 0,
        }
