"""The reference's own Particles<float,3> as an engine of the slab
decomposition (pbf_b200.slabs.SlabDistributor): stages over explicit spans,
arrays in the reference's order, particles appended and dropped at the end,
construct_fluid over a box.

TEST INFRASTRUCTURE ONLY: the CPU engine of the multi-rank tests
(tests/test_slabs_gloo.py); nothing in the product imports it.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .ref_scene import Workload, ref_params
from .reflib import ref_lib

POSITIONS, POSITION_STARS, VELOCITIES, SCRATCH, DENSITIES, LAMBDAS = range(6)
STAGE = {"apply_external_forces": 0, "predict_positions": 1, "find_neighbors": 2, "compute_densities": 3,
         "compute_pressure_lambdas": 4, "compute_pressure_dps": 5, "update_position_stars": 6,
         "update_velocities": 7, "apply_surface_tension": 8, "apply_viscosity": 9, "compute_vorticity": 10,
         "apply_vorticity": 11, "update_positions": 12}


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class RefEngine:
    """One rank's particles inside the reference build.  `serial` selects the
    single-threaded build (deterministic in-place XSPH order)."""

    def __init__(self, w: Workload, capacity: int, rest_density: float, serial: bool = True, box_max=None):
        self.lib = ref_lib(serial)
        self.rp = ref_params(w, box_max=box_max, capacity=capacity, rest_density=rest_density)
        self.h = self.lib.ref_create(C.byref(self.rp))
        if not self.h:
            raise RuntimeError("ref_create: " + self.lib.ref_last_error().decode())

    def close(self):
        if self.h:
            self.lib.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _ok(self, rc):
        if rc:
            raise RuntimeError(self.lib.ref_last_error().decode())

    def local_count(self) -> int:
        return int(self.lib.ref_count(self.h))

    def get_array(self, which: int) -> np.ndarray:
        n = self.local_count()
        if which <= SCRATCH:
            out = np.empty((n, 3), np.float32)
            self.lib.ref_get_vec(self.h, which, _p(out))
        else:
            out = np.empty(n, np.float32)
            self.lib.ref_get_scalar(self.h, which - DENSITIES, _p(out))
        return out

    def set_array(self, which: int, a) -> None:
        a = np.ascontiguousarray(a, np.float32)
        if which <= SCRATCH:
            self.lib.ref_set_vec(self.h, which, _p(a))
        else:
            self.lib.ref_set_scalar(self.h, which - DENSITIES, _p(a))

    def append(self, x, x_star, v) -> None:
        x = np.ascontiguousarray(x, np.float32).reshape(-1, 3)
        n0 = self.local_count()
        self._ok(self.lib.ref_add(self.h, _p(x), _p(np.ascontiguousarray(v, np.float32)), x.shape[0]))
        xs = self.get_array(POSITION_STARS)
        xs[n0:] = x_star
        self.set_array(POSITION_STARS, xs)

    def remove(self, k: int) -> None:
        if k:
            self._ok(self.lib.ref_remove(self.h, int(k)))

    def construct_fluid(self, mn, mx, velocity=(0.0, 0.0, 0.0)) -> int:
        a = np.asarray(mn, np.float32)
        b = np.asarray(mx, np.float32)
        v = np.asarray(velocity, np.float32)
        k = int(self.lib.ref_construct_fluid_box(self.h, _p(a), _p(b), _p(v)))
        if k < 0:
            raise RuntimeError(self.lib.ref_last_error().decode())
        return k

    def _stage(self, name, a, b=(0, 0), sub=0):
        self._ok(self.lib.ref_stage_span(self.h, STAGE[name], sub, a[0], a[1], b[0], b[1]))

    def apply_external_forces(self, span):
        self._stage("apply_external_forces", span)

    def predict_positions(self, span):
        self._stage("predict_positions", span)

    def find_neighbors(self, bin_span, fill_span):
        self._stage("find_neighbors", bin_span, fill_span)

    def compute_densities(self, span):
        self._stage("compute_densities", span)

    def compute_pressure_lambdas(self, span):
        self._stage("compute_pressure_lambdas", span)

    def compute_pressure_dps(self, span, substep=0):
        self._stage("compute_pressure_dps", span, sub=substep)

    def update_position_stars(self, span):
        self._stage("update_position_stars", span)

    def update_velocities(self, span):
        self._stage("update_velocities", span)

    def apply_surface_tension(self, color_span, st_span):
        self._stage("apply_surface_tension", color_span, st_span)

    def apply_viscosity(self, span):
        self._stage("apply_viscosity", span)

    def compute_vorticity(self, span):
        self._stage("compute_vorticity", span)

    def apply_vorticity(self, span):
        self._stage("apply_vorticity", span)

    def update_positions(self, span):
        self._stage("update_positions", span)
