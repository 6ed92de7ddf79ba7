"""The dam-break workloads of the benchmark, built from the reference's own
build and numpy alone, and the timed runs of the reference on them.

TEST INFRASTRUCTURE ONLY: bench.py's reference arm and CPU baseline, and the
tests that check these workloads equal the product's (tests/test_ref_arm.py).
Nothing here imports the product package or loads its library, so the
reference arm's process maps only the reference build.

A workload is the reference's own scene set-up with the benchmark's values:
  - parameters: Parameters::derive_from_input (Common/parameters.h:123-148)
    inside the reference build (ref_create), h = 1, spacing 0.5h, bin
    spacing derived (1.2h), gamma 0, the mover sphere parked outside the box;
  - rest density: the reference's find_neighbors + compute_densities
    (Simulation/Source/neighbors.h:197-230, particles.h:292-313) on an
    unjittered 9^3 construct_fluid lattice, read at its centre particle;
  - positions: the reference's construct_fluid (particles.h:231-250) over
    [0, lattice * spacing], then a seeded jitter, uniform in +-0.005h per
    axis, from a SplitMix64 counter stream (Steele, Lea and Flood, "Fast
    splittable pseudorandom number generators", OOPSLA 2014) restated below
    in numpy: value k of the stream is splitmix64(seed + k * 0x9E3779B97F4A7C15)
    for k = 3 * particle + axis, its top 24 bits scaled to u in [0, 1), and
    the jitter (2u - 1) * amplitude, all in float32, added to the lattice.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field

import numpy as np

from .reflib import RefParams, host_cores, ref_available, ref_lib

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)


@dataclass(frozen=True)
class Workload:
    name: str
    lattice: tuple[int, int, int]          # particles per axis (x, y, z)
    box_max: tuple[float, float, float]    # boundary max; boundary min is the origin
    solve_steps: int = 3
    neighbor_cap: int = 60
    h: float = 1.0
    spacing: float = 0.5
    gravity: float = -9.8
    time_step: float = 0.016
    lambda_epsilon: float = 600.0
    visc_c: float = 0.01
    vorticity_coef: float = 0.0005
    gamma: float = 0.0
    jitter: float = 0.005                  # in units of h
    seed: int = 20161201
    mover_center: tuple[float, float, float] = field(default=(-1.5, -2.0, -1.5))

    @property
    def n(self) -> int:
        return int(self.lattice[0] * self.lattice[1] * self.lattice[2])

    @property
    def fluid_extent(self) -> tuple[float, float, float]:
        """The lattice's extent, lattice * spacing per axis."""
        return tuple(float(self.lattice[a] * self.spacing) for a in range(3))

    @property
    def fluid_max(self) -> tuple[float, float, float]:
        """The box construct_fluid fills: half a spacing past the lattice's
        extent, so that its floor(extent / spacing) count is the lattice's
        whatever the rounding of extent / spacing (the points themselves are
        index * spacing + min + spacing / 2, independent of the box's max)."""
        return tuple(float((self.lattice[a] + 0.5) * self.spacing) for a in range(3))


# The benchmark's dam breaks (lattice, box, Jacobi iterations, neighbor cap).
WORKLOADS: dict[str, Workload] = {
    "dam_65k": Workload("dam_65k", (32, 32, 64), (40.0, 40.0, 40.0), 3),
    "dam_1m": Workload("dam_1m", (128, 128, 64), (160.0, 160.0, 80.0), 3),
    "dam_16m": Workload("dam_16m", (256, 256, 256), (320.0, 320.0, 320.0), 4, neighbor_cap=64),
    "dam_2k": Workload("dam_2k", (16, 16, 8), (13.0, 13.0, 13.0), 3),
    "dam_8k": Workload("dam_8k", (16, 16, 32), (20.0, 20.0, 20.0), 3),
}


def ref_params(w: Workload, box_max=None, fluid_max=None, capacity: int | None = None,
               rest_density: float = -1.0) -> RefParams:
    r = RefParams()
    r.time_step = w.time_step
    r.gravity = w.gravity
    r.gamma = w.gamma
    r.visc_c = w.visc_c
    r.lambda_epsilon = w.lambda_epsilon
    r.k_stiff = 1.0
    r.vorticity_coef = w.vorticity_coef
    r.smoothing_radius = w.h
    r.neighbor_bin_spacing = -1.0       # derived: 1.2 h (parameters.h:132-133)
    r.rest_spacing = w.spacing
    box = w.box_max if box_max is None else box_max
    fmax = w.fluid_max if fluid_max is None else fluid_max
    for a in range(3):
        r.boundary_min[a] = 0.0
        r.boundary_max[a] = box[a]
        r.fluid_min[a] = 0.0
        r.fluid_max[a] = fmax[a]
        r.mover_center[a] = w.mover_center[a]
    r.solve_steps = w.solve_steps
    cap = w.n if capacity is None else capacity
    r.max_particles_local = cap
    r.global_particle_count = cap
    r.rest_density = rest_density
    return r


def derived(w: Workload) -> dict:
    """The reference's derived parameters (parameters.h:123-148) for w."""
    out = (C.c_float * 8)()
    lib = ref_lib()
    if lib.ref_derived(C.byref(ref_params(w)), out):
        raise RuntimeError("ref_derived: " + lib.ref_last_error().decode())
    keys = ("rest_spacing", "particle_radius", "smoothing_radius", "neighbor_bin_spacing", "rest_density",
            "rest_mass", "max_speed", "solve_steps")
    return dict(zip(keys, (float(v) for v in out)))


def rest_density(w: Workload, r: int = 4) -> float:
    """Density of the centre particle of an unjittered (2r+1)^3 lattice, from
    the reference's own construct_fluid, find_neighbors and compute_densities."""
    lib = ref_lib()
    n1 = 2 * r + 1
    ext = tuple(float((n1 + 0.5) * w.spacing) for _ in range(3))
    rp = ref_params(w, box_max=ext, fluid_max=ext, capacity=n1 ** 3)
    h = lib.ref_create(C.byref(rp))
    if not h:
        raise RuntimeError("ref_create: " + lib.ref_last_error().decode())
    try:
        if lib.ref_construct_fluid(h) != n1 ** 3:
            raise RuntimeError("ref_construct_fluid: " + lib.ref_last_error().decode())
        for stage in (2, 3):  # find_neighbors, compute_densities
            if lib.ref_stage(h, stage, 0):
                raise RuntimeError("ref_stage: " + lib.ref_last_error().decode())
        rho = np.empty(n1 ** 3, np.float32)
        lib.ref_get_scalar(h, 0, rho.ctypes.data_as(C.c_void_p))
        return float(rho[r * n1 * n1 + r * n1 + r])
    finally:
        lib.ref_destroy(h)


def splitmix64(z: np.ndarray) -> np.ndarray:
    z = z + _GOLDEN
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def jitter(n: int, seed: int, amplitude: float) -> np.ndarray:
    """(n, 3) float32 jitter of the seeded counter stream described above."""
    k = np.arange(3 * n, dtype=np.uint64)
    with np.errstate(over="ignore"):
        r = splitmix64(np.uint64(seed) + _GOLDEN * k)
    u = (r >> np.uint64(40)).astype(np.float32) * np.float32(2.0 ** -24)
    return ((u * np.float32(2.0) - np.float32(1.0)) * np.float32(amplitude)).reshape(n, 3)


class RefRun:
    """One workload inside the reference build: its parameters, rest density
    and jittered construct_fluid lattice; steps run by the reference's
    main.cpp stage loop (ref_step)."""

    def __init__(self, w: Workload, threads: int | None = None, serial: bool = False):
        self.w = w
        self.lib = ref_lib(serial)
        if threads is not None:
            self.lib.ref_set_threads(threads)
        self.rho0 = rest_density(w)
        self.rp = ref_params(w, rest_density=self.rho0)
        self.h = self.lib.ref_create(C.byref(self.rp))
        if not self.h:
            raise RuntimeError("ref_create: " + self.lib.ref_last_error().decode())
        if self.lib.ref_construct_fluid(self.h) != w.n:
            raise RuntimeError("ref_construct_fluid did not build the workload's lattice")
        x = self.get(0)
        x += jitter(w.n, w.seed, w.jitter * w.h)
        self.set(0, x)
        self.set(1, x)  # x* = x, as construct_fluid adds them

    def get(self, which: int) -> np.ndarray:
        out = np.empty((self.w.n, 3), np.float32)
        self.lib.ref_get_vec(self.h, which, out.ctypes.data_as(C.c_void_p))
        return out

    def set(self, which: int, a: np.ndarray) -> None:
        a = np.ascontiguousarray(a, np.float32)
        self.lib.ref_set_vec(self.h, which, a.ctypes.data_as(C.c_void_p))

    def step(self, n: int = 1) -> None:
        if self.lib.ref_step(self.h, n):
            raise RuntimeError("ref_step: " + self.lib.ref_last_error().decode())

    def time_steps(self, n: int) -> float:
        t = self.lib.ref_time_steps(self.h, n)
        if t < 0:
            raise RuntimeError("ref_step: " + self.lib.ref_last_error().decode())
        return t

    def close(self) -> None:
        if self.h:
            self.lib.ref_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def time_reference(w: Workload, steps: int, warmup: int, threads: int, budget_s: float | None = None) -> dict:
    """particle-steps/s of the reference build on `threads` host threads:
    `warmup` untimed steps, then `steps` steps timed with std::chrono inside
    the build (at most as many as fit in budget_s, judged from one step)."""
    if not ref_available():
        raise RuntimeError("the reference build (oracle/_ref) is missing")
    with RefRun(w, threads=threads) as run:
        if warmup:
            run.step(warmup)
        if budget_s is not None:
            one = run.time_steps(1)
            steps = max(1, min(steps, int(budget_s / max(one, 1e-6))))
        dt = run.time_steps(steps)
    return {"value": w.n * steps / dt, "unit": "particle-steps/s", "cores": threads, "kind": "reference",
            "sample": f"{w.name}: {w.n} particles, {steps} timed full steps after {warmup} warm-up step(s) "
                      f"(+1 sizing step) on {threads} thread(s), std::chrono wall time {dt:.2f} s"
            if budget_s is not None else
            f"{w.name}: {w.n} particles, {steps} timed full steps after {warmup} warm-up step(s) on "
            f"{threads} thread(s), std::chrono wall time {dt:.2f} s",
            "steps": steps, "seconds": dt}


def all_cores() -> int:
    return host_cores()
