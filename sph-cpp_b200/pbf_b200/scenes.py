"""Dam-break workloads of the PBF step.

All scenes share the physics of the reference's runtime INI with the values
the benchmark configurations fix: h = 1, lattice spacing 0.5h, bin spacing
s = 1.2h (parameters.h:132-133), g = -9.8 on y (particles.h:268), dt = 0.016,
relaxation epsilon 600, XSPH c = 0.01, vorticity epsilon 0.0005, gamma = 0
(surface tension off), the mover sphere parked outside the box
(Runtime/params.ini:24-25), rest density taken from an interior lattice
particle, and a seeded +-0.005h jitter on the construct_fluid lattice.

  dam_65k    65,536 particles, 32x32x64 lattice in a 40^3 box, K = 3
  dam_1m     1,048,576 particles, 128x128x64 lattice, 160x160x80 box, K = 3
  dam_16m    16,777,216 particles, 256^3 lattice, 320^3 box, K = 4, cap 64
plus small cases for tests, and batches of independent dam-break scenes
(make_batch): counts drawn log-uniform from a seed, lattice blocks of random
aspect ratio, each in its own box 1.5x its extent.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, replace

import numpy as np

from . import _abi


@dataclass(frozen=True)
class Scene:
    name: str
    lattice: tuple[int, int, int]          # particles per axis (x, y, z)
    box_max: tuple[float, float, float]    # boundary max; boundary min is the origin
    solve_steps: int = 3
    steps: int = 100
    h: float = 1.0
    spacing: float = 0.5
    fluid_min: tuple[float, float, float] = (0.0, 0.0, 0.0)
    gravity: float = -9.8
    time_step: float = 0.016
    lambda_epsilon: float = 600.0
    visc_c: float = 0.01
    vorticity_coef: float = 0.0005
    gamma: float = 0.0
    jitter: float = 0.005                  # in units of h
    seed: int = 20161201
    neighbor_cap: int = 60
    mover_center: tuple[float, float, float] = (-1.5, -2.0, -1.5)
    scorr: tuple[float, float, float] = (0.0, 4.0, 0.2)  # (k, n, dq/h); k = 0 is the reference's Δp
    exact_math: int = 0
    solver: int = 0                        # 0 plain K iterations, 1 learned warm start
    residual_tol: float = 0.01             # learned solver: mean clamped density error target
    max_iterations: int = 8                # learned solver: iterations per step at most
    residual_sample: int = 1               # learned solver: residual over every S-th run of 32 slots

    @property
    def n(self) -> int:
        return int(self.lattice[0] * self.lattice[1] * self.lattice[2])

    @property
    def fluid_max(self) -> tuple[float, float, float]:
        return tuple(self.fluid_min[a] + self.lattice[a] * self.spacing for a in range(3))

    def with_(self, **kw) -> "Scene":
        return replace(self, **kw)

    def params(self) -> _abi.PbfParams:
        """Parameter block as Parameters::derive_from_input builds it (parameters.h:123-148),
        with rest density from the interior of the unjittered lattice."""
        lib = _abi.load()
        p = _abi.PbfParams()
        lib.pbf_params_init(C.byref(p))
        p.time_step = self.time_step
        p.gravity = self.gravity
        p.gamma = self.gamma
        p.visc_c = self.visc_c
        p.lambda_epsilon = self.lambda_epsilon
        p.vorticity_coef = self.vorticity_coef
        p.smoothing_radius = self.h
        p.neighbor_bin_spacing = -1.0
        p.solve_steps = self.solve_steps
        p.neighbor_cap = self.neighbor_cap
        for a in range(3):
            p.boundary_min[a] = 0.0
            p.boundary_max[a] = self.box_max[a]
            p.mover_center[a] = self.mover_center[a]
        p.scorr_k, p.scorr_n, p.scorr_dq = self.scorr
        p.exact_math = self.exact_math
        p.solver = self.solver
        p.residual_tol = self.residual_tol
        p.max_iterations = self.max_iterations
        p.residual_sample = self.residual_sample
        rc = lib.pbf_params_derive(C.byref(p), self.spacing, -1.0)
        if rc:
            raise RuntimeError(f"pbf_params_derive failed ({rc})")
        rho0 = C.c_float()
        rc = lib.pbf_lattice_rest_density(C.byref(p), self.spacing, C.byref(rho0))
        if rc:
            raise RuntimeError(f"pbf_lattice_rest_density failed ({rc})")
        p.rest_density = rho0.value
        return p

    def positions(self) -> np.ndarray:
        """construct_fluid lattice (particles.h:231-250) with the seeded jitter, AoS float32 (N, 3)."""
        lib = _abi.load()
        x = np.empty((self.n, 3), np.float32)
        mn = (C.c_float * 3)(*self.fluid_min)
        d = (C.c_int64 * 3)(*self.lattice)
        rc = lib.pbf_build_lattice(mn, d, self.spacing, self.jitter * self.h, self.seed,
                                   x.ctypes.data_as(C.POINTER(C.c_float)))
        if rc:
            raise RuntimeError(f"pbf_build_lattice failed ({rc})")
        return x


SCENES: dict[str, Scene] = {
    # 65k dam break: small enough for the reference's CPU build to run in full
    "dam_65k": Scene("dam_65k", (32, 32, 64), (40.0, 40.0, 40.0), solve_steps=3, steps=100),
    # 1M dam break: the throughput workload
    "dam_1m": Scene("dam_1m", (128, 128, 64), (160.0, 160.0, 80.0), solve_steps=3, steps=200),
    # 16.8M dam break: single-GPU memory sizing, lists capped at 64
    "dam_16m": Scene("dam_16m", (256, 256, 256), (320.0, 320.0, 320.0), solve_steps=4, steps=50,
                     neighbor_cap=64),
    # small parity cases
    "dam_2k": Scene("dam_2k", (16, 16, 8), (13.0, 13.0, 13.0), solve_steps=3, steps=20),
    "dam_8k": Scene("dam_8k", (16, 16, 32), (20.0, 20.0, 20.0), solve_steps=3, steps=50),
}


def make_scene(name: str, **overrides) -> Scene:
    s = SCENES[name]
    return s.with_(**overrides) if overrides else s


# ---------------------------------------------------------------- batches
@dataclass(frozen=True)
class Batch:
    """Independent scenes advanced by one context (pbf_create_batch), sharing
    the physics of scenes[0]; particles are the scenes' concatenated in order."""
    name: str
    scenes: tuple[Scene, ...]

    @property
    def n(self) -> int:
        return sum(s.n for s in self.scenes)

    @property
    def counts(self) -> list[int]:
        return [s.n for s in self.scenes]

    @property
    def offsets(self) -> np.ndarray:
        return np.concatenate([[0], np.cumsum(self.counts)]).astype(np.int64)

    def with_(self, **kw) -> "Batch":
        return Batch(self.name, tuple(s.with_(**kw) for s in self.scenes))

    def params(self) -> _abi.PbfParams:
        return self.scenes[0].params()

    def scene_structs(self) -> list:
        out = []
        for s in self.scenes:
            sc = _abi.PbfScene()
            for a in range(3):
                sc.boundary_min[a] = 0.0
                sc.boundary_max[a] = s.box_max[a]
            sc.count = s.n
            out.append(sc)
        return out

    def positions(self) -> np.ndarray:
        return np.concatenate([s.positions() for s in self.scenes])


def _box_extent(extent: float, s: float = 1.2) -> float:
    """1.5x the fluid extent, moved off a multiple of the bin spacing s (a box
    max that is a multiple of s leaves its +s re-hash outside the reference's
    grid, neighbors.h:69-71)."""
    b = round(1.5 * extent, 3)
    while abs(b / s - round(b / s)) < 1e-3:
        b += 0.05
    return b


def make_batch(scenes: int = 64, seed: int = 20161202, n_min: int = 4096, n_max: int = 262144,
               name: str = "batch_64", **physics) -> Batch:
    """Seeded batch of dam breaks: particle counts log-uniform in [n_min,
    n_max], each a lattice block (spacing 0.5h) with y/x and z/x aspect ratios
    uniform in [0.5, 2], the block at the origin of its own box 1.5x its
    extent; scene i jitters with seed + i."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(scenes):
        target = float(np.exp(rng.uniform(np.log(n_min), np.log(n_max))))
        ay, az = rng.uniform(0.5, 2.0, 2)
        nx = max(1, int(round((target / (ay * az)) ** (1.0 / 3.0))))

        def dims(nx):
            return nx, max(1, int(round(ay * nx))), max(1, int(round(az * nx)))

        while np.prod(dims(nx)) < n_min:
            nx += 1
        while np.prod(dims(nx)) > n_max and nx > 1:
            nx -= 1
        lat = dims(nx)
        sp = physics.get("spacing", 0.5)
        box = tuple(_box_extent(lat[a] * sp) for a in range(3))
        out.append(Scene(f"{name}[{i}]", lat, box, seed=seed + i, **physics))
    return Batch(name, tuple(out))
