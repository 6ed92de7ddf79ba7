"""Python host side of the B200 PBF step (libpbf_b200.so through its C ABI).

`Particles` mirrors the reference's sim::Particles<float,3> call surface
(Simulation/Source/particles.h:256-487): the same stage names, the same span
arguments ([0, N) on a single rank) and the same error behaviour (a failing
call raises RuntimeError, as the reference throws std::runtime_error).
`scenes` builds the dam-break workloads.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import PbfParams, PbfStats  # noqa: F401
from .scenes import SCENES, Batch, Scene, make_batch, make_scene  # noqa: F401

__all__ = ["Particles", "PbfParams", "PbfStats", "Scene", "SceneGroup", "make_scene", "SCENES", "lib",
           "params_init"]


def lib() -> C.CDLL:
    return _abi.load()


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def params_init() -> PbfParams:
    p = PbfParams()
    lib().pbf_params_init(C.byref(p))
    return p


class Particles:
    """A device-resident particle set plus its PBF solver (one pbf_ctx).

    Particles(params, capacity) holds one scene; Particles.batch(batch) holds
    the independent scenes of a scenes.Batch, advanced in the same launches
    (particles indexed as the scenes concatenated in order)."""

    def __init__(self, params: PbfParams, capacity: int, scenes=None):
        self._lib = lib()
        self._ctx = C.c_void_p()
        self.scene_offsets = None
        if scenes is None:
            rc = self._lib.pbf_create(C.byref(params), int(capacity), C.byref(self._ctx))
        else:
            arr = (_abi.PbfScene * len(scenes))(*scenes)
            rc = self._lib.pbf_create_batch(C.byref(params), arr, len(scenes), C.byref(self._ctx))
            self.scene_offsets = np.concatenate([[0], np.cumsum([int(sc.count) for sc in scenes])])
            capacity = int(self.scene_offsets[-1])
        if rc != 0:
            raise RuntimeError(f"pbf_create failed ({rc}): {self._lib.pbf_create_error().decode()}")
        self.capacity = int(capacity)

    @classmethod
    def batch(cls, batch) -> "Particles":
        return cls(batch.params(), 0, scenes=batch.scene_structs())

    # -- growing the set, state files --
    def add_particles(self, x: np.ndarray, v: np.ndarray | None = None) -> None:
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, 3)
        if v is not None:
            v = np.ascontiguousarray(v, dtype=np.float32).reshape(-1, 3)
        self._check(self._lib.pbf_add_particles(self._ctx, _ptr(x), _ptr(v), x.shape[0]), "add_particles")

    def append(self, x: np.ndarray, x_star: np.ndarray, v: np.ndarray) -> None:
        """Particles::add (particles.h:184-199): append particles with their own
        x, x* and v (the multi-rank driver's arrivals and halos)."""
        x = np.ascontiguousarray(x, np.float32).reshape(-1, 3)
        if x.shape[0] == 0:
            return
        n0 = self.local_count()
        self.add_particles(x, np.ascontiguousarray(v, np.float32).reshape(-1, 3))
        xs = self.position_stars()
        xs[n0:] = x_star
        self.set_array(_abi.ARRAY_POSITION_STARS, xs)

    def remove(self, k: int) -> None:
        """Particles::remove (particles.h:146-154): drop the last k particles
        (reference order); x, x* and v of the others are kept (density, lambda
        and scratch are recomputed by the stages before they are read)."""
        if k <= 0:
            return
        keep = self.local_count() - int(k)
        if keep < 0:
            raise RuntimeError("remove: more particles than held")
        x, xs, v = self.positions()[:keep], self.position_stars()[:keep], self.velocities()[:keep]
        self.upload(x, v)
        if keep:
            self.set_array(_abi.ARRAY_POSITION_STARS, xs)

    def construct_fluid(self, fluid_min, fluid_max, velocity=(0.0, 0.0, 0.0)) -> int:
        """Particles::construct_fluid: append the lattice of the box; returns the count added."""
        mn, mx, vel = (C.c_float * 3)(*fluid_min), (C.c_float * 3)(*fluid_max), (C.c_float * 3)(*velocity)
        added = C.c_size_t()
        self._check(self._lib.pbf_construct_fluid(self._ctx, mn, mx, vel, C.byref(added)), "construct_fluid")
        return int(added.value)

    def emit(self, center, velocity=(0.0, 0.0, 0.0)) -> int:
        """The reference's emitter (distributor.h:357-369): construct_fluid on the
        box of extent 1.1 * spacing centred at `center`; call before each step."""
        sp = np.float32(self.params().particle_rest_spacing)
        ext = np.float32(1.1) * sp
        mn = [np.float32(c) - np.float32(0.5) * ext for c in center]
        mx = [m + ext for m in mn]
        return self.construct_fluid(mn, mx, velocity)

    def step_count(self) -> int:
        return int(self._lib.pbf_step_count(self._ctx))

    def save_state(self, path) -> None:
        self._check(self._lib.pbf_save_state(self._ctx, str(path).encode()), "save_state")

    def load_state(self, path) -> None:
        self._check(self._lib.pbf_load_state(self._ctx, str(path).encode()), "load_state")

    def scene_count(self) -> int:
        return int(self._lib.pbf_scene_count(self._ctx))

    def scene_stats(self, scene: int) -> dict:
        st = PbfStats()
        self._check(self._lib.pbf_scene_stats(self._ctx, int(scene), C.byref(st)), "scene_stats")
        return st.as_dict()

    def split(self, a: np.ndarray) -> list[np.ndarray]:
        """Per-scene views of an array indexed by particle (a batch's order)."""
        o = self.scene_offsets if self.scene_offsets is not None else np.array([0, len(a)])
        return [a[o[i]:o[i + 1]] for i in range(len(o) - 1)]

    # -- lifetime --
    def close(self) -> None:
        if self._ctx:
            self._lib.pbf_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, what: str) -> None:
        if rc != 0:
            raise RuntimeError(f"{what} failed ({rc}): {self._lib.pbf_last_error(self._ctx).decode()}")

    @property
    def ctx(self) -> C.c_void_p:
        return self._ctx

    # -- state --
    def local_count(self) -> int:
        return int(self._lib.pbf_count(self._ctx))

    def span(self) -> tuple[int, int]:
        return 0, self.local_count()

    def upload(self, x: np.ndarray, v: np.ndarray | None = None) -> None:
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, 3)
        if v is not None:
            v = np.ascontiguousarray(v, dtype=np.float32).reshape(-1, 3)
            assert v.shape == x.shape
        self._check(self._lib.pbf_upload(self._ctx, _ptr(x), _ptr(v), x.shape[0]), "upload")

    def download(self) -> dict:
        n = self.local_count()
        x = np.empty((n, 3), np.float32)
        v = np.empty((n, 3), np.float32)
        rho = np.empty(n, np.float32)
        lam = np.empty(n, np.float32)
        self._check(self._lib.pbf_download(self._ctx, _ptr(x), _ptr(v), _ptr(rho), _ptr(lam)), "download")
        return {"x": x, "v": v, "rho": rho, "lambda": lam}

    def get_array(self, which: int) -> np.ndarray:
        n = self.local_count()
        out = np.empty((n, 3) if which <= _abi.ARRAY_SCRATCH else (n,), np.float32)
        self._check(self._lib.pbf_get_array(self._ctx, which, _ptr(out)), "get_array")
        return out

    def set_array(self, which: int, values: np.ndarray) -> None:
        a = np.ascontiguousarray(values, dtype=np.float32)
        self._check(self._lib.pbf_set_array(self._ctx, which, _ptr(a)), "set_array")

    def positions(self) -> np.ndarray:
        return self.get_array(_abi.ARRAY_POSITIONS)

    def position_stars(self) -> np.ndarray:
        return self.get_array(_abi.ARRAY_POSITION_STARS)

    def velocities(self) -> np.ndarray:
        return self.get_array(_abi.ARRAY_VELOCITIES)

    def densities(self) -> np.ndarray:
        return self.get_array(_abi.ARRAY_DENSITIES)

    def lambdas(self) -> np.ndarray:
        return self.get_array(_abi.ARRAY_LAMBDAS)

    def scratch(self) -> np.ndarray:
        return self.get_array(_abi.ARRAY_SCRATCH)

    # -- stages (particles.h:256-487) --
    def apply_external_forces(self, span=None):
        self._check(self._lib.pbf_apply_external_forces(self._ctx, *(span or self.span())), "apply_external_forces")

    def predict_positions(self, span=None):
        self._check(self._lib.pbf_predict_positions(self._ctx, *(span or self.span())), "predict_positions")

    def find_neighbors(self, bin_span=None, fill_span=None):
        b = bin_span or self.span()
        f = fill_span or self.span()
        self._check(self._lib.pbf_find_neighbors(self._ctx, b[0], b[1], f[0], f[1]), "find_neighbors")

    def compute_densities(self, span=None):
        self._check(self._lib.pbf_compute_densities(self._ctx, *(span or self.span())), "compute_densities")

    def compute_pressure_lambdas(self, span=None):
        self._check(self._lib.pbf_compute_pressure_lambdas(self._ctx, *(span or self.span())),
                    "compute_pressure_lambdas")

    def compute_pressure_dps(self, span=None, substep: int = 0):
        s = span or self.span()
        self._check(self._lib.pbf_compute_pressure_dps(self._ctx, s[0], s[1], substep), "compute_pressure_dps")

    def update_position_stars(self, span=None):
        self._check(self._lib.pbf_update_position_stars(self._ctx, *(span or self.span())), "update_position_stars")

    def update_velocities(self, span=None):
        self._check(self._lib.pbf_update_velocities(self._ctx, *(span or self.span())), "update_velocities")

    def apply_surface_tension(self, color_span=None, st_span=None):
        c = color_span or self.span()
        s = st_span or self.span()
        self._check(self._lib.pbf_apply_surface_tension(self._ctx, c[0], c[1], s[0], s[1]), "apply_surface_tension")

    def apply_viscosity(self, span=None):
        self._check(self._lib.pbf_apply_viscosity(self._ctx, *(span or self.span())), "apply_viscosity")

    def compute_vorticity(self, span=None):
        self._check(self._lib.pbf_compute_vorticity(self._ctx, *(span or self.span())), "compute_vorticity")

    def apply_vorticity(self, span=None):
        self._check(self._lib.pbf_apply_vorticity(self._ctx, *(span or self.span())), "apply_vorticity")

    def update_positions(self, span=None):
        self._check(self._lib.pbf_update_positions(self._ctx, *(span or self.span())), "update_positions")

    # -- fused, graph-captured step (main.cpp:71-124) --
    def step(self, nsteps: int = 1) -> None:
        self._check(self._lib.pbf_step(self._ctx, int(nsteps)), "step")

    def sync(self) -> None:
        self._check(self._lib.pbf_sync(self._ctx), "sync")

    def stream_handle(self) -> int:
        """The cudaStream_t the context launches on (as an integer handle)."""
        out = C.c_void_p()
        self._check(self._lib.pbf_get_stream(self._ctx, C.byref(out)), "get_stream")
        return int(out.value or 0)

    def stats(self) -> dict:
        st = PbfStats()
        self._check(self._lib.pbf_stats(self._ctx, C.byref(st)), "stats")
        return st.as_dict()

    def neighbors(self, cap: int) -> tuple[np.ndarray, np.ndarray]:
        n = self.local_count()
        idx = np.empty((n, cap), np.int32)
        cnt = np.empty(n, np.int32)
        self._check(self._lib.pbf_get_neighbors(self._ctx, _ptr(idx), _ptr(cnt)), "get_neighbors")
        return idx, cnt

    def bins(self) -> dict:
        n = self.local_count()
        B = int(self._lib.pbf_num_bins(self._ctx))
        keys = np.empty(n, np.uint32)
        ids = np.empty(n, np.uint32)
        begin = np.empty(B, np.uint32)
        end = np.empty(B, np.uint32)
        self._check(self._lib.pbf_get_bins(self._ctx, _ptr(keys), _ptr(ids), _ptr(begin), _ptr(end)), "get_bins")
        return {"sorted_keys": keys, "sorted_ids": ids, "bin_begin": begin, "bin_end": end}

    def params(self) -> PbfParams:
        p = PbfParams()
        self._check(self._lib.pbf_get_params(self._ctx, C.byref(p)), "get_params")
        return p

    def set_params(self, p: PbfParams) -> None:
        self._check(self._lib.pbf_set_params(self._ctx, C.byref(p)), "set_params")

    # -- learned warm start (the per-particle MLP) --
    def mlp_init(self, seed: int = 0) -> None:
        self._check(self._lib.pbf_mlp_init(self._ctx, int(seed)), "mlp_init")

    def mlp_get(self) -> tuple[np.ndarray, np.ndarray]:
        params = np.empty(_abi.MLP_PARAMS, np.float32)
        norm = np.empty(_abi.MLP_NORM, np.float32)
        self._check(self._lib.pbf_mlp_get(self._ctx, _ptr(params), _ptr(norm)), "mlp_get")
        return params, norm

    def mlp_set(self, params: np.ndarray, norm: np.ndarray) -> None:
        params = np.ascontiguousarray(params, np.float32)
        norm = np.ascontiguousarray(norm, np.float32)
        assert params.size == _abi.MLP_PARAMS and norm.size == _abi.MLP_NORM
        self._check(self._lib.pbf_mlp_set(self._ctx, _ptr(params), _ptr(norm)), "mlp_set")

    def set_recording(self, on: bool) -> None:
        self._check(self._lib.pbf_set_recording(self._ctx, int(on)), "set_recording")

    def training_data(self) -> tuple[np.ndarray, np.ndarray]:
        n = self.local_count()
        f = np.empty((n, _abi.MLP_FEATURES), np.float32)
        lab = np.empty(n, np.float32)
        self._check(self._lib.pbf_get_training_data(self._ctx, _ptr(f), _ptr(lab)), "get_training_data")
        return f, lab

    def mlp_train(self, adam_steps: int, batch: int, lr: float, seed: int = 0) -> float:
        loss = C.c_float()
        self._check(self._lib.pbf_mlp_train(self._ctx, int(adam_steps), int(batch), float(lr), int(seed),
                                            C.byref(loss)), "mlp_train")
        return float(loss.value)

    def mlp_gradients(self, features: np.ndarray, targets: np.ndarray) -> tuple[np.ndarray, float]:
        f = np.ascontiguousarray(features, np.float32)
        t = np.ascontiguousarray(targets, np.float32)
        g = np.empty(_abi.MLP_PARAMS, np.float32)
        loss = C.c_float()
        self._check(self._lib.pbf_mlp_gradients(self._ctx, _ptr(f), _ptr(t), t.size, _ptr(g), C.byref(loss)),
                    "mlp_gradients")
        return g, float(loss.value)

    def mlp_predict(self, features: np.ndarray) -> np.ndarray:
        f = np.ascontiguousarray(features, np.float32)
        y = np.empty(f.shape[0], np.float32)
        self._check(self._lib.pbf_mlp_predict(self._ctx, _ptr(f), f.shape[0], _ptr(y)), "mlp_predict")
        return y

    def selftest_mlp_wait_timeout(self) -> int:
        """Run the network kernel with nothing arriving on its completion
        barrier (pbf_selftest_mlp_wait_timeout); returns the flags it raised."""
        out = C.c_uint32(0)
        self._check(self._lib.pbf_selftest_mlp_wait_timeout(self._ctx, C.byref(out)), "selftest_mlp_wait_timeout")
        return int(out.value)

    def set_persistent(self, enable: bool = True) -> None:
        """Run each step's list fill and gather passes as one persistent
        launch, each scene of the batch at its own pace (pbf_set_persistent)."""
        self._check(self._lib.pbf_set_persistent(self._ctx, int(enable)), "set_persistent")

    def selftest_persistent_wait_timeout(self) -> int:
        """Run the persistent step's scheduler on a dependency that is never
        met (pbf_selftest_persistent_wait_timeout); returns the flags it raised."""
        out = C.c_uint32(0)
        self._check(self._lib.pbf_selftest_persistent_wait_timeout(self._ctx, C.byref(out)),
                    "selftest_persistent_wait_timeout")
        return int(out.value)

    # -- instrumentation --
    def set_timing(self, on: bool) -> None:
        self._check(self._lib.pbf_set_timing(self._ctx, int(on)), "set_timing")

    def reset_timing(self) -> None:
        self._check(self._lib.pbf_reset_timing(self._ctx), "reset_timing")

    def kernel_times(self) -> dict:
        k = 64
        names = (C.c_char_p * k)()
        launches = (C.c_int64 * k)()
        total = (C.c_double * k)()
        nk = C.c_int()
        self._check(self._lib.pbf_kernel_times(self._ctx, k, names, launches, total, C.byref(nk)), "kernel_times")
        return {names[i].decode(): {"launches": int(launches[i]), "total_ms": float(total[i])} for i in range(nk.value)}

    def launches_per_step(self) -> int:
        out = C.c_int64()
        self._check(self._lib.pbf_launches_per_step(self._ctx, C.byref(out)), "launches_per_step")
        return int(out.value)

    # launch shapes of the fast gather kernels: {family: (lanes, block)}
    def tuning(self) -> dict:
        t = _abi.PbfTuning()
        self._check(self._lib.pbf_get_tuning(self._ctx, C.byref(t)), "get_tuning")
        return t.as_dict()

    def set_tuning(self, shapes: dict) -> None:
        """{family: (lanes, block) or (lanes, block, staged)}; unnamed families keep theirs."""
        t = _abi.PbfTuning()
        cur = self.tuning()
        cur.update({f: tuple(v) + (0,) * (3 - len(v)) for f, v in shapes.items()})
        for i, f in enumerate(_abi.TUNE_FAMILIES):
            t.lanes[i], t.block[i], t.staged[i] = cur[f]
        self._check(self._lib.pbf_set_tuning(self._ctx, C.byref(t)), "set_tuning")

    def autotune(self, steps: int = 3) -> tuple[dict, dict]:
        """Time every candidate shape on `steps` steps of the current state
        (restored afterwards), apply the fastest per family; returns (chosen,
        {(lanes, block, staged): {family: ms per step}})."""
        t = _abi.PbfTuning()
        nc, nf = len(_abi.TUNE_CANDIDATES), len(_abi.TUNE_FAMILIES)
        ms = (C.c_double * (nc * nf))()
        self._check(self._lib.pbf_autotune(self._ctx, int(steps), C.byref(t), ms), "autotune")
        table = {cand: {f: float(ms[c * nf + i]) for i, f in enumerate(_abi.TUNE_FAMILIES)}
                 for c, cand in enumerate(_abi.TUNE_CANDIDATES)}
        return t.as_dict(), table


class SceneGroup:
    """Independent contexts (one scene each) advanced together by one graph
    launch (pbf_group_*): every scene's step chain is a child graph of the
    launch, with no dependency between scenes, so each advances at its own
    pace; each context's results are its own `step` results, bit for bit."""

    def __init__(self, contexts):
        self._lib = lib()
        self.contexts = list(contexts)
        arr = (C.c_void_p * len(self.contexts))(*[c.ctx.value for c in self.contexts])
        self._g = C.c_void_p()
        rc = self._lib.pbf_group_create(arr, len(self.contexts), C.byref(self._g))
        if rc != 0:
            raise RuntimeError(f"pbf_group_create failed ({rc}): {self._lib.pbf_last_error(None).decode()}")

    def step(self, nsteps: int = 1) -> None:
        rc = self._lib.pbf_group_step(self._g, int(nsteps))
        if rc != 0:
            raise RuntimeError(f"pbf_group_step failed ({rc}): {self._lib.pbf_last_error(None).decode()}")

    def sync(self) -> None:
        if self._lib.pbf_group_sync(self._g) != 0:
            raise RuntimeError(self._lib.pbf_last_error(None).decode())

    def stream_handle(self) -> int:
        out = C.c_void_p()
        self._lib.pbf_group_get_stream(self._g, C.byref(out))
        return out.value or 0

    def close(self) -> None:
        if self._g:
            self._lib.pbf_group_destroy(self._g)
            self._g = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        self.close()
