"""The x-slab decomposition (pbf_b200.slabs.SlabDistributor) on CPU ranks.

Every test runs 2 or 3 gloo ranks as spawned processes, each driving the
reference's own build (oracle/ref_engine.py) through the distributor, so
the decomposition is checked without a GPU:
  - slab bounds, particle counts and the interior/edge/halo spans after a
    domain sync, and the counts after a particle crosses a slab boundary:
    the scenarios of the reference's Simulation/Tests/Parallel/
    distributor_tests.cpp:33-558 on its distributor_test.ini scene (a 9x4x1
    lattice at spacing 1 in an 11x5x2 box, edge width 1.2), restated;
  - a dam break advanced 8 steps on 2 and on 3 slabs equals the same dam
    advanced by the reference on one rank, particle by particle, within the
    tolerance that the changed particle order allows (neighbour summation
    order and the reference's in-place XSPH order), on a lattice whose
    neighbour lists stay below the cap (so the cap's truncation order does
    not enter).
"""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
pytestmark = pytest.mark.skipif(not (ROOT / "oracle" / "_ref" / "libpbf_ref_serial.so").exists(),
                                reason="the reference build (oracle/_ref) is absent")


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_entry(rank, world, port, q, fn_name, args):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    for p in (ROOT, ROOT / "sph-cpp_b200"):
        sys.path.insert(0, str(p))
    import datetime

    import torch.distributed as dist
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    try:
        import test_slabs_gloo as mod
        q.put((rank, getattr(mod, fn_name)(rank, world, *args)))
    except Exception as e:  # reported to the parent, never a hang
        q.put((rank, {"error": repr(e)}))
    finally:
        dist.destroy_process_group()


def _run(world: int, fn_name: str, *args) -> dict:
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    env = os.environ.get("PYTHONPATH", "")
    os.environ["PYTHONPATH"] = os.pathsep.join([str(ROOT / "tests"), str(ROOT), str(ROOT / "sph-cpp_b200"), env])
    try:
        procs = [ctx.Process(target=_rank_entry, args=(r, world, port, q, fn_name, args)) for r in range(world)]
        for p in procs:
            p.start()
        out = dict(q.get(timeout=300) for _ in range(world))
        for p in procs:
            p.join(timeout=60)
            assert p.exitcode == 0
    finally:
        os.environ["PYTHONPATH"] = env
    for r, v in out.items():
        assert not (isinstance(v, dict) and "error" in v), (r, v)
    return out


# ---------------------------------------------------------------- rank bodies
def _dist_scene():
    from oracle.ref_scene import Workload
    # distributor_test.ini: InitialFluid [0,9]x[0,4]x[0,1], Boundary [0,11]x[0,5]x[0,2], spacing 1, h 1
    return Workload("distributor_test", (9, 4, 1), (11.0, 5.0, 2.0), 3, h=1.0, spacing=1.0, jitter=0.0)


def _spans(d) -> dict:
    return {"domain": list(d.domain), "resident": d.resident_span(), "local": d.local_span(),
            "edge": d.edge_span(), "halo": d.halo_span(), "interior": d.interior_span(),
            "counts": (d.resident_count(), d.edge_count(), d.halo_count(), d.interior_count(), d.local_count())}


def rank_initialize_and_sync(rank, world, move_first: bool):
    from oracle.ref_engine import POSITION_STARS, RefEngine
    from pbf_b200.slabs import SlabDistributor, Transport
    w = _dist_scene()
    eng = RefEngine(w, capacity=100, rest_density=1.0)
    t = Transport()
    d = SlabDistributor(t, edge_width=1.2 * w.h)
    out = {"left": d.domain_to_left(), "right": d.domain_to_right(), "first": d.is_first_domain(),
           "last": d.is_last_domain()}
    d.set_domain_bounds(0.0, 9.0, 0.0, 11.0)
    d.distribute_fluid(eng, (0.0, 0.0, 0.0), (9.0, 4.0, 1.0), 1.0)
    out["initial_local"] = eng.local_count()
    out["initial_domain"] = list(d.domain)
    if move_first and rank == 0:
        xs = eng.get_array(POSITION_STARS)
        xs[0, 0] = 3.1
        eng.set_array(POSITION_STARS, xs)
    d.invalidate_halo(eng)
    d.domain_sync(eng)
    out.update(_spans(d))
    out["engine_local"] = eng.local_count()
    out["global_resident"] = d.global_resident_count()
    eng.close()
    return out


def _dam():
    from oracle.ref_scene import Workload
    # spacing 0.55h: about 43 neighbours per particle, below the reference's cap of 60
    return Workload("dam_slabs", (16, 12, 8), (14.0, 13.0, 13.0), 3, spacing=0.55, seed=99)


# the whole block starts moving toward +x, so particles cross the slab bounds
V0 = np.array([4.0, 0.0, 0.0], np.float32)


def _dam_state():
    from oracle.ref_scene import RefRun, rest_density
    w = _dam()
    with RefRun(w) as run:
        x = run.get(0)
    return w, x, rest_density(w)


def rank_dam(rank, world, steps):
    from oracle.ref_engine import POSITIONS, VELOCITIES, RefEngine
    from pbf_b200.slabs import SlabDistributor, Transport
    w, x, rho0 = _dam_state()
    eng = RefEngine(w, capacity=x.shape[0], rest_density=rho0)
    t = Transport()
    d = SlabDistributor(t, edge_width=1.2 * w.h)
    d.set_domain_bounds(0.0, w.fluid_extent[0], 0.0, w.box_max[0])
    b, e = np.float32(d.domain[0]), np.float32(d.domain[1])
    mine = (x[:, 0] >= b) & ((x[:, 0] < e) if not d.is_last_domain() else (x[:, 0] <= e))
    ids = np.nonzero(mine)[0]
    eng.append(x[ids], x[ids], np.broadcast_to(V0, x[ids].shape))
    d.adopt(eng, ids)
    halos = []
    for _ in range(steps):
        d.step(eng, w.solve_steps)
        c = d.last_sync
        halos.append((c.halo_left, c.halo_right, c.oob_left, c.oob_right))
    R = d.resident_count()
    res = {"ids": d.ids[:R].copy(), "x": eng.get_array(POSITIONS)[:R], "v": eng.get_array(VELOCITIES)[:R],
           "halos": halos, "domain": list(d.domain)}
    eng.close()
    return res


# ---------------------------------------------------------------- tests
def test_three_slabs_bounds_counts_and_spans():
    """distributor_tests.cpp:33-110 (neighbours), :80-170 (bounds and counts)
    and :172-300 (spans after a domain sync), 3D, 3 ranks."""
    out = _run(3, "rank_initialize_and_sync", False)
    assert [out[r]["left"] for r in range(3)] == [None, 0, 1]
    assert [out[r]["right"] for r in range(3)] == [1, 2, None]
    assert out[0]["first"] and out[2]["last"] and not out[1]["first"] and not out[1]["last"]
    assert [out[r]["initial_domain"] for r in range(3)] == [[0.0, 3.0], [3.0, 6.0], [6.0, 11.0]]
    assert [out[r]["initial_local"] for r in range(3)] == [12, 12, 12]
    assert [out[r]["local"] for r in range(3)] == [(0, 16), (0, 20), (0, 16)]
    assert all(out[r]["resident"] == (0, 12) for r in range(3))
    assert [out[r]["edge"] for r in range(3)] == [(4, 12), (4, 12), (8, 12)]
    assert [out[r]["halo"] for r in range(3)] == [(12, 16), (12, 20), (12, 16)]
    assert [out[r]["interior"] for r in range(3)] == [(0, 4), (0, 4), (0, 8)]
    assert [out[r]["engine_local"] for r in range(3)] == [16, 20, 16]
    assert all(out[r]["global_resident"] == 36 for r in range(3))


def test_three_slabs_out_of_bounds_migration():
    """distributor_tests.cpp:302-558: rank 0's first particle moved to
    x* = 3.1 migrates to rank 1 at the domain sync."""
    out = _run(3, "rank_initialize_and_sync", True)
    assert [out[r]["local"] for r in range(3)] == [(0, 16), (0, 21), (0, 16)]
    assert [out[r]["resident"] for r in range(3)] == [(0, 11), (0, 13), (0, 12)]
    assert [out[r]["edge"] for r in range(3)] == [(4, 11), (4, 13), (8, 12)]
    assert [out[r]["halo"] for r in range(3)] == [(11, 16), (13, 21), (12, 16)]
    assert [out[r]["interior"] for r in range(3)] == [(0, 4), (0, 4), (0, 8)]
    assert all(out[r]["global_resident"] == 36 for r in range(3))


def test_two_slabs_bounds_and_counts():
    """The same scene on 2 ranks: slabs [0, 4.5] and [4.5, 11]; the
    lattice spacing is kept across the boundary (distribute_fluid,
    distributor.h:318-353): 4 columns on rank 0, 5 on rank 1."""
    out = _run(2, "rank_initialize_and_sync", False)
    assert [out[r]["initial_domain"] for r in range(2)] == [[0.0, 4.5], [4.5, 11.0]]
    assert [out[r]["initial_local"] for r in range(2)] == [16, 20]
    # edges (within 1.2 of a slab bound): rank 0's columns 0.5 and 3.5,
    # rank 1's columns 4.5 and 5.5; halos are the other rank's edges next to it
    assert out[0]["edge"] == (8, 16) and out[1]["edge"] == (12, 20)
    assert out[0]["halo"] == (16, 24) and out[1]["halo"] == (20, 24)


@pytest.mark.parametrize("world", [2, 3])
def test_slabs_advance_the_dam_as_one_rank_does(world):
    """8 steps of a 1,536-particle dam, the block launched toward +x at 4
    units/s, on `world` slabs (particles migrate and halos refresh every
    iteration) against the reference's single-rank run of the same state: every particle ends within 2e-5 of the box of its
    single-rank position, and within 1e-3 of the largest speed in velocity."""
    import ctypes as C

    from oracle.ref_scene import ref_params
    from oracle.reflib import ref_lib
    steps = 8
    out = _run(world, "rank_dam", steps)
    ids = np.concatenate([out[r]["ids"] for r in range(world)])
    x = np.concatenate([out[r]["x"] for r in range(world)])
    v = np.concatenate([out[r]["v"] for r in range(world)])
    w, x0, rho0 = _dam_state()
    n = x0.shape[0]
    assert np.array_equal(np.sort(ids), np.arange(n))  # every particle on exactly one slab
    assert sum(h[0] + h[1] for r in range(world) for h in out[r]["halos"]) > 0
    assert sum(h[2] + h[3] for r in range(world) for h in out[r]["halos"]) > 0  # particles migrated
    lib = ref_lib(serial=True)
    rp = ref_params(w, capacity=n, rest_density=rho0)
    h = lib.ref_create(C.byref(rp))
    try:
        v0 = np.ascontiguousarray(np.broadcast_to(V0, x0.shape))
        assert lib.ref_add(h, x0.ctypes.data_as(C.c_void_p), v0.ctypes.data_as(C.c_void_p), n) == 0
        assert lib.ref_step(h, steps) == 0
        xr = np.empty_like(x0)
        vr = np.empty_like(x0)
        lib.ref_get_vec(h, 0, xr.ctypes.data_as(C.c_void_p))
        lib.ref_get_vec(h, 2, vr.ctypes.data_as(C.c_void_p))
        idx = np.empty((n, 60), np.int32)
        cnt = np.empty(n, np.int32)
        lib.ref_get_neighbors(h, idx.ctypes.data_as(C.c_void_p), cnt.ctypes.data_as(C.c_void_p), 60)
    finally:
        lib.ref_destroy(h)
    assert cnt.max() < 60  # the cap never truncates, so list order alone differs
    order = np.argsort(ids)
    dx = np.abs(x[order] - xr).max()
    dv = np.abs(v[order] - vr).max()
    assert dx <= 2e-5 * max(w.box_max), dx
    assert dv <= 1e-3 * np.abs(vr).max(), (dv, np.abs(vr).max())
