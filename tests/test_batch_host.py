"""Batched scenes without a GPU: the seeded batch generator (64 dam breaks,
counts log-uniform in [4096, 262144], lattice blocks of aspect ratio in
[0.5, 2], each in its own box 1.5x its extent) and the batch constructor's
validation, which runs before any device is touched."""
from __future__ import annotations

import ctypes as C

import numpy as np

from pbf_b200 import _abi, make_batch


def test_generator_follows_the_batch_workload():
    b = make_batch()
    assert len(b.scenes) == 64
    counts = np.array(b.counts)
    assert counts.min() >= 4096 and counts.max() <= 262144
    assert b.n == counts.sum() and b.offsets[-1] == b.n
    # log-uniform: the log-counts spread over the whole range
    lo, hi = np.log(4096), np.log(262144)
    u = (np.log(counts) - lo) / (hi - lo)
    assert u.min() < 0.15 and u.max() > 0.85 and 0.3 < np.median(u) < 0.7
    for s in b.scenes:
        nx, ny, nz = s.lattice
        assert 0.45 <= ny / nx <= 2.1 and 0.45 <= nz / nx <= 2.1
        for a in range(3):
            ext = s.lattice[a] * s.spacing
            assert 1.5 * ext <= s.box_max[a] <= 1.5 * ext + 0.2
            assert abs(s.box_max[a] / 1.2 - round(s.box_max[a] / 1.2)) > 1e-4  # off the bin spacing
        assert s.fluid_min == (0.0, 0.0, 0.0)
    # seeded: the same batch again, another seed another batch
    assert make_batch().counts == b.counts
    assert make_batch(seed=7).counts != b.counts
    assert len({s.seed for s in b.scenes}) == 64


def test_every_scene_has_a_valid_grid():
    b = make_batch()
    lib = _abi.load()
    for s in b.scenes:
        p = s.params()
        d = (C.c_int64 * 3)()
        assert lib.pbf_grid_dims(C.byref(p), d) == 0
        assert all(d[a] >= 3 for a in range(3))


def test_create_batch_validates_every_scene_first():
    lib = _abi.load()
    b = make_batch(scenes=4, n_max=8192)
    p = b.params()
    ctx = C.c_void_p()
    sc = b.scene_structs()
    bad = (_abi.PbfScene * 4)(*sc)
    bad[2].boundary_min[1] = -1.0
    assert lib.pbf_create_batch(C.byref(p), bad, 4, C.byref(ctx)) == _abi.PBF_ERR_PARAMS
    msg = lib.pbf_create_error()
    assert b"scene 2" in msg and b"boundary min" in msg
    bad = (_abi.PbfScene * 4)(*sc)
    bad[3].boundary_min[1] = 2.0  # grid sized by the extent but hashed from 0: the far wall's bins leave it
    assert lib.pbf_create_batch(C.byref(p), bad, 4, C.byref(ctx)) == _abi.PBF_ERR_PARAMS
    assert b"scene 3" in lib.pbf_create_error()
    assert lib.pbf_create_batch(C.byref(p), (_abi.PbfScene * 4)(*sc), 0, C.byref(ctx)) == _abi.PBF_ERR_ARG
    empty = (_abi.PbfScene * 1)()
    empty[0].boundary_max[:] = [10.0, 10.0, 10.0]
    assert lib.pbf_create_batch(C.byref(p), empty, 1, C.byref(ctx)) == _abi.PBF_ERR_ARG
