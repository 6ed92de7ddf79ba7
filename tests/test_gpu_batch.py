"""Batched scenes on the GPU (pbf_create_batch).

The bar: a batch advances every scene exactly as a context created for that
scene alone with the same launch shapes - bins, lists and every particle
array bit for bit, in exact and in fast math - and, through the single-scene
parity, as the oracle does.  Plus the batch's bookkeeping: global bin keys,
per-scene statistics, the count check, the autotuner and the learned solver
on a batch, and the 64-scene workload itself.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle.oracle import ARRAY_POSITIONS, ARRAY_VELOCITIES, OracleSim
from pbf_b200 import Particles, _abi, make_batch

pytestmark = pytest.mark.gpu
ARRAYS = (_abi.ARRAY_POSITIONS, _abi.ARRAY_POSITION_STARS, _abi.ARRAY_VELOCITIES, _abi.ARRAY_SCRATCH,
          _abi.ARRAY_DENSITIES, _abi.ARRAY_LAMBDAS)


def small_batch(**kw):
    return make_batch(scenes=6, seed=11, n_min=512, n_max=20000, name="batch_small", **kw)


def run_batch(batch, steps):
    g = Particles.batch(batch)
    g.upload(batch.positions())
    g.step(steps)
    return g


def run_solo(scene, steps):
    g = Particles(scene.params(), scene.n)
    g.upload(scene.positions())
    g.step(steps)
    return g


@pytest.mark.parametrize("exact", [1, 0])
def test_batch_equals_independent_runs_bitwise(exact):
    b = small_batch(exact_math=exact)
    g = run_batch(b, 12)
    assert g.scene_count() == len(b.scenes)
    per = {w: g.split(g.get_array(w)) for w in ARRAYS}
    idx, cnt = g.neighbors(60)
    o = b.offsets
    for i, sc in enumerate(b.scenes):
        s = run_solo(sc, 12)
        for w in ARRAYS:
            assert np.array_equal(per[w][i], s.get_array(w)), (i, w)
        si, sn = s.neighbors(60)
        assert np.array_equal(cnt[o[i]:o[i + 1]], sn), i
        bi = idx[o[i]:o[i + 1]]
        assert np.array_equal(np.where(bi >= 0, bi - o[i], -1), si), i
        a, r = g.scene_stats(i), s.stats()
        for k in ("mean_density_error", "max_density_error", "kinetic_energy", "mean_neighbors"):
            assert a[k] == pytest.approx(r[k], rel=1e-9, abs=1e-12), (i, k)
        assert a["cap_hits"] == r["cap_hits"] and a["n"] == sc.n
    assert g.stats()["error_flags"] == 0


def test_batch_scene_against_the_oracle():
    b = small_batch(exact_math=1)
    g = run_batch(b, 4)
    i = int(np.argmin(b.counts))
    sc = b.scenes[i]
    o = OracleSim(sc.params(), sc.n)
    o.set_state(sc.positions())
    o.step(4)
    for w in (ARRAY_POSITIONS, ARRAY_VELOCITIES):
        assert np.array_equal(g.split(g.get_array(w))[i], o.get(w)), w


def test_batch_bins_are_in_global_key_space():
    b = small_batch()
    g = run_batch(b, 1)
    bins = g.bins()
    keys = bins["sorted_keys"]
    assert np.all(np.diff(keys.astype(np.int64)) >= 0)
    ids = bins["sorted_ids"].astype(np.int64)
    o = b.offsets
    # every scene's particles form one run of the sorted order, in scene order
    scene_of = np.searchsorted(o, ids, side="right") - 1
    assert np.all(np.diff(scene_of) >= 0)
    for i in range(len(b.scenes)):
        assert np.array_equal(np.flatnonzero(scene_of == i), np.arange(o[i], o[i + 1]))


def test_batch_upload_takes_exactly_the_scenes_particles():
    b = small_batch()
    g = Particles.batch(b)
    x = b.positions()
    with pytest.raises(RuntimeError, match="takes exactly"):
        g.upload(x[:-1])
    g.upload(x)
    with pytest.raises(RuntimeError, match="out of"):
        g.scene_stats(len(b.scenes))


def test_batch_autotune_and_learned_solver():
    b = small_batch(lambda_epsilon=1.0)
    g = run_batch(b, 3)
    before = g.positions()
    chosen, table = g.autotune(1)
    assert np.array_equal(g.positions(), before)
    g.step(2)
    assert g.stats()["error_flags"] == 0
    lb = small_batch(lambda_epsilon=1.0, solver=1, max_iterations=4, residual_tol=0.01)
    h = Particles.batch(lb)
    h.mlp_init(5)
    h.upload(lb.positions())
    h.step(5)
    st = h.stats()
    assert st["error_flags"] == 0 and 1 <= st["solver_iterations"] <= 4
    assert np.isfinite(h.positions()).all()


def test_batch_64_scenes_workload():
    b = make_batch()
    g = run_batch(b, 10)
    st = g.stats()
    assert st["error_flags"] == 0 and st["n"] == b.n
    x = g.positions()
    assert np.isfinite(x).all()
    for i, sc in enumerate(b.scenes):  # every particle stays in its own scene's box
        xi = g.split(x)[i]
        assert (xi >= 0).all() and (xi <= np.array(sc.box_max, np.float32)).all(), i
    # two scenes against their own contexts, bit for bit
    for i in (int(np.argmin(b.counts)), int(np.argmax(b.counts))):
        s = run_solo(b.scenes[i], 10)
        assert np.array_equal(g.split(x)[i], s.positions()), i


def test_scene_group_equals_each_context_stepping_alone():
    """A scene group (pbf_group_*) advances its contexts by one graph launch
    whose members are independent child graphs: every context ends exactly
    where its own pbf_step would put it (graph cached per step count and
    rebuilt after a member changes its particle count)."""
    from pbf_b200 import SceneGroup
    b = small_batch()
    ctxs = []
    for sc in b.scenes:
        c = Particles(sc.params(), sc.n)
        c.upload(sc.positions())
        ctxs.append(c)
    with SceneGroup(ctxs) as grp:
        grp.step(5)
        grp.step(5)     # the cached 5-step graph again
        grp.step(2)
        grp.sync()
        for sc, c in zip(b.scenes, ctxs):
            s = run_solo(sc, 12)
            for w in ARRAYS:
                assert np.array_equal(c.get_array(w), s.get_array(w)), (sc.name, w)
            assert c.step_count() == 12
        # a member with a new particle count: the group rebuilds its graph
        sc0 = b.scenes[0]
        ctxs[0].upload(sc0.positions()[: sc0.n // 2])
        grp.step(5)
        s = Particles(sc0.params(), sc0.n)
        s.upload(sc0.positions()[: sc0.n // 2])
        s.step(5)
        assert np.array_equal(ctxs[0].get_array(_abi.ARRAY_POSITIONS), s.get_array(_abi.ARRAY_POSITIONS))
    for c in ctxs:
        assert c.stats()["error_flags"] == 0
        c.close()
