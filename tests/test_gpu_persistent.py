"""The persistent step on batches of scenes (pbf_set_persistent).

One launch runs all the gather passes of a step, blocks taking
(pass, tile) tasks from a queue and each tile waiting only for the previous
pass in the scenes it covers.  The bar: every particle array and every list
bit for bit those of the launch-per-pass step at the same launch shapes, over
many steps (a missed dependency or a stale read shows as a difference); the
bounded wait gives up cleanly; the configurations it does not run are
refused.
"""
from __future__ import annotations

import numpy as np
import pytest

from pbf_b200 import Particles, _abi, make_batch, make_scene

pytestmark = pytest.mark.gpu
ARRAYS = (_abi.ARRAY_POSITIONS, _abi.ARRAY_POSITION_STARS, _abi.ARRAY_VELOCITIES, _abi.ARRAY_SCRATCH,
          _abi.ARRAY_DENSITIES, _abi.ARRAY_LAMBDAS)
# the persistent step's fixed shapes, given to the launch-per-pass step it is compared with
SHAPES = {"density": (2, 128, 0), "delta_p": (2, 128, 0), "viscosity": (2, 128, 0), "vorticity": (4, 128, 0),
          "apply_vorticity": (2, 128, 0)}


def small_batch(**kw):
    return make_batch(scenes=6, seed=11, n_min=512, n_max=20000, name="batch_small", **kw)


def pair(batch):
    a = Particles.batch(batch)
    b = Particles.batch(batch)
    for g in (a, b):
        g.set_tuning(SHAPES)
        g.upload(batch.positions())
    b.set_persistent(True)
    return a, b


def assert_same(a, b):
    for w in ARRAYS:
        assert np.array_equal(a.get_array(w), b.get_array(w)), w
    ia, ca = a.neighbors(60)
    ib, cb = b.neighbors(60)
    assert np.array_equal(ca, cb)
    assert np.array_equal(ia, ib)


@pytest.mark.parametrize("steps", [1, 60])
def test_persistent_step_equals_the_launch_per_pass_step(steps):
    """Graph-captured steps: 60 of them take the small batch's narrow scenes
    into their collapse (crowded bins, run-walked fills)."""
    a, b = pair(small_batch())
    with a, b:
        a.step(steps)
        b.step(steps)
        assert_same(a, b)
        assert b.stats()["error_flags"] == 0


def test_eager_persistent_steps_launch_one_kernel_for_the_passes():
    a, b = pair(small_batch())
    with a, b:
        b.set_timing(True)
        b.step(3)
        kt = b.kernel_times()
        b.set_timing(False)
        assert kt["persistent_step"]["launches"] == 3
        assert kt["fill_neighbors"]["launches"] == 3
        for k in ("density_lambda", "dp_update", "viscosity", "vorticity", "apply_vorticity", "viscosity_final"):
            assert k not in kt, k
        assert sum(v["launches"] for v in kt.values()) == 3 * b.launches_per_step()
        a.step(3)
        assert_same(a, b)


def test_persistent_wait_gives_up_and_the_context_stays_usable():
    batch = small_batch()
    a, b = pair(batch)
    with a, b:
        flags = b.selftest_persistent_wait_timeout()
        assert flags & _abi.PBF_FLAG_WAIT_TIMEOUT
        a.step(4)
        b.step(4)
        assert_same(a, b)
        assert b.stats()["error_flags"] == 0  # the self-test raised its own status word, not the context's


def test_persistent_step_rules():
    sc = make_scene("dam_2k")
    with Particles(sc.params(), sc.n) as g:
        with pytest.raises(RuntimeError, match="batches of scenes"):
            g.set_persistent(True)
    with Particles.batch(small_batch(exact_math=1)) as g:
        with pytest.raises(RuntimeError, match="fast math"):
            g.set_persistent(True)
    a, b = pair(small_batch())
    with a, b:
        assert b.launches_per_step() < a.launches_per_step()
        b.set_persistent(False)
        assert b.launches_per_step() == a.launches_per_step()
