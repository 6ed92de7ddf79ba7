"""Launch shapes of the fast gather kernels (lanes per particle x threads per
block) and the autotuner that picks them.

A shape changes only the order of the floating-point sums inside one
particle, so every shape must meet the fast path's bars: lists bit-exact,
positions after one step within 1e-5 (relative to the box) of the
reference's golden output, 100-step statistics within the bars the default
shape meets.  The autotuner must hand back the particle state it was given.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from pbf_b200 import Particles, _abi, make_scene

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
REL_TOL = 1e-5
# bars of the 100-step averaged statistics at eps 600: twice the reference's
# own run-to-run spread, as for the default shape against the oracle, except
# the max.  The max density error is set by how many particles pile exactly
# into a wall corner, a discrete chaotic count: averaged over steps 81-100 of
# the 65k dam, four launch shapes of the same build gave 3.67-3.93 (7%).  It
# has the 10% bar it has against the reference's OpenMP build.
BARS = {"mean_density_error": 0.014, "max_density_error": 0.10, "kinetic_energy": 0.02}


# the library's default shapes (include/pbf.h)
DEFAULT = {"density": (2, 128, 0), "delta_p": (2, 128, 0), "viscosity": (2, 256, 0), "vorticity": (4, 256, 0),
           "apply_vorticity": (2, 256, 0)}


def _all_families(shape):
    return {f: tuple(shape) + (0,) * (3 - len(shape)) for f in _abi.TUNE_FAMILIES}


@pytest.mark.parametrize("shape", _abi.TUNE_CANDIDATES)
def test_every_shape_matches_reference_golden(shape):
    gd = np.load(GOLDEN / "dam_2k_step1.npz")
    sc = make_scene("dam_2k")
    g = Particles(sc.params(), sc.n)
    g.set_tuning(_all_families(shape))
    assert g.tuning() == _all_families(shape)
    g.upload(gd["x0"])
    g.step(1)
    np.testing.assert_allclose(g.positions(), gd["x1"], rtol=0, atol=REL_TOL * max(sc.box_max))
    idx, cnt = g.neighbors(60)
    assert np.array_equal(cnt, gd["cnt"].astype(np.int32))
    mask = np.arange(60)[None, :] < cnt[:, None]
    assert np.array_equal(np.where(mask, idx, -1), np.where(mask, gd["nbr"].astype(np.int32), -1))


@pytest.mark.parametrize("shape", _abi.TUNE_CANDIDATES)
def test_every_shape_reads_only_live_list_entries(shape):
    """The list buffer keeps entries past each particle's count from earlier
    fills (other states, other particles).  A step from a given state must not
    depend on them: a context whose list buffer holds a different history
    steps bit for bit as a fresh one, under every launch shape."""
    sc = make_scene("dam_8k")
    p = sc.params()
    with Particles(p, sc.n) as w:
        w.upload(sc.positions())
        w.step(40)  # a later state, with long lists in the crowded floor layer
        d = w.download()
    with Particles(p, sc.n) as a, Particles(p, sc.n) as b:
        for g in (a, b):
            g.set_tuning(_all_families(shape))
        a.upload(sc.positions())
        a.step(3)  # the list buffer now holds the early state's lists
        a.upload(d["x"], d["v"])
        b.upload(d["x"], d["v"])
        a.step(1)
        b.step(1)
        assert np.array_equal(a.positions(), b.positions())
        assert np.array_equal(a.velocities(), b.velocities())


def _averaged(g, steps=100, window=20):
    g.step(steps - window)
    acc = []
    for _ in range(window):
        g.step(1)
        st = g.stats()
        acc.append([st[k] for k in BARS])
    return dict(zip(BARS, np.mean(acc, axis=0)))


def test_shapes_agree_on_100_step_statistics():
    sc = make_scene("dam_65k")
    x = sc.positions()
    out = {}
    for shape in ((4, 128, 1), (8, 256, 0)):
        g = Particles(sc.params(), sc.n)
        g.set_tuning(_all_families(shape))
        g.upload(x)
        out[shape] = _averaged(g)
        assert g.stats()["error_flags"] == 0
    a, b = out[(4, 128, 1)], out[(8, 256, 0)]
    for k in BARS:
        assert a[k] == pytest.approx(b[k], rel=BARS[k]), (k, a[k], b[k])


def test_set_tuning_rejects_unsupported_shapes():
    sc = make_scene("dam_2k")
    g = Particles(sc.params(), sc.n)
    for bad in ((16, 256), (8, 512), (3, 128), (8, 96)):
        with pytest.raises(RuntimeError, match="not a supported shape"):
            g.set_tuning({"viscosity": bad})
    assert g.tuning() == DEFAULT  # unchanged
    with pytest.raises(RuntimeError, match="not a supported shape"):
        g.set_tuning({"density": (8, 256, 1)})  # staged is 4 lanes x 128 threads only


def test_autotune_restores_state_and_applies_its_choice():
    sc = make_scene("dam_65k")
    p = sc.params()
    g = Particles(p, sc.n)
    g.upload(sc.positions())
    g.step(5)
    before = {k: g.get_array(k) for k in (_abi.ARRAY_POSITIONS, _abi.ARRAY_POSITION_STARS, _abi.ARRAY_VELOCITIES,
                                          _abi.ARRAY_DENSITIES, _abi.ARRAY_LAMBDAS)}
    chosen, table = g.autotune(2)
    for k, a in before.items():
        assert np.array_equal(g.get_array(k), a), k
    assert g.tuning() == chosen
    assert set(table) == set(_abi.TUNE_CANDIDATES)
    for cand, per_family in table.items():
        for f, ms in per_family.items():
            assert ms > 0.0, (cand, f)
    direct = [c for c in table if not c[2]]
    for f, shape in chosen.items():  # the fastest direct shape, or staging where it is faster still
        best_direct = min(table[c][f] for c in direct)
        if shape[2]:
            assert table[shape][f] < best_direct
        else:
            assert table[shape][f] == best_direct
    # the next step is the step a fresh context with the chosen shapes takes
    # from the same state (the slot order after the sort depends only on the
    # bins and the original indices)
    d = g.download()
    g.step(1)
    h = Particles(p, sc.n)
    h.set_tuning(chosen)
    h.upload(d["x"], d["v"])
    h.step(1)
    assert np.array_equal(g.positions(), h.positions())
    assert np.array_equal(g.velocities(), h.velocities())


def test_autotune_learned_solver_and_exact_math():
    sc = make_scene("dam_8k", lambda_epsilon=1.0, solver=1, max_iterations=4, residual_tol=0.005)
    g = Particles(sc.params(), sc.n)
    g.mlp_init(3)
    g.upload(sc.positions())
    g.step(3)
    chosen, table = g.autotune(1)
    assert all(table[c]["density"] > 0.0 for c in table)  # the residual check counts for the density family
    g.step(2)
    assert g.stats()["error_flags"] == 0
    ex = Particles(make_scene("dam_2k", exact_math=1).params(), 4096)
    ex.upload(make_scene("dam_2k").positions())
    ex.step(1)
    chosen, table = ex.autotune(1)
    assert chosen == DEFAULT
    assert all(ms == 0.0 for c in table for ms in table[c].values())


def test_staged_gathers_stage_most_tiles_and_match_direct():
    """The staged shape reads most tiles from shared memory (the rest walk the
    int32 lists) and agrees with the direct shape after a few fast steps."""
    sc = make_scene("dam_65k")
    x = sc.positions()
    res = {}
    for staged in (1, 0):
        g = Particles(sc.params(), sc.n)
        g.set_tuning(_all_families((4, 128, staged)))
        g.upload(x)
        g.step(5)
        st = g.stats()
        res[staged] = (g.positions(), g.velocities(), st)
    st = res[1][2]
    assert st["tiles"] == (sc.n + 31) // 32 and st["tiles_staged"] > 0.8 * st["tiles"], st
    assert res[0][2]["tiles"] == 0
    scale = max(sc.box_max)
    np.testing.assert_allclose(res[1][0], res[0][0], rtol=0, atol=1e-4 * scale)
    np.testing.assert_allclose(res[1][1], res[0][1], rtol=0, atol=1e-3)
