"""The order of the fast path's neighbour lists.

Fast math walks a particle's 27 bins in slot order (z offset outer, x
inner: the bins come in ascending keys, so the gathers read neighbouring
slots together) while few lists reach the cap.  The cap keeps the first
entries in the reference's order (x offset outer), so a slot-order list that
reaches it is walked again in that order, and once more than 1 in 64 lists
reach it the fill walks in the reference's order until the share drops.
Whatever the order, the exported lists are the reference's, bit for bit.
An upload starts the choice afresh.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle.oracle import OracleSim
from pbf_b200 import Particles, _abi, make_scene

pytestmark = pytest.mark.gpu


def _shapes(staged):
    return {f: (4, 128, staged) for f in _abi.TUNE_FAMILIES}


def _compressed(sc, factor=0.9):
    """The lattice squeezed toward the box's low corner: the interior
    particles have more neighbours than the cap, the ones near the free
    surface fewer."""
    return (sc.positions() * np.float32(factor)).astype(np.float32)


def _compare(g, o, p):
    gi, gc = g.neighbors(p.neighbor_cap)
    oi, oc = o.neighbors()
    assert np.array_equal(gc, oc), "neighbor counts differ"
    assert np.array_equal(gi, oi), "neighbor lists differ"
    return g.stats()


def _fill_and_compare(g, p, x):
    """Upload x (which starts the order choice afresh) and fill the lists
    as a step does; the lists must be the oracle's.  Returns the stats and
    the oracle, whose lists a refill of the same state must match too."""
    o = OracleSim(p, len(x))
    g.upload(x)
    o.set_state(x)
    for i, fn in enumerate((g.apply_external_forces, g.predict_positions, g.find_neighbors)):
        fn()
        o.stage(i)
    return _compare(g, o, p), o


def test_fresh_dam_walks_in_slot_order():
    sc = make_scene("dam_8k")
    with Particles(sc.params(), sc.n) as g:
        g.upload(sc.positions())
        g.step(2)
        st = g.stats()
        assert st["cap_hits"] == 0 and st["lists_slot_order"] == 1, st
    with Particles(sc.with_(exact_math=1).params(), sc.n) as g:
        g.upload(sc.positions())
        g.step(1)
        assert g.stats()["lists_slot_order"] == 0  # exact math: always the reference's order


@pytest.mark.parametrize("staged", [0, 1])
def test_capped_lists_are_the_references_in_both_orders(staged):
    """After the upload the fill walks in slot order: the capped lists are
    walked again in the reference's order.  With most lists capped, the next
    fill of the same state walks in the reference's order.  Both times the
    lists are the oracle's."""
    sc = make_scene("dam_8k")
    p = sc.params()
    x = _compressed(sc)
    with Particles(p, sc.n) as g:
        g.set_tuning(_shapes(staged))
        st, o = _fill_and_compare(g, p, x)
        assert st["lists_slot_order"] == 1
        assert 64 * st["cap_hits"] > sc.n and st["cap_hits"] < sc.n, st  # capped and uncapped lists both
        g.find_neighbors()
        st = _compare(g, o, p)
        assert st["lists_slot_order"] == 0, st
        assert st["error_flags"] == 0


def test_order_returns_to_slot_once_few_lists_are_capped():
    sc = make_scene("dam_8k")
    p = sc.params()
    with Particles(p, sc.n) as g:
        _fill_and_compare(g, p, _compressed(sc))
        g.find_neighbors()
        assert g.stats()["lists_slot_order"] == 0
        g.set_array(_abi.ARRAY_POSITION_STARS, sc.positions())  # an uncrowded state, no upload
        g.find_neighbors()
        st = g.stats()  # this fill still walked in the reference's order
        assert st["lists_slot_order"] == 0 and st["cap_hits"] == 0, st
        g.find_neighbors()
        assert g.stats()["lists_slot_order"] == 1


def test_upload_starts_the_order_choice_afresh():
    """After an upload a context steps bit for bit as a fresh one, whatever
    order its earlier fills had come to."""
    sc = make_scene("dam_8k")
    p = sc.params()
    with Particles(p, sc.n) as g, Particles(p, sc.n) as h:
        _fill_and_compare(g, p, _compressed(sc))  # its next fill would walk in the reference's order
        for c in (g, h):
            c.upload(sc.positions())
            c.step(3)
        assert g.stats()["lists_slot_order"] == h.stats()["lists_slot_order"] == 1
        assert np.array_equal(g.positions(), h.positions())
        assert np.array_equal(g.velocities(), h.velocities())


def _crowded(sc, seed=5):
    """The lattice with 3,000 particles scattered (not piled) inside a cube of
    2 x 2 x 2 bins near the floor: bins of 350-400 particles, crowded but
    short of the run-by-run walk, beside ordinary ones."""
    x = sc.positions()
    s = sc.params().neighbor_bin_spacing
    rng = np.random.default_rng(seed)
    x[:3000] = (np.float32(3.0 * s) + rng.uniform(0.0, 2.0 * s, (3000, 3))).astype(np.float32)
    return x


@pytest.mark.parametrize("exact,staged", [(1, 0), (0, 0), (0, 1)])
def test_crowded_bins_bit_exact(exact, staged):
    sc = make_scene("dam_8k", exact_math=exact)
    p = sc.params()
    x = _crowded(sc)
    s = p.neighbor_bin_spacing
    keys = np.floor(x / s).astype(np.int64)
    _, per_bin = np.unique(keys, axis=0, return_counts=True)
    assert per_bin.max() > 256 and per_bin.max() <= 512, per_bin.max()  # crowded, short of the run walk
    with Particles(p, sc.n) as g:
        if not exact:
            g.set_tuning(_shapes(staged))
        st, o = _fill_and_compare(g, p, x)
        assert st["error_flags"] == 0
        g.find_neighbors()  # fast math: this fill walks in the reference's order
        assert _compare(g, o, p)["error_flags"] == 0


def test_staged_step_with_capped_lists_matches_direct():
    """Tiles holding a capped slot-order list walk the int32 lists; the step
    agrees with the direct shape's."""
    sc = make_scene("dam_8k")
    x = _compressed(sc)
    res = {}
    for staged in (1, 0):
        with Particles(sc.params(), sc.n) as g:
            g.set_tuning(_shapes(staged))
            g.upload(x)
            g.step(2)
            res[staged] = (g.positions(), g.velocities(), g.stats())
    assert res[1][2]["error_flags"] == 0 and res[0][2]["error_flags"] == 0
    scale = max(sc.box_max)
    np.testing.assert_allclose(res[1][0], res[0][0], rtol=0, atol=1e-4 * scale)
    np.testing.assert_allclose(res[1][1], res[0][1], rtol=0, atol=1e-3)
