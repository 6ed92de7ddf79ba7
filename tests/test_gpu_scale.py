"""The 1M-particle dam on the CUDA path: one step against the oracle at full
size, and size-independent properties of the neighbor search (sortedness,
bin bounds, per-bin order, permutation)."""
from __future__ import annotations

import numpy as np
import pytest

from oracle.oracle import ARRAY_POSITIONS, OracleSim
from pbf_b200 import Particles, make_scene

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dam_1m_one_step():
    sc = make_scene("dam_1m", exact_math=1)
    p = sc.params()
    x = sc.positions()
    g = Particles(p, sc.n)
    g.upload(x)
    g.step(1)
    o = OracleSim(p, sc.n)
    o.set_state(x)
    o.step(1)
    yield sc, p, g, o
    g.close()
    o.close()


def test_1m_positions_bit_exact_after_one_step(dam_1m_one_step):
    sc, p, g, o = dam_1m_one_step
    assert np.array_equal(g.positions(), o.get(ARRAY_POSITIONS))


def test_1m_lists_bit_exact(dam_1m_one_step):
    sc, p, g, o = dam_1m_one_step
    gi, gc = g.neighbors(p.neighbor_cap)
    oi, oc = o.neighbors()
    assert np.array_equal(gc, oc)
    assert np.array_equal(gi, oi)


def test_1m_bin_structure_properties(dam_1m_one_step):
    sc, p, g, o = dam_1m_one_step
    b = g.bins()
    keys, ids, b0, b1 = b["sorted_keys"], b["sorted_ids"], b["bin_begin"], b["bin_end"]
    assert np.all(np.diff(keys.astype(np.int64)) >= 0)                      # sorted by bin
    assert np.array_equal(np.sort(ids), np.arange(sc.n, dtype=np.uint32))  # a permutation
    same = keys[1:] == keys[:-1]
    assert np.all(ids[1:][same] > ids[:-1][same])                           # stable: ascending id within a bin
    B = b0.size
    counts = np.bincount(keys, minlength=B)
    assert np.array_equal(b1.astype(np.int64) - b0.astype(np.int64), counts)
    assert np.array_equal(b0, np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.uint32))
    assert np.array_equal(o.bins()["sorted_ids"], ids)


def test_1m_fast_step_within_tolerance():
    sc = make_scene("dam_1m")
    p = sc.params()
    x = sc.positions()
    g = Particles(p, sc.n)
    g.upload(x)
    g.step(1)
    o = OracleSim(p, sc.n)
    o.set_state(x)
    o.step(1)
    np.testing.assert_allclose(g.positions(), o.get(ARRAY_POSITIONS), rtol=0, atol=1e-5 * max(sc.box_max))
    st = g.stats()
    assert st["error_flags"] == 0 and st["n"] == sc.n
