"""The 1M- and 16.8M-particle dams on the CUDA path: one step against the
oracle at full size (1M), and size-independent properties of the neighbor
search (sortedness, bin bounds, per-bin order, permutation, sampled lists
against the reference's fill restated in float32)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from oracle.oracle import ARRAY_POSITIONS, OracleSim
from pbf_b200 import Particles, _abi, make_scene

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


# ---------------------------------------------------------------- 16.8M particles
def _ref_fill(p, xs, ids, b0, b1, dims, s, s2, cap):
    """Neighbors::fill_neighbors for one particle (neighbors.h:172-230) in
    float32: the 27 bins of the float re-hash coord + i*s (x offset outer, z
    inner), candidates in ascending reference index, strict d^2 < s^2, self
    skipped, the first cap kept."""
    x = xs[p]
    off = [np.float32(i) * s for i in (-1, 0, 1)]

    def axis_bin(c):
        return int(np.floor(np.float32(np.float32(c + s) / s)))

    out = []
    for i in range(3):
        cx = axis_bin(np.float32(x[0] + off[i]))
        for j in range(3):
            cy = axis_bin(np.float32(x[1] + off[j]))
            for k in range(3):
                cz = axis_bin(np.float32(x[2] + off[k]))
                nb = dims[0] * dims[1] * cz + cy * dims[0] + cx
                cand = ids[b0[nb]:b1[nb]].astype(np.int64)
                d = x[None, :] - xs[cand]
                d2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
                out.extend(int(q) for q in cand[(d2 < s2) & (cand != p)])
    return out[:cap]


def test_16m_neighbor_search_and_steps():
    """The 16.8M dam (256^3 lattice, 320^3 box, K = 4, cap 64): bins and
    permutation checked whole, the lists of a random sample of particles bit
    for bit against the reference's fill restated in float32, then fused
    steps without error flags."""
    sc = make_scene("dam_16m")
    p = sc.params()
    g = Particles(p, sc.n)
    g.upload(sc.positions())
    g.apply_external_forces()
    g.predict_positions()
    g.find_neighbors()
    b = g.bins()
    keys, ids, b0, b1 = b["sorted_keys"], b["sorted_ids"], b["bin_begin"], b["bin_end"]
    assert np.all(np.diff(keys.astype(np.int64)) >= 0)
    assert np.array_equal(np.sort(ids), np.arange(sc.n, dtype=np.uint32))
    same = keys[1:] == keys[:-1]
    assert np.all(ids[1:][same] > ids[:-1][same])
    counts = np.bincount(keys, minlength=b0.size)
    assert np.array_equal(b1.astype(np.int64) - b0.astype(np.int64), counts)
    xs = g.position_stars()
    gi, gc = g.neighbors(p.neighbor_cap)
    d = (C.c_int64 * 3)()
    assert _abi.load().pbf_grid_dims(C.byref(p), d) == 0
    dims = tuple(d)
    s = np.float32(p.neighbor_bin_spacing)
    s2 = np.float32(s * s)
    rng = np.random.default_rng(5)
    sample = np.concatenate([rng.choice(sc.n, 2000, replace=False), [0, sc.n - 1]])
    for q in sample:
        ref = _ref_fill(int(q), xs, ids, b0, b1, dims, s, s2, p.neighbor_cap)
        assert gc[q] == len(ref) and list(gi[q, :gc[q]]) == ref, int(q)
    del gi
    g.step(2)
    st = g.stats()
    assert st["error_flags"] == 0 and st["n"] == sc.n and np.isfinite(st["kinetic_energy"])
    assert 40.0 < st["mean_neighbors"] < 64.0
