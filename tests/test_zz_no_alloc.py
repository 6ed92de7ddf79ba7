"""pbf_find_neighbors_noalloc: the neighbor search for callers that may not
allocate device memory (hosts that own every device allocation through their
own pool or a fixed budget, or that cannot afford the device-wide
synchronisation of cudaMalloc/cudaFree).  Its working memory is a file-scope
device array inside the library; the caller passes only device inputs and
outputs.

Checked against the oracle's lists (the reference's fill_neighbors,
neighbors.h:197-230, restated) on dam_2k, dam_8k and dam_65k (65,536
particles on 46,656 bins: the advertised particle maximum) and on 16,384
particles crowded into one bin; against the regular entry points
(pbf_find_neighbors + pbf_get_neighbors) on two calls in a row with different
point sets, so the second call also proves that state left in the shared
array by the first does not leak into its result, and on 65,536 particles
piled onto 64 points of one bin (the run walk), which must also finish
quickly; and out-of-grid input must come back as PBF_FLAG_KEY_RANGE in the
caller's flag word.  Collected last on purpose."""
from __future__ import annotations

import ctypes as C
import time

import numpy as np
import pytest

from oracle.oracle import OracleSim
from pbf_b200 import Particles, _abi, make_scene

pytestmark = pytest.mark.gpu


def _regular_lists(p, x):
    with Particles(p, x.shape[0]) as g:
        g.upload(x)
        g.find_neighbors()
        return g.neighbors(p.neighbor_cap)


def _oracle_lists(p, x):
    o = OracleSim(p, x.shape[0])
    o.set_state(x)
    o.stage(2)  # find_neighbors
    idx, cnt = o.neighbors()
    o.close()
    return idx, cnt


def _noalloc(p, x, flags=True):
    """One call through the C ABI; returns (lists, counts, flags, seconds)."""
    import torch
    lib = _abi.load()
    n, cap = x.shape[0], p.neighbor_cap
    dx = torch.from_numpy(np.ascontiguousarray(x, np.float32)).cuda()
    nbr = torch.full((n, cap), 12345, dtype=torch.int32, device="cuda")
    cnt = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    fl = torch.full((1,), 0x7777, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rc = lib.pbf_find_neighbors_noalloc(C.byref(p), C.c_void_p(dx.data_ptr()), n, C.c_void_p(nbr.data_ptr()),
                                        C.c_void_p(cnt.data_ptr()), C.c_void_p(fl.data_ptr()) if flags else None,
                                        C.c_void_p(stream))
    assert rc == 0, lib.pbf_last_error(None).decode()
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    return nbr.cpu().numpy(), cnt.cpu().numpy(), int(fl.cpu().numpy()[0]), dt


def _assert_lists_equal(idx, cnt, ref_idx, ref_cnt, what):
    assert np.array_equal(cnt, ref_cnt), what
    live = np.arange(idx.shape[1])[None, :] < cnt[:, None]
    assert np.array_equal(np.where(live, idx, -1), np.where(live, ref_idx, -1)), what
    assert (idx[~live] == -1).all(), what  # -1 past the count


def _one_bin(p, n, seed):
    """n points uniform inside one bin near the grid's centre."""
    s = float(p.neighbor_bin_spacing)
    c = np.floor(np.array(p.boundary_max[:3], np.float64) / 2 / s) * s
    rng = np.random.default_rng(seed)
    return (c + rng.uniform(0.01 * s, 0.99 * s, (n, 3))).astype(np.float32)


def test_noalloc_matches_the_oracle_twice_in_a_row():
    for name in ("dam_8k", "dam_2k"):
        sc = make_scene(name)
        p, x = sc.params(), sc.positions()
        idx, cnt, flags, _ = _noalloc(p, x)
        assert flags == 0, name
        _assert_lists_equal(idx, cnt, *_oracle_lists(p, x), name)
        _assert_lists_equal(idx, cnt, *_regular_lists(p, x), name)


def test_noalloc_at_its_maximum_of_particles_matches_the_oracle():
    sc = make_scene("dam_65k")
    assert sc.n == _abi.NOALLOC_MAX_PARTICLES
    p, x = sc.params(), sc.positions()
    idx, cnt, flags, _ = _noalloc(p, x)
    assert flags == 0
    _assert_lists_equal(idx, cnt, *_oracle_lists(p, x), "dam_65k")


def test_noalloc_with_every_particle_in_one_bin_matches_the_oracle():
    p = make_scene("dam_8k").params()
    x = _one_bin(p, 16384, seed=5)
    idx, cnt, flags, _ = _noalloc(p, x)
    assert flags == 0
    assert (cnt == p.neighbor_cap).all()
    _assert_lists_equal(idx, cnt, *_oracle_lists(p, x), "one bin")


def test_noalloc_on_piles_in_one_bin_is_fast_and_matches_the_regular_path():
    """65,536 particles on 64 points of one bin, consecutive indices sharing a
    point: the radix sort stays linear and the fill decides a pile with one
    distance test, so the call takes milliseconds (a per-bin quadratic sort
    or a one-by-one walk would take seconds)."""
    p = make_scene("dam_8k").params()
    n = _abi.NOALLOC_MAX_PARTICLES
    pts = _one_bin(p, 64, seed=9)
    x = np.repeat(pts, n // 64, axis=0)
    _noalloc(p, x)  # first call on the device: address look-up, module load
    idx, cnt, flags, dt = _noalloc(p, x)
    assert flags == 0
    _assert_lists_equal(idx, cnt, *_regular_lists(p, x), "piles")
    assert dt < 0.5, dt


def test_noalloc_reports_out_of_grid_input_in_the_flag_word():
    sc = make_scene("dam_2k")
    p, x = sc.params(), sc.positions().copy()
    x[17] = (-5.0, 2.0, 2.0)            # outside the bin grid
    _, _, flags, _ = _noalloc(p, x)
    assert flags & _abi.PBF_FLAG_KEY_RANGE
    x[17] = (np.nan, 2.0, 2.0)          # non-finite
    _, _, flags, _ = _noalloc(p, x)
    assert flags & _abi.PBF_FLAG_KEY_RANGE
    # the next clean call starts from a clear error word; a NULL flag word is allowed
    _, _, flags, _ = _noalloc(p, sc.positions())
    assert flags == 0
    _noalloc(p, sc.positions(), flags=False)


def test_noalloc_rejects_sizes_beyond_its_maximum():
    lib = _abi.load()
    p = make_scene("dam_2k").params()
    n = _abi.NOALLOC_MAX_PARTICLES + 1
    rc = lib.pbf_find_neighbors_noalloc(C.byref(p), C.c_void_p(16), n, C.c_void_p(16), C.c_void_p(16), None, None)
    assert rc == _abi.PBF_ERR_CAPACITY
    assert b"exceed the maximum" in lib.pbf_last_error(None)
    big = make_scene("dam_65k").params()  # 36^3 = 46,656 bins: allowed
    assert lib.pbf_find_neighbors_noalloc(C.byref(big), None, 0, None, None, None, None) == 0
    huge = make_scene("dam_1m").params()  # 1.28M bins: beyond the grid maximum
    rc = lib.pbf_find_neighbors_noalloc(C.byref(huge), C.c_void_p(16), 10, C.c_void_p(16), C.c_void_p(16), None,
                                        None)
    assert rc == _abi.PBF_ERR_CAPACITY
    assert b"bins exceeds the maximum" in lib.pbf_last_error(None)
