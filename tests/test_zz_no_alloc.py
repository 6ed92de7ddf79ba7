"""pbf_find_neighbors_noalloc: the neighbor search for callers that may not
allocate device memory (hosts that own every device allocation through their
own pool or a fixed budget, or that cannot afford the device-wide
synchronisation of cudaMalloc/cudaFree).  Its working memory is a file-scope
device array inside the library; the caller passes only device inputs and
outputs.  Checked against the regular entry points (pbf_find_neighbors +
pbf_get_neighbors) on two calls in a row with different point sets, so the
second call also proves that state left in the shared array by the first
does not leak into its result.  Collected last on purpose."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from pbf_b200 import Particles, _abi, make_scene

pytestmark = pytest.mark.gpu


def _reference_lists(scene):
    p = scene.params()
    x = scene.positions()
    with Particles(p, scene.n) as g:
        g.upload(x)
        g.find_neighbors()
        idx, cnt = g.neighbors(p.neighbor_cap)
    return p, x, idx, cnt


def _noalloc(p, x):
    import torch
    lib = _abi.load()
    n, cap = x.shape[0], p.neighbor_cap
    dx = torch.from_numpy(np.ascontiguousarray(x, np.float32)).cuda()
    nbr = torch.full((n, cap), 12345, dtype=torch.int32, device="cuda")
    cnt = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.pbf_find_neighbors_noalloc(C.byref(p), C.c_void_p(dx.data_ptr()), n, C.c_void_p(nbr.data_ptr()),
                                        C.c_void_p(cnt.data_ptr()), C.c_void_p(stream))
    assert rc == 0, lib.pbf_last_error(None).decode()
    torch.cuda.synchronize()
    return nbr.cpu().numpy(), cnt.cpu().numpy()


def test_noalloc_matches_regular_entry_point_twice_in_a_row():
    for name in ("dam_8k", "dam_2k"):
        p, x, idx, cnt = _reference_lists(make_scene(name))
        got_idx, got_cnt = _noalloc(p, x)
        assert np.array_equal(got_cnt, cnt), name
        assert np.array_equal(got_idx, idx), name


def test_noalloc_rejects_sizes_beyond_its_maximum():
    lib = _abi.load()
    p = make_scene("dam_2k").params()
    n = _abi.NOALLOC_MAX_PARTICLES + 1
    rc = lib.pbf_find_neighbors_noalloc(C.byref(p), C.c_void_p(16), n, C.c_void_p(16), C.c_void_p(16), None)
    assert rc == _abi.PBF_ERR_CAPACITY
    assert b"exceed the maximum" in lib.pbf_last_error(None)
    big = make_scene("dam_65k").params()  # 36^3 = 46,656 bins: allowed
    assert lib.pbf_find_neighbors_noalloc(C.byref(big), None, 0, None, None, None) == 0
    huge = make_scene("dam_1m").params()  # 1.28M bins: beyond the grid maximum
    rc = lib.pbf_find_neighbors_noalloc(C.byref(huge), C.c_void_p(16), 10, C.c_void_p(16), C.c_void_p(16), None)
    assert rc == _abi.PBF_ERR_CAPACITY
    assert b"bins exceeds the maximum" in lib.pbf_last_error(None)
