"""State files and the emitter on the GPU.

- pbf_save_state / pbf_load_state: the loaded arrays are the saved ones, and
  a context resumed from the file takes bit-identical steps (plain exact and
  fast math, the learned solver with its network and lambda history).
- pbf_construct_fluid / the emitter: the appended particles are the
  reference's construct_fluid lattice, and the steps after them equal the
  oracle's (exact math) on the grown set.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from oracle.oracle import ARRAY_POSITIONS, ARRAY_VELOCITIES, OracleSim
from pbf_b200 import Particles, _abi, make_batch, make_scene
from pbf_b200.learn import warm_start_scene

pytestmark = pytest.mark.gpu
C_PARAMS_BYTES = C.sizeof(_abi.PbfParams)
ARRAYS = (_abi.ARRAY_POSITIONS, _abi.ARRAY_VELOCITIES, _abi.ARRAY_DENSITIES, _abi.ARRAY_LAMBDAS)


def _resume_check(sc, tmp_path, network=False):
    p = sc.params()
    a = Particles(p, sc.n)
    if network:
        a.mlp_init(11)
    a.upload(sc.positions())
    a.step(8)
    f = tmp_path / "state.pbf"
    a.save_state(f)
    saved = {w: a.get_array(w) for w in ARRAYS}
    a.step(6)
    b = Particles(p, sc.n)  # a fresh context, default shapes and no network
    b.load_state(f)
    assert b.step_count() == 8 and b.local_count() == sc.n
    for w, arr in saved.items():
        assert np.array_equal(b.get_array(w), arr), w
    assert b.tuning() == a.tuning()
    b.step(6)
    for w in (_abi.ARRAY_POSITIONS, _abi.ARRAY_VELOCITIES):
        assert np.array_equal(a.get_array(w), b.get_array(w)), w
    assert b.step_count() == a.step_count() == 14


@pytest.mark.parametrize("exact", [1, 0])
def test_resume_from_state_file_is_bitwise(exact, tmp_path):
    _resume_check(make_scene("dam_8k", exact_math=exact), tmp_path)


def test_resume_learned_solver_with_network(tmp_path):
    _resume_check(warm_start_scene("dam_8k", solver=1, max_iterations=4, residual_tol=0.01), tmp_path, network=True)


def test_resume_after_autotune_keeps_shapes(tmp_path):
    sc = make_scene("dam_8k")
    a = Particles(sc.params(), sc.n)
    a.upload(sc.positions())
    a.step(2)
    a.set_tuning({"density": (8, 128), "viscosity": (4, 256)})
    _ = a.get_array(_abi.ARRAY_POSITIONS)
    a.save_state(tmp_path / "s.pbf")
    b = Particles(sc.params(), sc.n)
    b.load_state(tmp_path / "s.pbf")
    assert b.tuning() == a.tuning()
    a.step(3)
    b.step(3)
    assert np.array_equal(a.positions(), b.positions())


def test_state_file_errors(tmp_path):
    sc = make_scene("dam_2k")
    a = Particles(sc.params(), sc.n)
    a.upload(sc.positions())
    a.save_state(tmp_path / "s.pbf")
    small = Particles(sc.params(), sc.n // 2)
    with pytest.raises(RuntimeError, match="capacity"):
        small.load_state(tmp_path / "s.pbf")
    (tmp_path / "junk.pbf").write_bytes(b"not a state file at all" * 8)
    with pytest.raises(RuntimeError, match="not a PBF state file"):
        a.load_state(tmp_path / "junk.pbf")
    raw = (tmp_path / "s.pbf").read_bytes()
    (tmp_path / "cut.pbf").write_bytes(raw[: len(raw) // 2])
    with pytest.raises(RuntimeError, match="truncated"):
        a.load_state(tmp_path / "cut.pbf")
    with pytest.raises(RuntimeError, match="cannot open"):
        a.load_state(tmp_path / "missing.pbf")
    # header layout as documented in pbf.h
    assert raw[:8] == b"PBFSTATE"
    version, pbytes, n, steps = np.frombuffer(raw[8:32], dtype="<u4,<u4,<u8,<u8")[0]
    assert version == 1 and pbytes == C_PARAMS_BYTES and n == sc.n and steps == 0
    x = np.frombuffer(raw, "<f4", count=3 * sc.n, offset=104 + pbytes).reshape(-1, 3)
    assert np.array_equal(x, a.positions())



def test_construct_fluid_and_emitter_match_the_oracle():
    sc = make_scene("dam_8k", exact_math=1)
    p = sc.params()
    g = Particles(p, sc.n + 200)
    g.upload(sc.positions())
    g.step(3)
    n0 = g.local_count()
    # construct_fluid of a 2x2x3-particle block, and one emitter particle
    added = g.construct_fluid((12.0, 12.0, 12.0), (13.0, 13.0, 13.5), velocity=(0.5, -1.0, 0.25))
    assert added == 12
    assert g.emit((15.0, 15.0, 15.0), velocity=(0.0, -2.0, 0.0)) == 1
    assert g.local_count() == n0 + 13
    x = g.positions()
    sp = np.float32(p.particle_rest_spacing)
    new = x[n0:n0 + 12]
    ref = np.array([[np.float32(i) * sp + np.float32(12.0) + sp / np.float32(2.0),
                     np.float32(j) * sp + np.float32(12.0) + sp / np.float32(2.0),
                     np.float32(k) * sp + np.float32(12.0) + sp / np.float32(2.0)]
                    for k in range(3) for j in range(2) for i in range(2)], np.float32)
    assert np.array_equal(new, ref)
    assert np.array_equal(g.velocities()[n0:n0 + 12], np.tile(np.float32([0.5, -1.0, 0.25]), (12, 1)))
    # the oracle continues from the grown set
    o = OracleSim(p, g.local_count())
    o.set_state(g.positions(), g.velocities())
    g.step(4)
    o.step(4)
    assert np.array_equal(g.get_array(ARRAY_POSITIONS), o.get(ARRAY_POSITIONS))
    assert np.array_equal(g.get_array(ARRAY_VELOCITIES), o.get(ARRAY_VELOCITIES))
    with pytest.raises(RuntimeError, match="capacity"):
        g.construct_fluid((1.0, 1.0, 1.0), (10.0, 10.0, 10.0))
    b = make_batch(scenes=2, n_max=8192)
    h = Particles.batch(b)
    h.upload(b.positions())
    with pytest.raises(RuntimeError, match="fixed particle counts"):
        h.add_particles(np.zeros((1, 3), np.float32))
