"""Pin the oracle (oracle/pbf_oracle.c) against the reference.

1. The reference's own known-answer tests (Simulation/Tests/Serial/*.cpp),
   restated: kernels_test, neighbor_test (3D), particle_test, aabb_test,
   parameters_test — checked on the oracle and, where it is built, on the
   reference itself.
2. The golden vectors under tests/golden/, generated from the reference's
   own sources (tests/golden/make_golden.py), bit-exact.
3. Live oracle vs reference runs, bit-exact, when oracle/_ref is present.
"""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np
import pytest

from oracle.oracle import (ARRAY_DENSITIES, ARRAY_LAMBDAS, ARRAY_POSITION_STARS, ARRAY_POSITIONS, ARRAY_SCRATCH,
                           ARRAY_VELOCITIES, OracleSim, RefSim, oracle_lib, ref_available)
from pbf_b200 import make_scene, params_init

GOLDEN = Path(__file__).resolve().parent / "golden"
needs_ref = pytest.mark.skipif(not ref_available(True), reason="reference build oracle/_ref not present")


def neighbor_test_params(cap: int = 60):
    """neighbor_test.ini: 5x5x5 box, bin spacing 1.0, h = 1 (Simulation/Tests/Serial/neighbor_test.ini)."""
    p = params_init()
    p.time_step = 0.016
    p.gravity = -9.8
    p.gamma = 0.0
    p.visc_c = 0.01
    p.lambda_epsilon = 600.0
    p.vorticity_coef = 0.0005
    p.smoothing_radius = 1.0
    p.neighbor_bin_spacing = 1.0
    p.solve_steps = 3
    p.neighbor_cap = cap
    for a in range(3):
        p.boundary_min[a] = 0.0
        p.boundary_max[a] = 5.0
        p.mover_center[a] = -1.5
    p.rest_density = 8.0
    p.rest_mass = 1.0
    p.max_speed = 1.0
    p.particle_rest_spacing = 0.5
    return p


def construct_points(nx, ny, nz, spacing):
    """builders.cpp:47-62: spacing*i + spacing/2 per axis, z outer."""
    pts = []
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                pts.append([np.float32(spacing) * np.float32(i) + np.float32(spacing / 2.0),
                            np.float32(spacing) * np.float32(j) + np.float32(spacing / 2.0),
                            np.float32(spacing) * np.float32(k) + np.float32(spacing / 2.0)])
    return np.array(pts, np.float32)


# ---------------------------------------------------------------- kernels_test.cpp
def test_poly6_zero_at_and_beyond_h():
    lib = oracle_lib()
    h = 0.05
    assert lib.oracle_poly6(h, h) == pytest.approx(0.0)
    assert lib.oracle_poly6(h, h + h * 0.01) == 0.0


def test_poly6_normalised_3d():
    """kernels_test.cpp:72-103: sum over a 101^3 grid of spacing 2h/100 is 1 within 0.1%."""
    lib = oracle_lib()
    h = np.float32(0.05)
    dim = 101
    sp = np.float32(2.0 * h / (dim - 1))
    ax = (sp * np.arange(dim, dtype=np.float32) + np.float32(sp / 2.0)).astype(np.float32)
    mid = ax[dim // 2]
    dx, dy, dz = np.meshgrid(ax - mid, ax - mid, ax - mid, indexing="ij")
    r = np.sqrt(dx * dx + dy * dy + dz * dz).astype(np.float32).ravel()
    norm = np.float32(315.0 / (64.0 * math.pi * float(h) ** 9))
    a = (h * h - r * r).astype(np.float32)
    w = np.where(r > h, np.float32(0), norm * a * a * a).astype(np.float64)
    total = w.sum() * float(sp) ** 3
    assert total == pytest.approx(1.0, rel=1e-3)
    # the oracle's Poly6 agrees with this vectorised restatement pointwise
    for rr in (0.0, 0.01, 0.0333, 0.049, 0.05):
        ref = 0.0 if rr > h else float(norm * (h * h - np.float32(rr) ** 2) ** 3)
        assert lib.oracle_poly6(h, rr) == pytest.approx(ref, rel=1e-6, abs=1e-12)


def test_del_spikey_zero_at_h_beyond_h_and_origin():
    """kernels_test.cpp:131-207 (3D cases): zero at r = h, r > h and r = 0."""
    import ctypes as C
    lib = oracle_lib()
    out = (C.c_float * 3)()
    for q in ([0.05, 0.0, 0.0], [0.06, 0.0, 0.0], [0.0, 0.0, 0.0]):
        p = (C.c_float * 3)(0.0, 0.0, 0.0)
        qq = (C.c_float * 3)(*q)
        lib.oracle_del_spikey(0.05, p, qq, out)
        assert list(out) == pytest.approx([0.0, 0.0, 0.0], abs=1e-6)


def test_c_spline_zero_beyond_h():
    """kernels_test.cpp:209-239."""
    lib = oracle_lib()
    assert lib.oracle_c_spline(0.05, 0.05 + 0.05 * 0.01) == 0.0
    assert lib.oracle_c_spline(0.05, 0.05) == pytest.approx(0.0, abs=1e-9)


# ---------------------------------------------------------------- neighbor_test.cpp (3D)
def test_bin_ids_3d():
    """neighbor_test.cpp:84-120: exact bin ids in the padded 7x7x7 grid."""
    o = OracleSim(neighbor_test_params(), 1000)
    assert o.bin_id([-1.0, -1.0, -1.0]) == 0
    assert o.bin_id([0.0, 0.0, 0.0]) == 49 + 9 - 1
    assert o.bin_id([1.0, 1.0, 1.0]) == 49 + 49 + 17 - 1
    assert o.bin_id([4.999, 4.999, 4.999]) == 49 * 6 - 8 - 1


def _classify(i, j, k):
    edges = sum(1 for c in (i, j, k) if c in (0, 9))
    return {0: 26, 1: 17, 2: 11, 3: 7}[edges]


def test_lattice_neighbor_counts_3d():
    """neighbor_test.cpp:210-299: interior 26, face 17, edge 11, corner 7."""
    pts = construct_points(10, 10, 10, 0.5)
    o = OracleSim(neighbor_test_params(), 1000)
    o.set_state(pts)
    o.stage(2)
    _, cnt = o.neighbors()
    expect = np.array([_classify(i, j, k) for k in range(10) for j in range(10) for i in range(10)])
    assert np.array_equal(cnt, expect)


@needs_ref
def test_lattice_neighbor_lists_match_reference():
    pts = construct_points(10, 10, 10, 0.5)
    p = neighbor_test_params()
    o = OracleSim(p, 1000)
    r = RefSim(p, 1000, serial=True)
    assert r.bin_dims() == (7, 7, 7)
    for s in (o, r):
        s.set_state(pts)
        s.stage(2)
    io, co = o.neighbors()
    ir, cr = r.neighbors()
    assert np.array_equal(co, cr)
    assert np.array_equal(io, ir)


# ---------------------------------------------------------------- aabb_test.cpp / parameters
def test_bin_count_in_volume():
    """aabb_test.cpp:77-107."""
    import ctypes as C
    lib = oracle_lib()
    out = (C.c_int64 * 3)()
    lib.oracle_lattice_dims((C.c_float * 3)(0.0, -1.0, -2.0), (C.c_float * 3)(1.0, 2.0, -1.0), 1.0, out)
    assert list(out) == [1, 3, 1]
    lib.oracle_lattice_dims((C.c_float * 3)(0.0, 0.0, 0.0), (C.c_float * 3)(0.5, 1.4, 1.6), 0.5, out)
    assert list(out) == [1, 2, 3]


def test_particle_test_construct_fluid_count():
    """particle_test.cpp:84-120: the 3D particle_test.ini fluid box holds 27,000 particles."""
    import ctypes as C
    lib = oracle_lib()
    spacing = np.float32((8.0 / 28900.0) ** (1.0 / 3.0))
    out = (C.c_int64 * 3)()
    lib.oracle_lattice_dims((C.c_float * 3)(2.0, 2.0, 2.0), (C.c_float * 3)(4.0, 4.0, 4.0), float(spacing), out)
    assert out[0] * out[1] * out[2] == 27000


def test_particle_test_external_and_predict():
    """particle_test.cpp:122-225: v.y += g*dt only; x* = x + v*dt; clamp at the wall."""
    sc = make_scene("dam_2k")
    p = sc.params()
    x = sc.positions()
    o = OracleSim(p, sc.n)
    v = np.tile(np.array([[1.0, -1.0, 1.3]], np.float32), (sc.n, 1))
    o.set_state(x, v)
    o.stage(0)
    v1 = o.get(ARRAY_VELOCITIES)
    assert np.array_equal(v1[:, 0], v[:, 0]) and np.array_equal(v1[:, 2], v[:, 2])
    assert np.allclose(v1[:, 1], v[:, 1] + np.float32(p.gravity) * np.float32(p.time_step))
    o.stage(1)
    xs = o.get(ARRAY_POSITION_STARS)
    expect = np.clip(x + v1 * np.float32(p.time_step), 0.0, np.array(sc.box_max, np.float32))
    assert np.allclose(xs, expect, rtol=0, atol=1e-6)
    # a particle driven through the corner is clamped to the boundary minimum
    x2 = x.copy()
    x2[0] = 0.0
    v2 = np.zeros_like(x2)
    v2[0] = [-1.0, -2.0, -3.0]
    o.set_state(x2, v2)
    o.stage(1)
    assert np.array_equal(o.get(ARRAY_POSITION_STARS)[0], np.zeros(3, np.float32))


def test_particle_test_mean_density_within_5pct():
    """particle_test.cpp:247-266: 30^3 lattice, mean density within 5% of rest density."""
    p = params_init()
    spacing = np.float32((8.0 / 28900.0) ** (1.0 / 3.0))
    p.time_step = 1.0
    p.gravity = -9.8
    p.solve_steps = 4
    p.smoothing_radius = -1.0
    p.neighbor_bin_spacing = -1.0
    for a in range(3):
        p.boundary_min[a] = 0.0
        p.boundary_max[a] = 6.0
        p.mover_center[a] = (-1.5, -2.0, -1.5)[a]
    assert oracle_lib().oracle_params_derive(p, float(spacing), -1.0) == 0
    import ctypes as C
    d = (C.c_int64 * 3)(30, 30, 30)
    x = np.empty((27000, 3), np.float32)
    oracle_lib().oracle_build_lattice((C.c_float * 3)(2.0, 2.0, 2.0), d, float(spacing), 0.0, 0,
                                      x.ctypes.data_as(C.c_void_p))
    o = OracleSim(p, 27000)
    o.set_state(x)
    o.stage(2)
    o.stage(3)
    rho = o.get(ARRAY_DENSITIES)
    assert abs(rho.mean() - p.rest_density) < p.rest_density / 20.0


@needs_ref
def test_parameters_test_values_through_reference_reader(tmp_path):
    """parameters_test.cpp:33-54 through the reference's own read_INI and derive_from_input."""
    import ctypes as C
    ini = tmp_path / "params_test.ini"
    ini.write_text(PARAMS_TEST_INI)
    from oracle.oracle import ref_lib
    out = (C.c_float * 8)()
    counts = (C.c_uint64 * 3)()
    assert ref_lib(True).ref_derived_from_ini(str(ini).encode(), out, counts) == 0
    assert list(counts) == [100000, 30000, 4]
    assert out[0] == pytest.approx(0.03218, rel=1e-4)
    assert out[4] == pytest.approx(29999.99609, rel=1e-5)
    assert out[6] == pytest.approx(14.48234, rel=1e-5)


PARAMS_TEST_INI = """[SimParameters]
global_particle_count = 30000
number_solve_steps = 4
time_step = 0.008
max_particles_local = 100000

[PhysicalParameters]
g = -9.8
density = 1000.0
visc_c = 0.03
lambda_epsilon = 10.0
k_stiff = 1.0
gamma = 600.0
vorticity_coef = 0.00001

[Boundary]
min = 0.0, 0.0, 0.0
max = 1.5, 2.0, 1.5

[InitialFluid]
min = 0.0, 0.0, 0.0
max = 1.0, 1.0, 1.0

[Mover]
center = -1.5, -2.0, -1.5
"""


# ---------------------------------------------------------------- golden vectors
def _golden(name):
    return np.load(GOLDEN / name)


def test_oracle_matches_golden_step1():
    """Every stage array of step 1 of the 2,048-particle dam, bit-exact against
    the reference's own output (in-place viscosity order, as the serial reference)."""
    g = _golden("dam_2k_step1.npz")
    sc = make_scene("dam_2k")
    p = sc.params()
    assert np.float32(p.rest_density) == g["rest_density"]
    x0 = sc.positions()
    assert np.array_equal(x0, g["x0"])
    o = OracleSim(p, sc.n, visc_mode=1)
    o.set_state(x0)
    o.stage(0)
    o.stage(1)
    assert np.array_equal(o.get(ARRAY_POSITION_STARS), g["xs_pred"])
    o.stage(2)
    idx, cnt = o.neighbors()
    assert np.array_equal(cnt, g["cnt"].astype(np.int32))
    gi = g["nbr"].astype(np.int32)
    for i in range(sc.n):
        assert np.array_equal(idx[i, :cnt[i]], gi[i, :cnt[i]])
    b = o.bins()
    for k in ("sorted_ids", "sorted_keys", "bin_begin", "bin_end"):
        assert np.array_equal(b[k], g[k]), k
    for sub in range(p.solve_steps):
        o.stage(3, sub)
        o.stage(4, sub)
        o.stage(5, sub)
        if sub == 0:
            assert np.array_equal(o.get(ARRAY_DENSITIES), g["rho_it0"])
            assert np.array_equal(o.get(ARRAY_LAMBDAS), g["lam_it0"])
            assert np.array_equal(o.get(ARRAY_SCRATCH), g["dp_it0"])
        o.stage(6, sub)
    assert np.array_equal(o.get(ARRAY_POSITION_STARS), g["xs_solved"])
    for i in range(7, 13):
        o.stage(i)
    assert np.array_equal(o.get(ARRAY_POSITIONS), g["x1"])
    assert np.array_equal(o.get(ARRAY_VELOCITIES), g["v1"])
    assert np.array_equal(o.get(ARRAY_SCRATCH), g["vort1"])


def test_oracle_matches_golden_trajectory():
    g = _golden("dam_2k_traj.npz")
    sc = make_scene("dam_2k")
    p = sc.params()
    o = OracleSim(p, sc.n, visc_mode=1)
    o.set_state(sc.positions())
    o.step(int(g["steps"]))
    assert np.array_equal(o.get(ARRAY_POSITIONS), g["x_final"])


def test_oracle_matches_golden_8k_50_steps():
    g = _golden("dam_8k_stats.npz")
    sc = make_scene("dam_8k")
    o = OracleSim(sc.params(), sc.n, visc_mode=1)
    o.set_state(sc.positions())
    o.step(int(g["steps"]))
    assert np.array_equal(o.get(ARRAY_POSITIONS), g["x_final"])


def test_jacobi_viscosity_keeps_positions_of_step1():
    """The GPU's Jacobi XSPH only changes velocities: x after step 1 is x*
    before viscosity, identical in both orders."""
    g = _golden("dam_2k_step1.npz")
    sc = make_scene("dam_2k")
    o = OracleSim(sc.params(), sc.n, visc_mode=0)
    o.set_state(sc.positions())
    o.step(1)
    assert np.array_equal(o.get(ARRAY_POSITIONS), g["x1"])
    v = o.get(ARRAY_VELOCITIES)
    assert np.allclose(v, g["v1"], rtol=0, atol=1e-2 * np.abs(g["v1"]).max())


@needs_ref
def test_oracle_matches_reference_live_with_surface_tension():
    """gamma != 0 exercises apply_surface_tension (particles.h:400-431) and C_Spline."""
    sc = make_scene("dam_2k", gamma=600.0)
    p = sc.params()
    o = OracleSim(p, sc.n, visc_mode=1)
    r = RefSim(p, sc.n, serial=True)
    x = sc.positions()
    o.set_state(x)
    r.set_state(x)
    o.step(3)
    r.step(3)
    for w in (ARRAY_POSITIONS, ARRAY_VELOCITIES, ARRAY_DENSITIES, ARRAY_LAMBDAS, ARRAY_SCRATCH):
        assert np.array_equal(o.get(w), r.get(w)), w


@needs_ref
def test_oracle_matches_reference_live_65k_steps():
    sc = make_scene("dam_65k")
    p = sc.params()
    o = OracleSim(p, sc.n, visc_mode=1)
    r = RefSim(p, sc.n, serial=True)
    x = sc.positions()
    o.set_state(x)
    r.set_state(x)
    o.step(2)
    r.step(2)
    for w in (ARRAY_POSITIONS, ARRAY_VELOCITIES, ARRAY_DENSITIES, ARRAY_LAMBDAS):
        assert np.array_equal(o.get(w), r.get(w)), w
    io, co = o.neighbors()
    ir, cr = r.neighbors()
    assert np.array_equal(co, cr)
    mask = np.arange(60)[None, :] < co[:, None]
    assert np.array_equal(np.where(mask, io, -1), np.where(mask, ir, -1))
