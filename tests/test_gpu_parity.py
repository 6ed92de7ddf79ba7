"""CUDA path (libpbf_b200 through its C ABI) against the oracle and the
reference's golden vectors.

Bars:
  - neighbor search (bins, permutation, lists): bit-exact, always;
  - exact_math = 1: every array bit-exact against the oracle (Jacobi XSPH),
    stage by stage and over many fused steps;
  - exact_math = 0 (the fast default): positions after one step within 1e-5
    relative of the reference's own output; statistics after 100 steps
    within 1%.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle.oracle import (ARRAY_DENSITIES, ARRAY_LAMBDAS, ARRAY_POSITION_STARS, ARRAY_POSITIONS, ARRAY_SCRATCH,
                           ARRAY_VELOCITIES, OracleSim, RefSim, ref_available)
from pbf_b200 import Particles, _abi, make_scene

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
REL_TOL = 1e-5          # positions after one step, relative (to the coordinate scale of the box)
STAT_TOL = 0.01         # 100-step statistics, relative
ALL = (ARRAY_POSITIONS, ARRAY_POSITION_STARS, ARRAY_VELOCITIES, ARRAY_SCRATCH, ARRAY_DENSITIES, ARRAY_LAMBDAS)
NAMES = {ARRAY_POSITIONS: "x", ARRAY_POSITION_STARS: "x*", ARRAY_VELOCITIES: "v", ARRAY_SCRATCH: "scratch",
         ARRAY_DENSITIES: "rho", ARRAY_LAMBDAS: "lambda"}


def pair(scene, visc_mode=0, exact=1):
    sc = scene.with_(exact_math=exact)
    p = sc.params()
    g = Particles(p, sc.n)
    o = OracleSim(p, sc.n, visc_mode=visc_mode)
    x = sc.positions()
    g.upload(x)
    o.set_state(x)
    return sc, p, g, o


def assert_lists_equal(g, o, cap):
    gi, gc = g.neighbors(cap)
    oi, oc = o.neighbors()
    assert np.array_equal(gc, oc), "neighbor counts differ"
    assert np.array_equal(gi, oi), "neighbor lists differ"


def assert_arrays(g, o, which=ALL, exact=True, rtol=0.0, atol=0.0):
    for w in which:
        a, b = g.get_array(w), o.get(w)
        if exact:
            bad = np.flatnonzero(a.ravel() != b.ravel())
            assert bad.size == 0, f"{NAMES[w]}: {bad.size} values differ, first at {bad[:5]}"
        else:
            np.testing.assert_allclose(a, b, rtol=rtol, atol=atol, err_msg=NAMES[w])


# ---------------------------------------------------------------- stage by stage
@pytest.mark.parametrize("name", ["dam_2k", "dam_8k"])
def test_every_stage_bit_exact_vs_oracle(name):
    sc, p, g, o = pair(make_scene(name))
    g.apply_external_forces(); o.stage(0)
    assert_arrays(g, o)
    g.predict_positions(); o.stage(1)
    assert_arrays(g, o)
    g.find_neighbors(); o.stage(2)
    assert_lists_equal(g, o, p.neighbor_cap)
    gb, ob = g.bins(), o.bins()
    for k in ("sorted_keys", "sorted_ids", "bin_begin", "bin_end"):
        assert np.array_equal(gb[k], ob[k]), k
    for sub in range(p.solve_steps):
        g.compute_densities(); o.stage(3, sub)
        assert_arrays(g, o)
        g.compute_pressure_lambdas(); o.stage(4, sub)
        assert_arrays(g, o)
        g.compute_pressure_dps(substep=sub); o.stage(5, sub)
        assert_arrays(g, o)
        g.update_position_stars(); o.stage(6, sub)
        assert_arrays(g, o)
    for stage, fn in ((7, g.update_velocities), (9, g.apply_viscosity), (10, g.compute_vorticity),
                      (11, g.apply_vorticity), (9, g.apply_viscosity), (12, g.update_positions)):
        fn()
        o.stage(stage)
        assert_arrays(g, o)


def test_stages_fast_math_within_tolerance():
    sc, p, g, o = pair(make_scene("dam_2k"), exact=0)
    for i, fn in enumerate((g.apply_external_forces, g.predict_positions, g.find_neighbors)):
        fn()
        o.stage(i)
    assert_lists_equal(g, o, p.neighbor_cap)
    for sub in range(p.solve_steps):
        g.compute_densities(); o.stage(3)
        g.compute_pressure_lambdas(); o.stage(4)
        g.compute_pressure_dps(); o.stage(5)
        g.update_position_stars(); o.stage(6)
    np.testing.assert_allclose(g.get_array(ARRAY_DENSITIES), o.get(ARRAY_DENSITIES), rtol=1e-5)
    # lambda = -C/(sum|grad C|^2 + eps) with C = rho/rho0 - 1: a 1e-5 relative
    # density difference moves C by up to 1e-5, so lambda by 1e-5/eps.
    lam_g, lam_o = g.get_array(ARRAY_LAMBDAS), o.get(ARRAY_LAMBDAS)
    np.testing.assert_allclose(lam_g, lam_o, rtol=1e-4, atol=1e-5 / p.lambda_epsilon)
    np.testing.assert_allclose(g.get_array(ARRAY_POSITION_STARS), o.get(ARRAY_POSITION_STARS), rtol=0,
                               atol=REL_TOL * max(sc.box_max))


# ---------------------------------------------------------------- fused, graph-captured step
@pytest.mark.parametrize("steps", [1, 20])
def test_fused_step_bit_exact_vs_oracle(steps):
    sc, p, g, o = pair(make_scene("dam_8k"))
    g.step(steps)
    o.step(steps)
    assert_arrays(g, o, which=(ARRAY_POSITIONS, ARRAY_VELOCITIES, ARRAY_DENSITIES, ARRAY_LAMBDAS, ARRAY_SCRATCH))
    assert_lists_equal(g, o, p.neighbor_cap)


def test_fused_step_replay_is_deterministic():
    sc, p, g, _ = pair(make_scene("dam_2k"), exact=0)
    g.step(5)
    a = g.download()
    g.upload(sc.positions())
    g.step(5)
    b = g.download()
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def test_fused_step_fast_vs_reference_golden():
    """One fast step against the reference's own step-1 output (golden)."""
    gd = np.load(GOLDEN / "dam_2k_step1.npz")
    sc = make_scene("dam_2k")
    p = sc.params()
    assert np.float32(p.rest_density) == gd["rest_density"]
    g = Particles(p, sc.n)
    g.upload(gd["x0"])
    g.step(1)
    x = g.positions()
    scale = max(sc.box_max)
    np.testing.assert_allclose(x, gd["x1"], rtol=0, atol=REL_TOL * scale)
    # the lists the step built are the reference's, bit for bit
    idx, cnt = g.neighbors(60)
    assert np.array_equal(cnt, gd["cnt"].astype(np.int32))
    ref = gd["nbr"].astype(np.int32)
    mask = np.arange(60)[None, :] < cnt[:, None]
    assert np.array_equal(np.where(mask, idx, -1), np.where(mask, ref, -1))
    b = g.bins()
    for k in ("sorted_keys", "sorted_ids", "bin_begin", "bin_end"):
        assert np.array_equal(b[k], gd[k]), k


def test_fused_step_exact_positions_bitwise_vs_reference_golden():
    """exact_math: x after step 1 is bit-identical to the reference's."""
    gd = np.load(GOLDEN / "dam_2k_step1.npz")
    sc = make_scene("dam_2k", exact_math=1)
    g = Particles(sc.params(), sc.n)
    g.upload(gd["x0"])
    g.step(1)
    assert np.array_equal(g.positions(), gd["x1"])
    assert np.array_equal(g.densities(), gd["rho"])
    assert np.array_equal(g.lambdas(), gd["lam"])


def _stat_close(a: dict, b: dict, keys=("mean_density_error", "max_density_error", "kinetic_energy")):
    for k in keys:
        assert a[k] == pytest.approx(b[k], rel=STAT_TOL), (k, a[k], b[k])
    for i in range(3):
        assert a["center_of_mass"][i] == pytest.approx(b["center_of_mass"][i], rel=STAT_TOL)


def test_golden_trajectory_statistics_fast():
    gd = np.load(GOLDEN / "dam_2k_traj.npz")
    sc = make_scene("dam_2k")
    g = Particles(sc.params(), sc.n)
    g.upload(sc.positions())
    cols = list(gd["columns"])
    for s in range(int(gd["steps"])):
        g.step(1)
    st = g.stats()
    row = gd["stats"][-1]
    ref = {"mean_density_error": row[cols.index("mean_err")], "max_density_error": row[cols.index("max_err")],
           "kinetic_energy": row[cols.index("ke")],
           "center_of_mass": [row[cols.index("cx")], row[cols.index("cy")], row[cols.index("cz")]]}
    _stat_close(st, ref)


def test_65k_100_steps_exact_bitwise_vs_oracle():
    """exact_math over the full 100-step 65k run: every position and velocity
    bit-identical to the oracle (Jacobi XSPH), hence identical statistics."""
    sc, p, g, o = pair(make_scene("dam_65k"))
    g.step(sc.steps)
    o.step(sc.steps)
    assert_arrays(g, o, which=(ARRAY_POSITIONS, ARRAY_VELOCITIES, ARRAY_DENSITIES))
    a, b = g.stats(), o.stats()
    for k in ("mean_density_error", "max_density_error", "kinetic_energy"):
        assert a[k] == pytest.approx(b[k], rel=1e-12), k


# Statistics of the 65k dam over steps 81-100 (the mean of the 20 per-step
# values), fast math against the oracle and the reference.  The reference
# disagrees with ITSELF from run to run (its in-place XSPH and nudge races,
# particles.h:303-305, 436-447): single-step snapshots after 100 steps spread
# 7.5% (mean density error) and 22% (max) between its OpenMP runs at
# eps = 600.  Averaged over steps 81-100 the spread between the reference at 2
# and 8 threads, the oracle, and the oracle started 1 ulp off is:
#   eps = 600: mean err 0.69%, max err 0.55%, KE 1.01%, centre of mass 0.16%
#   eps = 1:   mean err 0.74%, max err 5.5%,  KE 0.06%, centre of mass 0.02%
# and one more reference run at eps = 600 gave an averaged max error of 3.683
# against 3.741-3.763 for the others (2.2%): at this eps the max is set by
# particles piled exactly into wall corners.
# Four runs bound the spread from below only, so the bars are twice the
# measured spread, and never tighter than 1%.
STAT_BARS = {
    600.0: {"mean_density_error": 0.014, "max_density_error": 0.044, "kinetic_energy": 0.02, "com": 0.01},
    1.0: {"mean_density_error": 0.015, "max_density_error": 0.11, "kinetic_energy": 0.01, "com": 0.01},
}
STAT_KEYS = ("mean_density_error", "max_density_error", "kinetic_energy")


def averaged_stats(sim, stats, steps=100, window=20):
    sim.step(steps - window)
    acc = []
    for _ in range(window):
        sim.step(1)
        st = stats()
        acc.append([st[k] for k in STAT_KEYS] + list(st["center_of_mass"]))
    m = np.mean(acc, axis=0)
    return dict(zip(STAT_KEYS, m[:3])) | {"center_of_mass": list(m[3:])}


def check_bars(a, b, bars):
    for k in STAT_KEYS:
        assert a[k] == pytest.approx(b[k], rel=bars[k]), (k, a[k], b[k])
    for i in range(3):
        assert a["center_of_mass"][i] == pytest.approx(b["center_of_mass"][i], rel=bars["com"])


@pytest.mark.parametrize("eps", [600.0, 1.0])
def test_65k_100_steps_fast_statistics(eps):
    sc, p, g, o = pair(make_scene("dam_65k", lambda_epsilon=eps), exact=0)
    a = averaged_stats(g, g.stats)
    b = averaged_stats(o, o.stats)
    check_bars(a, b, STAT_BARS[eps])
    assert g.stats()["error_flags"] == 0


# Against the reference's OpenMP build, whose in-place XSPH and density nudge
# race (every run differs, more so with more host threads): the max clamped
# density error at eps = 600, set by how many particles pile into a wall
# corner, is a discrete chaotic count.  Averaged over steps 81-100 the
# reference's runs have differed from each other by up to 2.2% and from this
# GPU path by up to 4.4% on the boxes of this build; its bar here is 10%.  The
# deterministic oracle keeps the 4.4% bar (test_65k_100_steps_fast_statistics).
REF_BUILD_BARS = dict(STAT_BARS[600.0], max_density_error=0.10)


def test_65k_100_steps_fast_vs_reference_build():
    """The same averaged statistics against the reference's own OpenMP build."""
    if not ref_available():
        pytest.skip("reference build not present")
    sc = make_scene("dam_65k")
    p = sc.params()
    x = sc.positions()
    g = Particles(p, sc.n)
    g.upload(x)
    r = RefSim(p, sc.n)
    r.set_state(x)
    check_bars(averaged_stats(g, g.stats), averaged_stats(r, lambda: r.stats(p)), REF_BUILD_BARS)


# ---------------------------------------------------------------- variants
def test_neighbor_cap_64_bit_exact():
    sc, p, g, o = pair(make_scene("dam_8k", neighbor_cap=64))
    g.step(3)
    o.step(3)
    assert_lists_equal(g, o, 64)
    assert_arrays(g, o, which=(ARRAY_POSITIONS, ARRAY_VELOCITIES))


def test_scorr_matches_oracle():
    sc, p, g, o = pair(make_scene("dam_2k", scorr=(0.1, 4.0, 0.2)), exact=1)
    g.step(2)
    o.step(2)
    np.testing.assert_allclose(g.positions(), o.get(ARRAY_POSITIONS), rtol=0, atol=REL_TOL * max(sc.box_max))


def test_surface_tension_bit_exact():
    sc, p, g, o = pair(make_scene("dam_2k", gamma=600.0))
    g.step(3)
    o.step(3)
    assert_arrays(g, o, which=(ARRAY_POSITIONS, ARRAY_VELOCITIES, ARRAY_DENSITIES, ARRAY_SCRATCH))
    sc, p, g, o = pair(make_scene("dam_2k", gamma=600.0))
    for i in range(3):
        [g.apply_external_forces, g.predict_positions, g.find_neighbors][i]()
        o.stage(i)
    g.compute_densities(); o.stage(3)
    g.apply_surface_tension(); o.stage(8)
    assert_arrays(g, o, which=(ARRAY_VELOCITIES, ARRAY_SCRATCH))


def test_mover_sphere_push():
    """apply_boundary_conditions (particles.h:514-522) with the mover inside the fluid."""
    sc, p, g, o = pair(make_scene("dam_2k", mover_center=(4.0, 2.0, 2.0)))
    g.step(2)
    o.step(2)
    assert_arrays(g, o, which=(ARRAY_POSITIONS, ARRAY_VELOCITIES))


# ---------------------------------------------------------------- edge cases and errors
def test_empty_and_single_particle():
    sc = make_scene("dam_2k")
    p = sc.params()
    g = Particles(p, 16)
    g.upload(np.zeros((0, 3), np.float32))
    g.step(3)
    assert g.local_count() == 0
    assert g.stats()["n"] == 0
    one = np.array([[3.0, 3.0, 3.0]], np.float32)
    g.upload(one)
    o = OracleSim(p, 16)
    o.set_state(one)
    g.step(2)
    o.step(2)
    assert np.array_equal(g.positions(), o.get(ARRAY_POSITIONS))
    idx, cnt = g.neighbors(p.neighbor_cap)
    assert cnt.tolist() == [0]


def test_errors_are_reported_not_faulted():
    sc = make_scene("dam_2k")
    p = sc.params()
    g = Particles(p, 100)
    with pytest.raises(RuntimeError, match="capacity"):
        g.upload(np.zeros((101, 3), np.float32))
    g.upload(sc.positions()[:100])
    with pytest.raises(RuntimeError, match="span"):
        g.apply_external_forces((10, 50))   # spans start at 0
    with pytest.raises(RuntimeError, match="span"):
        g.apply_external_forces((0, 101))   # past the held particles
    with pytest.raises(RuntimeError, match="neighbor lists"):
        g.compute_densities()
    g.find_neighbors()
    g.compute_densities()
    st = g.stats()
    assert st["error_flags"] == 0


def test_all_particles_in_one_cell():
    """Degenerate input: every particle at the same wall corner (coincident
    neighbours trigger the density nudge of particles.h:303-305)."""
    sc = make_scene("dam_2k")
    p = sc.params()
    x = np.zeros((100, 3), np.float32)
    v = np.tile(np.array([[0.5, -1.0, 0.25]], np.float32), (100, 1))
    g = Particles(p, 100)
    o = OracleSim(p, 100)
    g.upload(x, v)
    o.set_state(x, v)
    for i, fn in enumerate((g.apply_external_forces, g.predict_positions, g.find_neighbors)):
        fn()
        o.stage(i)
    assert_lists_equal(g, o, p.neighbor_cap)
    gi, gc = g.neighbors(p.neighbor_cap)
    assert gc.min() == 60


def _bin_face_positions(sc, s, frac=0.25, seed=5):
    """The jittered lattice with a share of its coordinates moved to values
    just below a bin face where the float re-hash of c - s, c, c + s
    (floor((v + s)/s) in float32, neighbors.h:109-114 and 172-185) does not
    give three consecutive bins.  Returns the positions and how many
    particles re-hash that way."""
    f = np.float32
    s = f(s)

    def axis_bin(v):
        return np.floor(f(f(v + s) / s))

    def rehash(c):
        return axis_bin(f(c - s)), axis_bin(c), axis_bin(f(c + s))

    quirks = set()
    for k in range(int(max(sc.box_max) / s) + 1):  # a few ulps either side of every face k*s
        for direction in (-np.inf, np.inf):
            v = f(f(k) * s)
            for _ in range(8):
                v = np.nextafter(v, f(direction), dtype=np.float32)
                b0, b1, b2 = rehash(v)
                if v > 0 and not (b0 + 1 == b1 and b1 + 1 == b2):
                    quirks.add(float(v))
    quirks = np.array(sorted(quirks), np.float32)
    assert quirks.size > 0
    x = sc.positions()
    rng = np.random.default_rng(seed)
    for a in range(3):
        for i in np.flatnonzero(rng.random(x.shape[0]) < frac):
            d = np.abs(quirks - x[i, a])
            j = int(np.argmin(d))
            if d[j] < 0.3 and quirks[j] < sc.box_max[a]:
                x[i, a] = quirks[j]
    b0, b1, b2 = rehash(x)
    odd = ~((b0 + 1 == b1) & (b1 + 1 == b2)).all(axis=1)
    return x, int(odd.sum())


def test_lists_at_bin_faces_bit_exact():
    """Particles whose float re-hash skips or repeats a bin walk their own 27
    bins; the others of their bin share one sweep of the bin's neighbourhood.
    Lists bit-exact against the oracle, in exact and in fast math."""
    sc = make_scene("dam_8k", gravity=0.0)
    x, odd = _bin_face_positions(sc, sc.params().neighbor_bin_spacing)
    assert odd > 200, odd
    for exact in (1, 0):
        p = sc.with_(exact_math=exact).params()
        g = Particles(p, sc.n)
        o = OracleSim(p, sc.n)
        g.upload(x)
        o.set_state(x)
        for i, fn in enumerate((g.apply_external_forces, g.predict_positions, g.find_neighbors)):
            fn()
            o.stage(i)
        assert np.array_equal(g.get_array(ARRAY_POSITION_STARS), x)  # the lists are built on these very values
        assert_lists_equal(g, o, p.neighbor_cap)


def _crowded_corner_positions(sc, seed=9):
    """The jittered lattice with a collapsed corner: every third particle of
    the first 6,000 piled onto one point near the box corner, and every third
    one after it (of the first 600) scattered inside the same bin, so the
    corner bin holds about 2,200 particles whose bit-identical runs are broken
    by distinct ones in index order."""
    x = sc.positions()
    rng = np.random.default_rng(seed)
    x[0:6000:3] = (0.05, 0.05, 0.05)
    k = len(range(1, 600, 3))
    x[1:600:3] = rng.uniform(0.0, 0.6, (k, 3)).astype(np.float32)
    return x


def test_crowded_corner_runs_bit_exact():
    """A bin of thousands of particles, most of them on one point: the fill
    decides each run of identical positions with one distance test.  Lists
    bit-exact against the oracle (stages, exact and fast math), and the fused
    exact step stays bit-identical to the oracle."""
    sc = make_scene("dam_8k")
    x = _crowded_corner_positions(sc)
    for exact in (1, 0):
        p = sc.with_(exact_math=exact).params()
        g = Particles(p, sc.n)
        o = OracleSim(p, sc.n)
        g.upload(x)
        o.set_state(x)
        for i, fn in enumerate((g.apply_external_forces, g.predict_positions, g.find_neighbors)):
            fn()
            o.stage(i)
        b = g.bins()
        assert (b["bin_end"].astype(np.int64) - b["bin_begin"]).max() > 2000  # the crowded bin is there
        assert_lists_equal(g, o, p.neighbor_cap)
    sc2, p, g, o = pair(sc)
    g.upload(x)
    o.set_state(x)
    g.step(3)
    o.step(3)
    assert_arrays(g, o, which=(ARRAY_POSITIONS, ARRAY_VELOCITIES, ARRAY_DENSITIES))
    assert_lists_equal(g, o, p.neighbor_cap)


def _coincident_scene():
    sc = make_scene("dam_2k")
    x = sc.positions()
    x[1::97] = x[0::97][: x[1::97].shape[0]]  # every 97th particle sits exactly on its predecessor
    v = np.zeros_like(x)
    v[:, 1] = -0.5
    v[::5, 0] = 0.25
    return sc, x, v


def test_coincident_particles_nudge_fused_bit_exact():
    """compute_densities' nudge of a particle sitting on a neighbour
    (particles.h:303-305), deterministic order, through the fused step."""
    sc, x, v = _coincident_scene()
    p = sc.with_(exact_math=1).params()
    g = Particles(p, sc.n)
    o = OracleSim(p, sc.n)
    g.upload(x, v)
    o.set_state(x, v)
    g.step(3)
    o.step(3)
    assert_arrays(g, o, which=(ARRAY_POSITIONS, ARRAY_VELOCITIES, ARRAY_DENSITIES, ARRAY_LAMBDAS))


def test_coincident_particles_nudge_stages_bit_exact():
    sc, x, v = _coincident_scene()
    p = sc.with_(exact_math=1).params()
    g = Particles(p, sc.n)
    o = OracleSim(p, sc.n)
    g.upload(x, v)
    o.set_state(x, v)
    for i, fn in enumerate((g.apply_external_forces, g.predict_positions, g.find_neighbors)):
        fn()
        o.stage(i)
    g.compute_densities(); o.stage(3)
    assert_arrays(g, o, which=(ARRAY_POSITION_STARS, ARRAY_DENSITIES))
    g.compute_pressure_lambdas(); o.stage(4)
    assert_arrays(g, o, which=(ARRAY_LAMBDAS,))


def test_timing_api_counts_every_kernel():
    sc = make_scene("dam_2k")
    g = Particles(sc.params(), sc.n)
    g.upload(sc.positions())
    g.set_timing(True)
    g.step(2)
    t = g.kernel_times()
    g.set_timing(False)
    launches = sum(v["launches"] for v in t.values())
    assert launches == 2 * g.launches_per_step()
    assert t["density_lambda"]["launches"] == 2 * sc.solve_steps
    assert all(v["total_ms"] > 0 for v in t.values())
