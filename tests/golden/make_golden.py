"""Generate the golden vectors under tests/golden/ from the reference itself.

The reference's own particles.h / neighbors.h, compiled from its sources by
oracle/ref_build/Makefile (Thrust CPP system: serial, deterministic), run
over [0, N) as its serial tests drive Particles.  Run in a checkout where the
reference sources exist:

    python sph-cpp_b200/build.py && python tests/golden/make_golden.py

Outputs (numpy .npz, compressed):
  dam_2k_step1.npz    2,048-particle dam: input x, then after one full step
                      the sorted ids, bin bounds, neighbor lists (int16),
                      counts, x*, rho, lambda, scratch and, after step one, x
                      and v; plus x* after predict and lists/rho/lambda/dp of
                      the first Jacobi iteration
  dam_2k_traj.npz     statistics after each of 20 steps
  dam_8k_stats.npz    statistics after 50 steps of an 8,192-particle dam
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "sph-cpp_b200"))

from pbf_b200 import make_scene  # noqa: E402
from oracle.oracle import (ARRAY_DENSITIES, ARRAY_LAMBDAS, ARRAY_POSITION_STARS, ARRAY_POSITIONS,  # noqa: E402
                           ARRAY_SCRATCH, ARRAY_VELOCITIES, RefSim)


def _stats_row(st: dict) -> list[float]:
    return [st["mean_density_error"], st["max_density_error"], st["kinetic_energy"], *st["center_of_mass"],
            st["mean_neighbors"], st["cap_hits"]]


def step1(name: str) -> None:
    sc = make_scene(name)
    p = sc.params()
    x0 = sc.positions()
    r = RefSim(p, sc.n, serial=True)
    r.set_state(x0)
    out = {"x0": x0, "rest_density": np.float32(p.rest_density)}
    r.stage(0)
    r.stage(1)
    out["xs_pred"] = r.get(ARRAY_POSITION_STARS)
    r.stage(2)
    idx, cnt = r.neighbors()
    b = r.bins()
    out["nbr"] = idx.astype(np.int16)
    out["cnt"] = cnt.astype(np.int16)
    out["sorted_ids"] = b["sorted_ids"].astype(np.uint32)
    out["sorted_keys"] = b["sorted_keys"].astype(np.uint32)
    out["bin_begin"] = b["bin_begin"].astype(np.uint32)
    out["bin_end"] = b["bin_end"].astype(np.uint32)
    for sub in range(p.solve_steps):
        r.stage(3, sub)
        r.stage(4, sub)
        r.stage(5, sub)
        if sub == 0:
            out["rho_it0"] = r.get(ARRAY_DENSITIES)
            out["lam_it0"] = r.get(ARRAY_LAMBDAS)
            out["dp_it0"] = r.get(ARRAY_SCRATCH)
        r.stage(6, sub)
    out["xs_solved"] = r.get(ARRAY_POSITION_STARS)
    out["rho"] = r.get(ARRAY_DENSITIES)
    out["lam"] = r.get(ARRAY_LAMBDAS)
    for i in range(7, 13):
        r.stage(i)
    out["x1"] = r.get(ARRAY_POSITIONS)
    out["v1"] = r.get(ARRAY_VELOCITIES)
    out["vort1"] = r.get(ARRAY_SCRATCH)
    np.savez_compressed(HERE / f"{name}_step1.npz", **out)
    print("wrote", name, {k: v.shape for k, v in out.items()})


def trajectory(name: str, steps: int, every: bool, fname: str) -> None:
    sc = make_scene(name)
    p = sc.params()
    r = RefSim(p, sc.n, serial=True)
    r.set_state(sc.positions())
    rows = []
    for s in range(steps):
        r.step(1)
        if every or s == steps - 1:
            rows.append(_stats_row(r.stats(p)))
    np.savez_compressed(HERE / fname, stats=np.array(rows, np.float64),
                        columns=np.array(["mean_err", "max_err", "ke", "cx", "cy", "cz", "mean_nbr", "cap_hits"]),
                        x_final=r.get(ARRAY_POSITIONS), steps=np.int32(steps))
    print("wrote", fname, rows[-1])


if __name__ == "__main__":
    step1("dam_2k")
    trajectory("dam_2k", 20, True, "dam_2k_traj.npz")
    trajectory("dam_8k", 50, False, "dam_8k_stats.npz")
