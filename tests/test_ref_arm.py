"""bench.py's reference arm builds its workload from the reference build and
numpy alone (oracle/ref_scene.py), so its process never maps the product's
library, and that workload is the GPU arm's bit for bit: the same derived
parameters, the same rest density, the same jittered lattice and the same
`config`.  CPU only."""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "sph-cpp_b200"))

pytestmark = pytest.mark.skipif(not (ROOT / "oracle" / "_ref" / "libpbf_ref.so").exists(),
                                reason="the reference build (oracle/_ref) is absent")


@pytest.mark.parametrize("name", ["dam_2k", "dam_8k", "dam_65k"])
def test_reference_workload_equals_the_product_scene(name):
    from oracle.ref_scene import WORKLOADS, RefRun, derived
    from pbf_b200 import make_scene
    w, s = WORKLOADS[name], make_scene(name)
    assert (w.lattice, w.box_max, w.solve_steps, w.neighbor_cap) == (s.lattice, s.box_max, s.solve_steps,
                                                                      s.neighbor_cap)
    assert (w.h, w.spacing, w.gravity, w.time_step, w.lambda_epsilon, w.visc_c, w.vorticity_coef, w.gamma,
            w.jitter, w.seed, w.mover_center) == (s.h, s.spacing, s.gravity, s.time_step, s.lambda_epsilon,
                                                  s.visc_c, s.vorticity_coef, s.gamma, s.jitter, s.seed,
                                                  s.mover_center)
    p = s.params()
    d = derived(w)
    assert np.float32(d["neighbor_bin_spacing"]) == np.float32(p.neighbor_bin_spacing)
    assert np.float32(d["max_speed"]) == np.float32(p.max_speed)
    with RefRun(w) as run:
        assert np.float32(run.rho0) == np.float32(p.rest_density)
        x = run.get(0)
        assert np.array_equal(x, s.positions())
        assert np.array_equal(run.get(1), x)


def test_every_bench_workload_is_defined_for_both_arms():
    from oracle.ref_scene import WORKLOADS
    from pbf_b200 import SCENES
    assert set(WORKLOADS) == set(SCENES)
    for k, w in WORKLOADS.items():
        s = SCENES[k]
        assert (w.lattice, w.box_max, w.solve_steps, w.neighbor_cap) == (s.lattice, s.box_max, s.solve_steps,
                                                                          s.neighbor_cap)


def test_reference_arm_maps_only_the_reference_build():
    """Run the arm as the driver does; its line lists the repository's
    libraries mapped into its process, and the product's is not among them.
    Its config is the GPU arm's for the same workload."""
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--scene", "dam_2k",
                        "--steps", "2", "--warmup", "1"], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["libraries_mapped"] == ["oracle/_ref/libpbf_ref.so"]
    import bench
    from pbf_b200 import make_scene
    s = make_scene("dam_2k")
    assert d["config"] == bench.workload_config(s.name, s.n, s.lattice, s.box_max, s.solve_steps,
                                                s.lambda_epsilon, s.neighbor_cap, 1)
    assert d["steps"] == 2 and d["warmup"] == 1 and d["value"] > 0


def test_reference_arm_module_imports_nothing_of_the_product():
    code = ("import sys; sys.path.insert(0, %r); import bench; from oracle import ref_scene; "
            "ref_scene.RefRun(ref_scene.WORKLOADS['dam_2k']).close(); "
            "mods = [m for m in sys.modules if m.split('.')[0] == 'pbf_b200']; "
            "maps = open('/proc/self/maps').read(); "
            "assert not mods, mods; assert 'libpbf_b200' not in maps; print('ok')") % str(ROOT)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120, cwd=ROOT)
    assert r.returncode == 0 and "ok" in r.stdout, r.stderr[-2000:]
