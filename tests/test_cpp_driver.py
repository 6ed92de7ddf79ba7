"""The C++ facade (include/pbf_particles.hpp) and the headless driver built on
it (sph-cpp_b200/apps/pbf_run.cpp), which runs the reference's main.cpp stage
loop verbatim.  CPU: the driver links against the library.  GPU: the per-stage
loop and the fused graph step give bit-identical states in exact mode."""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
APP = ROOT / "sph-cpp_b200" / "lib" / "pbf_run"

INI = """[SimParameters]
number_solve_steps = 3
time_step = 0.016
max_particles_local = 4096
exact_math = 1

[PhysicalParameters]
g = -9.8
gamma = 0.0
visc_c = 0.01
lambda_epsilon = 600.0
vorticity_coef = 0.0005
smoothing_radius = 1.0
rest_spacing = 0.5

[Boundary]
min = 0.0, 0.0, 0.0
max = 13.0, 13.0, 13.0

[InitialFluid]
min = 0.0, 0.0, 0.0
max = 8.0, 8.0, 4.0

[Mover]
center = -1.5, -2.0, -1.5
"""


def _build_module():
    import importlib.util
    spec = importlib.util.spec_from_file_location("pbf_build", ROOT / "sph-cpp_b200" / "build.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_driver_links_against_the_library():
    if not APP.exists():
        pytest.skip("the driver is built by sph-cpp_b200/build.py (build_app)")
    out = subprocess.run(["ldd", str(APP)], capture_output=True, text=True).stdout
    line = [l for l in out.splitlines() if "libpbf_b200" in l]
    assert line and "not found" not in line[0]


def test_facade_header_compiles_standalone(tmp_path):
    src = tmp_path / "t.cpp"
    src.write_text('#include "pbf_particles.hpp"\n'
                   'struct RefSpan { std::size_t begin, end; };\n'
                   'void f(sim::gpu::Particles& p) { RefSpan s{0, p.local_count()}; p.apply_external_forces(s);\n'
                   '  p.find_neighbors(s, s); p.compute_pressure_dps(s, 0); }\n')
    r = subprocess.run(["/usr/bin/g++", "-std=c++17", "-c", str(src), "-I", str(ROOT / "include"), "-o",
                        str(tmp_path / "t.o")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_facade_takes_the_reference_index_span(tmp_path):
    """The facade's stage methods accept the reference's own IndexSpan
    (Vec<std::size_t, 2> with begin/end members, Common/vec.h:114-121, 706):
    the reference's main.cpp loop body compiles against it unchanged."""
    ref = _build_module().REF_SOURCES
    if not (ref / "Common" / "vec.h").exists():
        pytest.skip("the reference's sources are not on this machine")
    src = tmp_path / "t.cpp"
    src.write_text('#include "vec.h"\n#include "pbf_particles.hpp"\n'
                   'void f(sim::gpu::Particles& particles, sim::gpu::Parameters& parameters) {\n'
                   '  IndexSpan local_span{0, particles.local_count()};\n'
                   '  IndexSpan resident_span{0, particles.local_count()};\n'
                   '  particles.apply_external_forces(local_span);\n'
                   '  particles.predict_positions(local_span);\n'
                   '  particles.find_neighbors(local_span, resident_span);\n'
                   '  for (int sub = 0; sub < (int)parameters.solve_step_count(); sub++) {\n'
                   '    particles.compute_densities(local_span);\n'
                   '    particles.compute_pressure_lambdas(local_span);\n'
                   '    particles.compute_pressure_dps(local_span, sub);\n'
                   '    particles.update_position_stars(local_span);\n'
                   '  }\n'
                   '  particles.update_velocities(local_span);\n'
                   '  particles.apply_surface_tension(resident_span, local_span);\n'
                   '  particles.apply_viscosity(local_span);\n'
                   '  particles.compute_vorticity(local_span);\n'
                   '  particles.apply_vorticity(local_span);\n'
                   '  particles.apply_viscosity(local_span);\n'
                   '  particles.update_positions(local_span);\n'
                   '}\n')
    r = subprocess.run(["/usr/bin/g++", "-std=c++17", "-c", str(src), "-I", str(ROOT / "include"), "-I",
                        str(ref / "Common"), "-o", str(tmp_path / "t.o")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def _run(tmp_path, fused: bool):
    ini = tmp_path / "dam.ini"
    ini.write_text(INI)
    dump = tmp_path / ("fused.bin" if fused else "stages.bin")
    cmd = [str(APP), str(ini), "5", "--jitter", "0.005", "--seed", "7", "--dump", str(dump)]
    if fused:
        cmd.append("--fused")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    raw = dump.read_bytes()
    n = int(np.frombuffer(raw[:8], np.uint64)[0])
    arr = np.frombuffer(raw[8:], np.float32)
    return n, arr[:3 * n].reshape(n, 3), arr[3 * n:].reshape(n, 3), r.stdout


@pytest.mark.gpu
def test_stage_loop_equals_fused_step(tmp_path):
    n1, x1, v1, out1 = _run(tmp_path, fused=False)
    n2, x2, v2, out2 = _run(tmp_path, fused=True)
    assert n1 == n2 == 16 * 16 * 8
    assert np.array_equal(x1, x2)
    assert np.array_equal(v1, v2)
    assert "flags 0" in out1 and "flags 0" in out2


@pytest.mark.gpu
def test_driver_save_resume_and_frames(tmp_path):
    """--save / --resume through state files: 4 + 3 resumed steps equal 7
    straight steps bit for bit; --frames writes one state file per K steps."""
    ini = tmp_path / "dam.ini"
    ini.write_text(INI)

    def run(*args):
        r = subprocess.run([str(APP), str(ini), *map(str, args)], capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, r.stdout + r.stderr
        return r.stdout

    run(7, "--fused", "--jitter", "0.005", "--seed", "7", "--dump", tmp_path / "straight.bin")
    run(4, "--fused", "--jitter", "0.005", "--seed", "7", "--save", tmp_path / "mid.pbf",
        "--frames", 2, tmp_path / "frame")
    run(3, "--fused", "--resume", tmp_path / "mid.pbf", "--dump", tmp_path / "resumed.bin")
    a = (tmp_path / "straight.bin").read_bytes()
    b = (tmp_path / "resumed.bin").read_bytes()
    assert a == b
    frames = sorted(p.name for p in tmp_path.glob("frame_*.pbf"))
    assert frames == ["frame_000000.pbf", "frame_000002.pbf"]
    assert (tmp_path / "frame_000002.pbf").read_bytes()[:8] == b"PBFSTATE"
