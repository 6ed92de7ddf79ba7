"""The C-ABI library without a GPU: it loads, exports every symbol
include/pbf.h declares, and its host-side parameter / scene code matches the
reference (derive_from_input, read_INI, construct_fluid, grid dims)."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from oracle.oracle import OracleSim, oracle_lib, ref_available, ref_lib, ref_params_from
from pbf_b200 import _abi, make_scene, params_init

ROOT = Path(__file__).resolve().parent.parent


def header_symbols() -> set[str]:
    text = "\n".join(p.read_text() for p in (ROOT / "include").glob("*.h"))
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(pbf_[a-z0-9_]+)\s*\(", text))


def test_library_exports_every_declared_symbol():
    lib = _abi.load()
    syms = header_symbols()
    assert len(syms) >= 40
    missing = [s for s in sorted(syms) if not hasattr(lib, s)]
    assert not missing, missing
    # and the ctypes table covers them all
    assert syms <= set(_abi.SIGNATURES), sorted(syms - set(_abi.SIGNATURES))


def test_params_derive_matches_reference_rules():
    p = params_init()
    p.time_step = 0.016
    p.solve_steps = 3
    p.smoothing_radius = -1.0
    p.neighbor_bin_spacing = -1.0
    assert _abi.load().pbf_params_derive(C.byref(p), 0.5, -1.0) == 0
    assert p.smoothing_radius == np.float32(1.8 * np.float32(0.5))
    assert p.neighbor_bin_spacing == np.float32(1.2 * np.float64(np.float32(0.9)))
    assert p.rest_density == np.float32(8.0)
    assert p.max_speed == np.float32(0.5 * np.float64(np.float32(0.9)) * 3 / np.float64(np.float32(0.016)))


@pytest.mark.skipif(not ref_available(True), reason="reference build not present")
def test_params_derive_bitwise_vs_reference():
    sc = make_scene("dam_65k")
    p = sc.params()
    q = params_init()
    for f in ("time_step", "solve_steps"):
        setattr(q, f, getattr(p, f))
    q.smoothing_radius = -1.0
    q.neighbor_bin_spacing = -1.0
    assert _abi.load().pbf_params_derive(C.byref(q), 0.5, -1.0) == 0
    rp = ref_params_from(q, 16)
    rp.smoothing_radius = -1.0
    rp.neighbor_bin_spacing = -1.0
    rp.rest_density = -1.0
    out = (C.c_float * 8)()
    assert ref_lib(True).ref_derived(C.byref(rp), out) == 0
    assert out[2] == q.smoothing_radius
    assert out[3] == q.neighbor_bin_spacing
    assert out[4] == q.rest_density
    assert out[6] == q.max_speed


def test_ini_reader_matches_parameters_test(tmp_path):
    """parameters_test.cpp:33-54 values through the product's INI reader."""
    from test_oracle_ref import PARAMS_TEST_INI
    ini = tmp_path / "params_test.ini"
    ini.write_text(PARAMS_TEST_INI)
    p = _abi.PbfParams()
    fmin = (C.c_float * 3)()
    fmax = (C.c_float * 3)()
    assert _abi.load().pbf_params_from_ini(str(ini).encode(), C.byref(p), fmin, fmax) == 0
    assert p.solve_steps == 4
    assert p.particle_rest_spacing == pytest.approx(0.03218, rel=1e-4)
    assert p.smoothing_radius == pytest.approx(1.8 * p.particle_rest_spacing, rel=1e-6)
    assert p.neighbor_bin_spacing == pytest.approx(1.2 * p.smoothing_radius, rel=1e-6)
    assert p.rest_density == pytest.approx(29999.99609, rel=1e-5)
    assert p.rest_mass == 1.0
    assert p.gravity == pytest.approx(-9.8)
    assert p.gamma == pytest.approx(600.0)
    assert p.lambda_epsilon == pytest.approx(10.0)
    assert p.visc_c == pytest.approx(0.03)
    assert p.time_step == pytest.approx(0.008)
    assert p.max_speed == pytest.approx(14.48234, rel=1e-5)
    assert p.vorticity_coef == pytest.approx(0.00001)
    assert list(p.boundary_max) == pytest.approx([1.5, 2.0, 1.5])
    assert list(fmax) == pytest.approx([1.0, 1.0, 1.0])
    assert list(p.mover_center) == pytest.approx([-1.5, -2.0, -1.5])


def test_ini_missing_file_is_an_error():
    p = _abi.PbfParams()
    assert _abi.load().pbf_params_from_ini(b"/nonexistent/params.ini", C.byref(p), None, None) == _abi.PBF_ERR_IO


@pytest.mark.parametrize("name", ["dam_2k", "dam_65k"])
def test_lattice_builder_matches_oracle(name):
    sc = make_scene(name)
    x = sc.positions()
    y = np.empty_like(x)
    oracle_lib().oracle_build_lattice((C.c_float * 3)(*sc.fluid_min), (C.c_int64 * 3)(*sc.lattice), sc.spacing,
                                      sc.jitter * sc.h, sc.seed, y.ctypes.data_as(C.c_void_p))
    assert np.array_equal(x, y)
    # jitter bounded by +-0.005h around the construct_fluid lattice
    base = np.empty_like(x)
    oracle_lib().oracle_build_lattice((C.c_float * 3)(*sc.fluid_min), (C.c_int64 * 3)(*sc.lattice), sc.spacing,
                                      0.0, 0, base.ctypes.data_as(C.c_void_p))
    d = np.abs(x - base)
    assert d.max() <= 0.005 * sc.h * 1.0001 and d.max() > 0.004 * sc.h


def test_rest_density_matches_oracle_lattice():
    sc = make_scene("dam_65k")
    p = sc.params()
    r = C.c_float()
    assert oracle_lib().oracle_lattice_rest_density(C.byref(p), sc.spacing, C.byref(r)) == 0
    assert r.value == p.rest_density
    # and equals the density of an interior particle of the scene's own unjittered lattice
    base = sc.with_(jitter=0.0)
    o = OracleSim(p, base.n)
    o.set_state(base.positions())
    o.stage(2)
    o.stage(3)
    rho = o.get(4)
    i = (32 * 32) * 32 + 32 * 16 + 16
    assert rho[i] == p.rest_density


@pytest.mark.skipif(not ref_available(True), reason="reference build not present")
@pytest.mark.parametrize("name", ["dam_65k", "dam_1m", "dam_16m"])
def test_grid_dims_match_reference(name):
    sc = make_scene(name)
    p = sc.params()
    d = (C.c_int64 * 3)()
    assert _abi.load().pbf_grid_dims(C.byref(p), d) == 0
    from oracle.oracle import RefSim
    q = make_scene(name).params()
    q.neighbor_cap = 60
    r = RefSim(q, 8, serial=True)
    assert tuple(d) == r.bin_dims()


def test_create_rejects_bad_parameters_before_touching_a_device():
    lib = _abi.load()
    ctx = C.c_void_p()
    p = make_scene("dam_2k").params()
    bad = _abi.PbfParams.from_buffer_copy(p)
    bad.boundary_min[0] = -1.0
    assert lib.pbf_create(C.byref(bad), 100, C.byref(ctx)) == _abi.PBF_ERR_PARAMS
    assert b"boundary min" in lib.pbf_create_error()
    bad = _abi.PbfParams.from_buffer_copy(p)
    bad.boundary_min[1] = 2.0  # grid sized by the extent but hashed from 0: the far wall's bins leave it
    assert lib.pbf_create(C.byref(bad), 100, C.byref(ctx)) == _abi.PBF_ERR_PARAMS
    bad = _abi.PbfParams.from_buffer_copy(p)
    bad.neighbor_cap = 65
    assert lib.pbf_create(C.byref(bad), 100, C.byref(ctx)) == _abi.PBF_ERR_PARAMS
    assert lib.pbf_create(C.byref(p), 0, C.byref(ctx)) == _abi.PBF_ERR_ARG
