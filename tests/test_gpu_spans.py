"""Per-stage calls over resident spans, as a multi-rank driver makes them
(Simulation/Source/main.adios): the particles of reference index below the
span's end are updated, the others (halo particles) are read as neighbours
and left as they are, and find_neighbors bins every particle but fills
lists for the fill span only.  Checked in exact math against the reference's
own build driven over the same spans (oracle/ref_engine.py): bit for bit up
to the velocity update, within a tolerance after the XSPH passes (the
reference updates velocities in place, in particle order; the GPU reads the
old ones, Jacobi)."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from pbf_b200 import Particles, make_scene

ROOT = Path(__file__).resolve().parents[1]
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (ROOT / "oracle" / "_ref" / "libpbf_ref_serial.so").exists(),
                                 reason="the reference build (oracle/_ref) is absent")]

POS, PST, VEL, SCR, RHO, LAM = range(6)


def _pair(resident: int):
    from oracle.ref_engine import RefEngine
    from oracle.ref_scene import WORKLOADS
    sc = make_scene("dam_2k", exact_math=1)
    p = sc.params()
    x = sc.positions()
    v = np.zeros_like(x)
    v[:, 0] = 0.7  # a sideways drift, so the halo particles' v matter
    g = Particles(p, sc.n)
    g.upload(x, v)
    ref = RefEngine(WORKLOADS["dam_2k"], capacity=sc.n, rest_density=float(p.rest_density))
    ref.append(x, x, v)
    return sc, g, ref, x, v


def _both(g, ref, name, *args):
    getattr(g, name)(*args)
    getattr(ref, name)(*args)


@pytest.mark.parametrize("resident", [1500, 2048])
def test_resident_spans_match_the_reference(resident):
    sc, g, ref, x0, v0 = _pair(resident)
    n = sc.n
    res, loc = (0, resident), (0, n)
    try:
        _both(g, ref, "apply_external_forces", res)
        _both(g, ref, "predict_positions", res)
        _both(g, ref, "find_neighbors", loc, res)
        idx, cnt = g.neighbors(60)
        ridx = np.full((n, 60), -1, np.int32)
        rcnt = np.empty(n, np.int32)
        import ctypes as C
        ref.lib.ref_get_neighbors(ref.h, ridx.ctypes.data_as(C.c_void_p), rcnt.ctypes.data_as(C.c_void_p), 60)
        assert np.array_equal(cnt[:resident], rcnt[:resident])
        live = np.arange(60)[None, :] < cnt[:resident, None]
        assert np.array_equal(np.where(live, idx[:resident], -1), np.where(live, ridx[:resident], -1))
        assert (cnt[resident:] == 0).all()  # halo particles get no list
        for sub in range(sc.solve_steps):
            _both(g, ref, "compute_densities", res)
            _both(g, ref, "compute_pressure_lambdas", res)
            _both(g, ref, "compute_pressure_dps", res, sub)
            _both(g, ref, "update_position_stars", res)
        _both(g, ref, "update_velocities", loc)
        for w in (POS, PST, VEL):
            a, b = g.get_array(w), ref.get_array(w)
            assert np.array_equal(a, b), w
        for w in (RHO, LAM):
            a, b = g.get_array(w), ref.get_array(w)
            assert np.array_equal(a[:resident], b[:resident]), w
        # halo particles: x and x* unchanged by the resident-span stages
        assert np.array_equal(g.get_array(POS)[resident:], x0[resident:])
        assert np.array_equal(g.get_array(PST)[resident:], x0[resident:])
        # the driver refreshes the halo densities before XSPH divides by them
        # (main.adios); here both engines get the same stand-in values
        if resident < n:
            rho0 = float(sc.params().rest_density)
            for eng in (g, ref):
                r = eng.get_array(RHO)
                r[resident:] = rho0
                eng.set_array(RHO, r)
        _both(g, ref, "apply_viscosity", res)
        _both(g, ref, "compute_vorticity", res)
        _both(g, ref, "apply_vorticity", res)
        _both(g, ref, "apply_viscosity", res)
        _both(g, ref, "update_positions", res)
        v_g, v_r = g.get_array(VEL), ref.get_array(VEL)
        assert np.abs(v_g - v_r).max() <= 1e-3 * np.abs(v_r).max()
        assert np.array_equal(g.get_array(POS), ref.get_array(POS))
        if resident < n:  # halo velocities are the update_velocities ones (local span), untouched after
            vh = g.get_array(VEL)[resident:]
            assert np.array_equal(vh, ref.get_array(VEL)[resident:])
        assert g.stats()["error_flags"] == 0
    finally:
        g.close()
        ref.close()


def test_span_rules():
    sc = make_scene("dam_2k")
    with Particles(sc.params(), sc.n) as g:
        g.upload(sc.positions())
        with pytest.raises(RuntimeError, match="span"):
            g.find_neighbors((0, 1000), (0, 1000))  # binning leaves out particles
        g.find_neighbors((0, sc.n), (0, 1000))
        _, cnt = g.neighbors(60)
        assert (cnt[1000:] == 0).all() and (cnt[:1000] > 0).all()
        with pytest.raises(RuntimeError, match="span"):
            g.compute_densities((5, 1000))


def test_one_slab_distributor_steps_as_the_fused_step():
    """The slab distributor on one rank drives the GPU context through its
    per-stage calls (spans, the partitions' reordering, appends and
    removals): its steps equal the fused, graph-captured step particle by
    particle (matched by their identifiers), within the summation-order
    tolerance (the partitions reorder the particles, hence the lists)."""
    import datetime
    import socket

    import torch.distributed as dist

    from pbf_b200.slabs import SlabDistributor, Transport
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        sc = make_scene("dam_2k", exact_math=1)
        p = sc.params()
        x = sc.positions()
        with Particles(p, sc.n) as g, Particles(p, sc.n) as f:
            d = SlabDistributor(Transport(), edge_width=1.2 * p.smoothing_radius)
            d.set_domain_bounds(0.0, sc.fluid_max[0], 0.0, sc.box_max[0])
            g.upload(x)
            d.adopt(g, np.arange(sc.n))
            for _ in range(3):
                d.step(g, sc.solve_steps)
            f.upload(x)
            f.step(3)
            assert np.array_equal(np.sort(d.ids), np.arange(sc.n))
            order = np.argsort(d.ids)
            xg, xf = g.get_array(POS)[order], f.get_array(POS)
            vg, vf = g.get_array(VEL)[order], f.get_array(VEL)
            assert np.abs(xg - xf).max() <= 1e-5 * max(sc.box_max)
            assert np.abs(vg - vf).max() <= 1e-3 * np.abs(vf).max()
    finally:
        dist.destroy_process_group()
