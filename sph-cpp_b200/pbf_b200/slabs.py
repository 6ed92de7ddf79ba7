"""Multi-rank x-slab decomposition of one scene.

The reference's `Distributor` (Simulation/Source/distributor.h) splits the
scene into slabs along x, one per rank: each rank holds its resident
particles, ordered [interior | edge-left | edge-right], followed by halo
particles (the neighbouring slabs' edge particles) [halo-left | halo-right].
Each step it migrates out-of-bounds particles to the neighbouring slab,
rebuilds the halos, and refreshes the halo values each stage reads
(Simulation/Source/main.adios: lambda and x* after every Jacobi iteration,
then density, velocity and vorticity).

`SlabDistributor` is that scheme, B200-side: one process per GPU, the
neighbour exchanges as torch.distributed point-to-point messages (counts
first, then the rows), so that rows land in the receiving GPU's own memory
(NCCL with CUDA tensors) or host memory (gloo with CPU tensors).  There are
no peer loads, no TMA and no multicast: every rank computes on its own copy.
It drives any engine with the reference's `Particles` stage surface over
spans ([0, e) = the resident or the local particles): `pbf_b200.Particles`
on a GPU (its per-stage calls honour resident spans, include/pbf.h), or the
reference's own build on CPU in the tests.

Engine methods used: local_count(), get_array(which), set_array(which, a),
append(x, x_star, v), remove(k), construct_fluid(min, max, velocity) and the
stage methods apply_external_forces ... update_positions taking spans.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

# array identifiers of the engines (include/pbf.h PBF_ARRAY_*)
POSITIONS, POSITION_STARS, VELOCITIES, SCRATCH, DENSITIES, LAMBDAS = range(6)


class Transport:
    """Neighbour exchange of one slab with the slabs to its left and right
    over torch.distributed (an initialised default process group).  Every
    rank calls `exchange` in the same order; counts travel first, so each
    receiver sizes its buffer exactly (NCCL needs both sides to agree)."""

    def __init__(self, device: str = "cpu"):
        import torch.distributed as dist
        self.dist = dist
        self.rank = dist.get_rank()
        self.size = dist.get_world_size()
        self.device = device

    @property
    def left(self) -> int | None:
        return self.rank - 1 if self.rank > 0 else None

    @property
    def right(self) -> int | None:
        return self.rank + 1 if self.rank < self.size - 1 else None

    def _pairs(self, sends: dict, recvs: dict) -> None:
        ops = []
        P2POp = self.dist.P2POp
        for peer, t in sends.items():
            ops.append(P2POp(self.dist.isend, t, peer))
        for peer, t in recvs.items():
            ops.append(P2POp(self.dist.irecv, t, peer))
        if ops:
            for r in self.dist.batch_isend_irecv(ops):
                r.wait()

    def exchange(self, to_left: np.ndarray, to_right: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        """Send rows to the left and right slabs, receive theirs (rows of the
        same trailing shape and dtype; an end slab's missing neighbour sends
        and receives nothing)."""
        import torch
        shape, dtype = to_left.shape[1:], to_left.dtype
        tdtype = torch.from_numpy(np.zeros(1, dtype)).dtype
        counts = {}
        sends, recvs = {}, {}
        for peer, rows in ((self.left, to_left), (self.right, to_right)):
            if peer is None:
                continue
            sends[peer] = torch.tensor([rows.shape[0]], dtype=torch.int64, device=self.device)
            counts[peer] = torch.zeros(1, dtype=torch.int64, device=self.device)
            recvs[peer] = counts[peer]
        self._pairs(sends, recvs)
        sends, recvs, bufs = {}, {}, {}
        for peer, rows in ((self.left, to_left), (self.right, to_right)):
            if peer is None:
                continue
            if rows.shape[0]:
                sends[peer] = torch.from_numpy(np.ascontiguousarray(rows)).to(self.device)
            k = int(counts[peer].item())
            if k:
                bufs[peer] = torch.empty((k, *shape), dtype=tdtype, device=self.device)
                recvs[peer] = bufs[peer]
        self._pairs(sends, recvs)
        empty = np.zeros((0, *shape), dtype)
        out = []
        for peer in (self.left, self.right):
            out.append(bufs[peer].cpu().numpy() if peer in bufs else empty)
        return out[0], out[1]

    def allreduce_sum(self, v: int) -> int:
        import torch
        t = torch.tensor([v], dtype=torch.int64, device=self.device)
        self.dist.all_reduce(t)
        return int(t.item())


@dataclass
class Counts:
    resident: int = 0
    edge_left: int = 0
    edge_right: int = 0
    halo_left: int = 0
    halo_right: int = 0
    oob_left: int = 0
    oob_right: int = 0


class SlabDistributor:
    """The reference's Distributor for one rank of a slab decomposition.
    `ids` carries a global identifier per local particle through migration
    (the reference keeps none; it lets results be gathered in a fixed
    order)."""

    def __init__(self, transport: Transport, edge_width: float):
        self.t = transport
        self.edge_width = float(edge_width)
        self.domain = [0.0, 0.0]
        self.c = Counts()
        self.last_sync = Counts()   # the counts after the last domain sync (halos included)
        self.ids = np.zeros(0, np.int64)

    # ---- ranks and spans (distributor.h:196-312) ----
    @property
    def rank(self) -> int:
        return self.t.rank

    def is_first_domain(self) -> bool:
        return self.t.rank == 0

    def is_last_domain(self) -> bool:
        return self.t.rank == self.t.size - 1

    def domain_to_left(self) -> int | None:
        return self.t.left

    def domain_to_right(self) -> int | None:
        return self.t.right

    def resident_count(self) -> int:
        return self.c.resident

    def edge_count(self) -> int:
        return self.c.edge_left + self.c.edge_right

    def halo_count(self) -> int:
        return self.c.halo_left + self.c.halo_right

    def interior_count(self) -> int:
        return self.c.resident - self.edge_count()

    def local_count(self) -> int:
        return self.c.resident + self.halo_count()

    def resident_span(self) -> tuple[int, int]:
        return (0, self.c.resident)

    def local_span(self) -> tuple[int, int]:
        return (0, self.local_count())

    def edge_span(self) -> tuple[int, int]:
        return (self.c.resident - self.edge_count(), self.c.resident)

    def halo_span(self) -> tuple[int, int]:
        return (self.c.resident, self.c.resident + self.halo_count())

    def interior_span(self) -> tuple[int, int]:
        return (0, self.interior_count())

    def global_resident_count(self) -> int:
        return self.t.allreduce_sum(self.c.resident)

    # ---- domains (distributor.h:105-184) ----
    def set_domain_bounds(self, fluid_min_x: float, fluid_max_x: float, boundary_min_x: float,
                          boundary_max_x: float) -> None:
        """Equal x-slabs of the initial fluid; the end slabs stretch to the boundary."""
        f = np.float32
        length = f(f(f(fluid_max_x) - f(fluid_min_x)) / f(self.t.size))
        begin = f(f(fluid_min_x) + f(self.t.rank) * length)
        self.domain = [float(begin), float(f(begin + length))]
        if self.is_last_domain():
            self.domain[1] = float(boundary_max_x)
        if self.is_first_domain():
            self.domain[0] = float(boundary_min_x)

    def balance_domains(self) -> None:
        """Move a shared boundary by 0.15 edge widths toward the slab with too
        many particles (more than 5% off the even share), keeping every slab
        at least 3 edge widths wide (distributor.h:134-184)."""
        f = np.float32
        even = self.global_resident_count() // self.t.size
        max_diff = int(even * 0.05)
        dx = float(f(f(self.edge_width) * f(0.15)))
        min_width = 3.0 * self.edge_width
        my = np.array([[self.c.resident]], np.int64)
        # the right slab's count and both neighbours' lengths
        _, right_count = self.t.exchange(my, my)
        mylen = np.array([[self.domain[1] - self.domain[0]]], np.float64)
        left_len, right_len = self.t.exchange(mylen, mylen)
        diff = self.c.resident - even
        if self.t.left is not None:
            ll = float(left_len[0, 0])
            if diff > max_diff and mylen[0, 0] > min_width:
                self.domain[0] += dx
            if diff < -max_diff and ll > min_width:
                self.domain[0] -= dx
        if self.t.right is not None:
            rd = int(right_count[0, 0]) - even
            rl = float(right_len[0, 0])
            if rd > max_diff and rl > min_width:
                self.domain[1] += dx
            if rd < -max_diff and mylen[0, 0] > min_width:
                self.domain[1] -= dx

    def distribute_fluid(self, engine, fluid_min, fluid_max, spacing: float, velocity=(0.0, 0.0, 0.0),
                         first_id: int = 0) -> int:
        """Fill this slab's part of the fluid box with the engine's lattice,
        keeping the global lattice spacing across slab boundaries
        (distributor.h:318-353).  Returns the particles added."""
        f = np.float32
        begin, end = f(self.domain[0]), f(self.domain[1])
        gmin, gmax = f(fluid_min[0]), f(fluid_max[0])
        starts = gmin >= begin and gmin <= end
        ends = gmax >= begin and gmax <= end
        filled = gmin <= begin and gmax >= begin
        if not (starts or ends or filled):
            return 0
        prev = max(f(0.0), f(math.floor(f(f(begin - gmin) / f(spacing)))))
        lo = list(fluid_min)
        hi = list(fluid_max)
        lo[0] = float(f(gmin + f(prev * f(spacing))))
        hi[0] = float(gmax if ends else end)
        added = engine.construct_fluid(lo, hi, velocity)
        self.ids = np.concatenate([self.ids, first_id + np.arange(added, dtype=np.int64)])
        self.c.resident += added
        return added

    def adopt(self, engine, ids: np.ndarray) -> None:
        """Take the engine's particles as this slab's residents (a caller that
        built its own initial set), with their global identifiers."""
        self.ids = np.asarray(ids, np.int64).copy()
        self.c = Counts(resident=engine.local_count())

    # ---- exchanges (distributor.h:379-736) ----
    def invalidate_halo(self, engine) -> None:
        engine.remove(self.halo_count())
        self.ids = self.ids[:self.c.resident]
        self.c.halo_left = self.c.halo_right = 0

    def _residents(self, engine):
        R = self.c.resident
        return (engine.get_array(POSITION_STARS)[:R], engine.get_array(POSITIONS)[:R],
                engine.get_array(VELOCITIES)[:R])

    def _reorder(self, engine, order: np.ndarray, xs, x, v) -> None:
        """Residents in `order` (the engine holds residents only here)."""
        engine.set_array(POSITIONS, x[order])
        engine.set_array(POSITION_STARS, xs[order])
        engine.set_array(VELOCITIES, v[order])
        self.ids = self.ids[order]

    @staticmethod
    def _pack(xs, x, v, ids) -> np.ndarray:
        return np.concatenate([xs, x, v, ids.view(np.float32).reshape(-1, 2)], axis=1)

    @staticmethod
    def _unpack(rows: np.ndarray):
        return (rows[:, 0:3], rows[:, 3:6], rows[:, 6:9],
                np.ascontiguousarray(rows[:, 9:11]).view(np.int64).reshape(-1))

    def domain_sync(self, engine) -> None:
        """Out-of-bounds migration, then the halo exchange (distributor.h:379-389);
        the halo of the previous step must have been invalidated."""
        if self.halo_count():
            raise RuntimeError("domain_sync: invalidate_halo first")
        self.oob_exchange(engine)
        self.halo_exchange(engine)
        self.last_sync = Counts(**vars(self.c))

    def oob_exchange(self, engine) -> None:
        """Residents whose x* left [begin, end] move to the slab on that side
        (distributor.h:544-641): arrays become {staying, oob-left, oob-right}, the
        leavers go, the arrivals are appended as residents (left's, then right's)."""
        xs, x, v = self._residents(engine)
        b, e = np.float32(self.domain[0]), np.float32(self.domain[1])
        px = xs[:, 0]
        stay = (px >= b) & (px <= e)
        left = ~stay & (px <= b)
        right = ~stay & ~left
        order = np.concatenate([np.nonzero(stay)[0], np.nonzero(left)[0], np.nonzero(right)[0]])
        self._reorder(engine, order, xs, x, v)
        xs, x, v, ids = xs[order], x[order], v[order], self.ids
        ns, nl = int(stay.sum()), int(left.sum())
        self.c.oob_left, self.c.oob_right = nl, int(right.sum())
        to_l = self._pack(xs[ns:ns + nl], x[ns:ns + nl], v[ns:ns + nl], ids[ns:ns + nl])
        to_r = self._pack(xs[ns + nl:], x[ns + nl:], v[ns + nl:], ids[ns + nl:])
        from_l, from_r = self.t.exchange(to_l, to_r)
        engine.remove(self.c.oob_left + self.c.oob_right)
        self.ids = self.ids[:ns]
        self.c.resident = ns
        for rows in (from_l, from_r):
            if rows.shape[0]:
                rxs, rx, rv, rid = self._unpack(rows)
                engine.append(rx, rxs, rv)
                self.ids = np.concatenate([self.ids, rid])
                self.c.resident += rows.shape[0]

    def halo_exchange(self, engine) -> None:
        """Residents within one edge width of a slab boundary are the edges,
        {interior, edge-left, edge-right}; each slab's edges become its
        neighbours' halos, appended after the residents (left's, then
        right's) (distributor.h:650-736)."""
        xs, x, v = self._residents(engine)
        el = np.float32(np.float32(self.domain[0]) + np.float32(self.edge_width))
        er = np.float32(np.float32(self.domain[1]) - np.float32(self.edge_width))
        px = xs[:, 0]
        interior = (px >= el) & (px <= er)
        left = ~interior & (px <= el)
        right = ~interior & ~left
        order = np.concatenate([np.nonzero(interior)[0], np.nonzero(left)[0], np.nonzero(right)[0]])
        self._reorder(engine, order, xs, x, v)
        xs, x, v, ids = xs[order], x[order], v[order], self.ids
        ni = int(interior.sum())
        self.c.edge_left, self.c.edge_right = int(left.sum()), int(right.sum())
        a, m = ni, ni + self.c.edge_left
        to_l = self._pack(xs[a:m], x[a:m], v[a:m], ids[a:m])
        to_r = self._pack(xs[m:], x[m:], v[m:], ids[m:])
        from_l, from_r = self.t.exchange(to_l, to_r)
        for rows, side in ((from_l, "left"), (from_r, "right")):
            if rows.shape[0]:
                rxs, rx, rv, rid = self._unpack(rows)
                engine.append(rx, rxs, rv)
                self.ids = np.concatenate([self.ids, rid])
            setattr(self.c, f"halo_{side}", rows.shape[0])

    def sync_halo(self, engine, which: int) -> None:
        """The halo rows of one array refreshed from their owners: edge-left
        rows go left, edge-right rows go right, and the received rows
        overwrite halo-left, then halo-right (distributor.h:391-448)."""
        a = engine.get_array(which)
        i0 = self.interior_count()
        i1 = i0 + self.c.edge_left
        R = self.c.resident
        rows_l, rows_r = a[i0:i1], a[i1:R]
        if a.ndim == 1:
            rows_l, rows_r = rows_l[:, None], rows_r[:, None]
        from_l, from_r = self.t.exchange(rows_l, rows_r)
        if from_l.shape[0] != self.c.halo_left or from_r.shape[0] != self.c.halo_right:
            raise RuntimeError("sync_halo: halo counts changed since the halo exchange")
        if self.halo_count() == 0:
            return
        h = np.concatenate([from_l, from_r])
        a = a.copy()
        a[R:R + self.halo_count()] = h[:, 0] if a.ndim == 1 else h
        engine.set_array(which, a)

    # ---- the step (Simulation/Source/main.adios) ----
    def step(self, engine, solve_steps: int, balance: bool = False, surface_tension: bool = False) -> None:
        """One time step of the multi-rank driver: the stages over resident
        or local spans, the domain sync after the prediction, and the halo
        refreshes of lambda, x*, density, velocity and vorticity.

        Surface tension (gamma != 0 only; with gamma = 0 the stage adds
        exactly zero and is skipped) runs over the resident span for both of
        its passes: the reference's driver passes the local span as the
        colour span, which reads the neighbour lists of halo particles, lists
        the fill span never builds."""
        res = self.resident_span()
        engine.apply_external_forces(res)
        engine.predict_positions(res)
        if balance:
            self.balance_domains()
        self.domain_sync(engine)
        res, loc = self.resident_span(), self.local_span()
        engine.find_neighbors(loc, res)
        for sub in range(solve_steps):
            engine.compute_densities(res)
            engine.compute_pressure_lambdas(res)
            self.sync_halo(engine, LAMBDAS)
            engine.compute_pressure_dps(res, sub)
            engine.update_position_stars(res)
            self.sync_halo(engine, POSITION_STARS)
            if surface_tension:
                engine.apply_surface_tension(res, res)
        engine.update_velocities(loc)
        self.sync_halo(engine, DENSITIES)
        if surface_tension:
            engine.apply_surface_tension(res, res)
        engine.apply_viscosity(res)
        self.sync_halo(engine, VELOCITIES)
        engine.compute_vorticity(res)
        self.sync_halo(engine, SCRATCH)
        engine.apply_vorticity(res)
        engine.apply_viscosity(res)
        engine.update_positions(res)
        self.invalidate_halo(engine)
