"""bench.py with more than one rank, on CPU.

The PBF step does not shard in this build (replicas only: every rank runs
its own scene on its own GPU), so the multi-rank part of bench.py is its
plumbing: the rank group's barrier and max-over-ranks reduction (the device
times of all ranks are reported as the slowest rank's), and the reference
arm, which rank 0 alone runs and prints while the other ranks exit 0
without work.  Both run here at world size 2 on gloo, no GPU needed.
"""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, str(ROOT))
    import bench
    group = bench.RankGroup(world, backend="gloo", device="cpu", timeout_s=60)
    group.barrier()
    slowest = group.max(1.0 + 10.0 * rank)  # rank r "took" 1 + 10 r seconds
    group.barrier()
    group.close()
    out.put((rank, slowest))


def test_rank_group_reports_the_slowest_rank():
    import torch.multiprocessing as mp
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == {0: 11.0, 1: 11.0}


def test_single_rank_group_makes_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench
    group = bench.RankGroup(1)
    assert group.dist is None
    group.barrier()
    assert group.max(3.5) == 3.5
    group.close()


def test_reference_arm_under_torchrun_prints_once_from_rank_0():
    if not (ROOT / "oracle" / "_ref" / "libpbf_ref.so").exists():
        pytest.skip("the reference build (oracle/_ref) is absent")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), str(ROOT / "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--scene", "dam_8k"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-3000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "reference" and d["e2e"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
