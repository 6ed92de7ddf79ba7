"""Benchmark of the B200 PBF step: particle-steps/s on the 1M-particle dam.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--scene dam_1m] [--impl reference]

One "step" is one full PBF time step (the stage order of the reference's
Simulation/Source/main.cpp:71-124) over the whole particle set.  Prints ONE
JSON line on rank 0.

  value        particle-steps/s of K graph-replayed steps, state resident in HBM,
               CUDA events on the library's stream, max over ranks
  e2e          the same metric through the public C ABI with host buffers:
               every step uploads x and v from pinned host memory, runs the
               step and downloads x and v
  roofline     the dominant kernel's algorithmic bytes per launch / its mean
               duration (CUDA events around each kernel of K eagerly launched
               steps on the library's stream), against the measured HBM copy
               bandwidth
  cpu_baseline the reference's own OpenMP build (oracle/_ref) on this host's
               cores, a bounded sample of the same workload, and the same on
               one thread
  tuning       the launch shapes (lanes per particle, threads per block) of the
               gather kernel families the library's autotuner picked during
               the warm-up (pbf_autotune; --no-autotune keeps the defaults)
Multi-GPU: the path does not shard in this build (replicas only): every rank
runs its own full scene on its own GPU; value sums the ranks' particle-steps
over the slowest rank's time.
`--impl reference` times the reference's CPU build instead (rank 0 only), on
the workload built from that build and numpy alone (oracle/ref_scene.py): its
process never loads the product's library, and its `config` is the GPU arm's.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
for _p in (ROOT, ROOT / "sph-cpp_b200"):
    if str(_p) not in sys.path:
        sys.path.insert(0, str(_p))

METRIC = "particle-steps/s at 1M (plain vs learned warm-start, equal density error)"
UNIT = "particle-steps/s"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--scene", default="dam_1m")
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--exact", action="store_true", help="exact_math=1 (bit-exact arithmetic)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the plain-vs-learned comparison")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="target length of the CPU baseline sample")
    ap.add_argument("--no-autotune", action="store_true", help="default launch shapes instead of the autotuner's")
    ap.add_argument("--no-batched", action="store_true", help="skip the 64-scene batch measurement")
    ap.add_argument("--profile-learned", type=int, default=0, metavar="K",
                    help="only run K steps of the learned warm start (eps 1, after its warm-up) and print "
                         "ms/step: the command the learned kernels' ncu summaries are captured from")
    ap.add_argument("--profile-training", type=int, default=0, metavar="K",
                    help="only record one 1M-dam step and run K Adam updates of the warm-start network "
                         "(batch 65,536) and print ms/update: the command the training kernel's ncu "
                         "summary is captured from")
    ap.add_argument("--residual-sample", type=int, default=1,
                    help="residual_sample of --profile-learned (1: full residual checks)")
    ap.add_argument("--learned-iterations", type=int, default=10,
                    help="iteration cap of --profile-learned (1: no conditional loop in the step's graph, "
                         "which ncu needs to profile the graph's kernels)")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the 16.8M dam, the 200-step trajectory and the s_corr run")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(
        os.environ.get("LOCAL_RANK", "0"))


class RankGroup:
    """The ranks of one run, one process per GPU (torchrun sets RANK,
    WORLD_SIZE, MASTER_ADDR/PORT): a barrier and the max of a value over the
    ranks (device times are reported as the max over ranks).  The bench uses
    NCCL on CUDA tensors; the same calls run on gloo with CPU tensors.  A
    single rank makes no process group and every call is a no-op.  The group
    has a short timeout, so that ranks waiting on a missing one end with an
    error."""

    def __init__(self, world: int, backend: str = "nccl", device: str = "cuda", timeout_s: float = 120.0):
        self.world = world
        self.device = device
        self.dist = None
        if world > 1:
            import datetime
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def barrier(self) -> None:
        if self.dist is not None:
            self.dist.barrier()

    def max(self, v: float) -> float:
        if self.dist is None:
            return v
        import torch
        t = torch.tensor([v], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self) -> None:
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (self.out or "").splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() in ("active", "1"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- algorithmic bytes
def kernel_bytes(name: str, n: int, nbar: float, K: int, nbins: int) -> float:
    """Compulsory DRAM bytes per launch of each kernel: each per-particle input
    read once, each output written once, int32 neighbor-list entries read once;
    gathered neighbour values counted as cache hits (they are re-reads of
    arrays already streamed by the same launch)."""
    L = 4.0 + 4.0 * nbar   # count + list
    per = {
        "ext_predict_hash": 16 + 16 + 16 + 16 + 4 + 4,           # x, v in; v, x*, key, rank out (+ histogram in L2)
        "scan_reduce": 4.0 * nbins / n,
        "scan_partials": 8.0 * nbins / n / 4096,                # one partial sum per scan tile of 4096 bins, read and written
        "scan_apply": 8.0 * nbins / n,
        "radix_hist": 4 + 2048.0 * 4 / 4096,                    # key in; per-tile digit counts out
        "radix_scan": 2048.0 * 4 / 4096,                        # digit counts (3 launches, per launch)
        "radix_scatter": 4 + 8 + 4 + 8,                         # key, pair in; key, pair out
        "warm_features": 16 + L + 16 + 16 + 4 + 16 + 32,       # x*, list, v, last lambda in; (x*, l1), v, bf16 features out
        "warm_mlp": 32 + 16 + 16 + 4 + 4,                       # features, (x*, l1) in; (x*, lambda), lambda, sum out
        "residual_check": 16 + L + 16 + 4 + 4,                  # as density_lambda
        "reorder": 8 + 4 + 3 * 16 + 3 * 16 + 4 + 4,             # pair, key, (x, x*, v) in and out, orig, key
        "runs": 16 + 4,                                         # x* in (the previous slot's is a cache hit); run end out
        "fill_neighbors": 16 + 4 * nbar + 4 + 8.0 * nbins / n + 32,  # own x*, list + count out, bin starts,
                                                                     # the visits' starts (seg) out
        "fill_redo": 4.0 * 5 / n,                               # the order words; its queue (capped slot-order
                                                                # lists, walked again) is empty unless lists reach the cap
        "density_lambda": 16 + L + 16 + 4 + 4,                  # x* in; list; (x*, lambda), rho, lambda out
        "lambda_fixup": 16 + L + 16 + 4,                        # exact math after a nudge: x* in, list; (x*, lambda), lambda out
        "dp_update": 16 + L + 16 + (32.0 / K),                  # (x*, lambda) in; list; x* out; last: x in, v out
        "viscosity": 16 + 16 + L + 16 + 2 * nbar,                # ...; v out and the weight of every entry (half)
        "vorticity": 16 + 16 + L + 16 + 16,
        "apply_vorticity": 16 + 16 + 16 + L + 16,
        "viscosity_final": 16 + 16 + L + 2 * nbar + 16 + 16 + 16 + 4 + 4,  # ...; the entries' weights in (half)
        "update_velocities": 16 + 16 + 16,
        # every gather pass of the step in one launch (pbf_set_persistent)
        "persistent_step": K * ((40 + L) + (32 + L)) + 32 + (48 + L + 2 * nbar) + (64 + L) + (64 + L)
                           + (96 + L + 2 * nbar),
        "color_field": 16 + 16 + L + 16,
        "surface_tension": 16 + 16 + 16 + L + 16,
    }
    return per.get(name, 0.0) * n


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def ncu_traffic(kernel: str, scene: str) -> float | None:
    """dram bytes per launch from a committed ncu summary, if one exists for this
    kernel and workload (profiles/<kernel>_<scene>.txt, line 'dram_bytes_per_launch: X')."""
    f = ROOT / "profiles" / f"{kernel}_{scene}.txt"
    if not f.exists():
        return None
    m = re.search(r"dram_bytes_per_launch:\s*([0-9.eE+]+)", f.read_text())
    return float(m.group(1)) if m else None


# ---------------------------------------------------------------- CPU reference
def workload_config(name: str, n: int, lattice, box, solve_steps: int, lambda_epsilon: float, neighbor_cap: int,
                    world: int) -> dict:
    """The `config` of both arms: the workload alone, nothing of either
    implementation (launch shapes, arithmetic mode) in it."""
    return {"workload": name, "particles": int(n), "lattice": [int(v) for v in lattice],
            "box": [float(v) for v in box], "solve_steps": int(solve_steps),
            "lambda_epsilon": float(lambda_epsilon), "neighbor_cap": int(neighbor_cap),
            "scorr": "off (reference has none)", "parallelism": f"replicas x{world}",
            "l2": "no flush: the per-step working set (neighbor lists ~230 MB + particle state) exceeds the 126 MB L2"}


def mapped_libraries() -> list[str]:
    """Shared libraries of this repository mapped into this process."""
    out = set()
    try:
        with open("/proc/self/maps") as f:
            for line in f:
                path = line.split()[-1] if len(line.split()) >= 6 else ""
                if path.endswith(".so") and path.startswith(str(ROOT)):
                    out.add(str(Path(path).relative_to(ROOT)))
    except OSError:
        pass
    return sorted(out)


def run_reference_cpu(name: str, steps: int, warmup: int, budget_s: float | None, threads: int | None = None) -> dict:
    """The reference's own OpenMP build (oracle/_ref) on `threads` host
    threads (all of them by default), on the workload built from that build
    and numpy alone (oracle/ref_scene.py)."""
    from oracle.ref_scene import WORKLOADS, all_cores, time_reference
    return time_reference(WORKLOADS[name], steps, warmup, threads or all_cores(), budget_s)


def reference_arm(args) -> int:
    """bench.py --impl reference: the reference's CPU build timed for the
    same workload and metric as the GPU arm (rank 0 alone; other ranks exit
    without work).  This process never loads the product's library."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from oracle.ref_scene import WORKLOADS, all_cores, time_reference
    w = WORKLOADS[args.scene]
    K, W = args.steps, args.warmup
    r = time_reference(w, K, W, all_cores())
    line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": r["steps"], "warmup": W, "ms_per_step": 1e3 * r["seconds"] / r["steps"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded jittered dam-break lattice, zero initial velocity)",
            "config": workload_config(w.name, w.n, w.lattice, w.box_max, w.solve_steps, w.lambda_epsilon,
                                      w.neighbor_cap, args.gpus),
            "cpu_baseline": {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": r["kind"],
                             "sample": r["sample"]},
            "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "libraries_mapped": mapped_libraries()}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- plain vs learned
def solver_run(scene, steps: int, warmup: int, params=None, norm=None, autotune: bool = True) -> dict:
    """Throughput of `steps` graph-replayed steps after `warmup` (the launch
    shapes autotuned half way through the warm-up), then the same run replayed
    (the fast path is deterministic) with the per-step mean clamped density
    error and iteration count read after every step."""
    import torch
    from pbf_b200 import Particles
    p = scene.params()
    out = {}
    with Particles(p, scene.n) as g:
        if scene.solver == 1:
            g.mlp_set(params, norm)
        stream = torch.cuda.ExternalStream(g.stream_handle())
        x0 = scene.positions()
        g.upload(x0)
        tuning = None
        for i in range(warmup):
            if autotune and i == warmup // 2:
                # 6 timed steps per candidate: the learned step's cost varies with the
                # iterations each step needs, and 2 steps picked shapes 2-4% slower
                tuning, _ = g.autotune(6)
            g.step(1)
        g.sync()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            g.step(1)
        e1.record(stream)
        e1.synchronize()
        t = e0.elapsed_time(e1) / 1e3
        g.upload(x0)
        for _ in range(warmup):
            g.step(1)
        err, its = [], []
        for _ in range(steps):
            g.step(1)
            st = g.stats()
            err.append(st["mean_density_error"])
            its.append(st["solver_iterations"])
        # per-kernel device time over the same window (eager launches with events)
        g.upload(x0)
        for _ in range(warmup):
            g.step(1)
        g.set_timing(True)
        g.reset_timing()
        g.step(steps)
        kt = g.kernel_times()
        g.set_timing(False)
    import numpy as np
    return {"value": scene.n * steps / t, "ms_per_step": 1e3 * t / steps,
            "mean_density_error": float(np.mean(err)), "max_step_density_error": float(np.max(err)),
            "mean_iterations": float(np.mean(its)), "tuning": tuning,
            "kernel_ms_per_step": {k: round(v["total_ms"] / steps, 4) for k, v in
                                   sorted(kt.items(), key=lambda kv: -kv[1]["total_ms"])}}


def learned_comparison(scene_name: str, steps: int, warmup: int, target: float = 0.01,
                       autotune: bool = True) -> dict:
    """Plain PBF against the learned warm start at equal mean density error
    <= target (1% of rest density): plain runs with the smallest K in 3..12
    that keeps its mean error over the window at or below the target; the
    learned solver iterates per step until its error is at or below it
    (`learned`: the residual checked over every 8th run of 32 slots;
    `learned_full_checks`: over every particle), and, by plain's protocol,
    with the smallest fixed count that keeps its mean error at or below it
    (`learned_fixed`).  Every error reported is the true mean over all
    particles, after each step."""
    from pbf_b200.learn import DEFAULT_MODEL, load_model, warm_start_scene
    if not DEFAULT_MODEL.exists():
        return {"unavailable": f"no trained network at {DEFAULT_MODEL.relative_to(ROOT)}"}
    params, norm, meta = load_model(DEFAULT_MODEL)
    base = warm_start_scene(scene_name, seed=4242)  # a jitter seed the network was not trained on
    tried = {}
    plain, K = None, None
    for k in range(3, 13):
        plain = solver_run(base.with_(solve_steps=k), steps, warmup, autotune=autotune)
        tried[k] = plain["mean_density_error"]
        K = k
        if plain["mean_density_error"] <= target:
            break
    # residual checks over every 8th run of 32 slots (the plain density pass
    # only when another iteration follows), and over every particle
    learned = solver_run(base.with_(solver=1, residual_tol=target, max_iterations=K, residual_sample=8), steps,
                         warmup, params, norm, autotune=autotune)
    full = solver_run(base.with_(solver=1, residual_tol=target, max_iterations=K), steps, warmup, params, norm,
                      autotune=autotune)
    # the same protocol as plain's: the smallest fixed count (network + plain
    # iterations, no residual checks) that keeps the mean error at or below it
    fixed, tried_fixed = None, {}
    for m in range(1, K + 1):
        fixed = solver_run(base.with_(solver=1, residual_tol=0.0, max_iterations=m), steps, warmup, params, norm,
                           autotune=autotune)
        tried_fixed[m] = fixed["mean_density_error"]
        if fixed["mean_density_error"] <= target:
            fixed = dict(fixed, iterations=m)
            break
    else:
        fixed = None
    return {"workload": f"{base.name}, relaxation epsilon {base.lambda_epsilon}, steps {warmup}..{warmup + steps}",
            "target_mean_density_error": target, "plain_errors_by_K": tried,
            "plain": dict(plain, iterations=K),
            "learned": dict(learned, residual_tol=target, max_iterations=K, residual_sample=8),
            "speedup": learned["value"] / plain["value"],
            "learned_full_checks": dict(full, residual_tol=target, max_iterations=K, residual_sample=1),
            "speedup_full_checks": full["value"] / plain["value"],
            "learned_fixed_errors_by_count": tried_fixed, "learned_fixed": fixed,
            "speedup_fixed": None if fixed is None else fixed["value"] / plain["value"],
            "network": {k: meta.get(k) for k in ("trajectories", "steps", "batch", "lr", "final_loss")}}


# ---------------------------------------------------------------- batched scenes
def batched_run(steps: int = 200, autotune: bool = True) -> dict:
    """The 64-scene batch (make_batch: counts log-uniform in [4096, 262144])
    advanced `steps` steps from its initial state by ONE graph launch, in two
    forms, against the same scenes and steps as 64 single-scene contexts each
    replaying its own one-step graph on its own stream (the streams run
    concurrently):
      value        the scene group: one graph launch whose members are the
                   64 contexts' `steps`-step chains (pbf_group_step), each
                   scene advancing at its own pace;
      one_context  one context holding all scenes (pbf_create_batch), every
                   launch covering every scene (pbf_step(ctx, steps)), and
                   (persistent_step) the same with each step's gather
                   passes in one persistent launch (pbf_set_persistent).
    Each graph is captured by an untimed run of the same call first."""
    import numpy as np
    import torch
    from pbf_b200 import Particles, make_batch
    b = make_batch()
    x0 = b.positions()
    out = {"workload": f"{b.name}: {len(b.scenes)} scenes, {b.n} particles (counts {min(b.counts)}.."
                       f"{max(b.counts)}), K = {b.scenes[0].solve_steps}, eps {b.scenes[0].lambda_epsilon}"}
    with Particles.batch(b) as g:
        g.upload(x0)
        g.step(3)
        tuning = g.autotune(2)[0] if autotune else g.tuning()
        g.upload(x0)
        g.step(steps)          # captures the steps-step graph (untimed)
        g.upload(x0)
        g.sync()
        stream = torch.cuda.ExternalStream(g.stream_handle())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        g.step(steps)
        e1.record(stream)
        e1.synchronize()
        t = e0.elapsed_time(e1) / 1e3
        errs = [g.scene_stats(i)["mean_density_error"] for i in range(len(b.scenes))]
        flags = g.stats()["error_flags"]
        launches = g.launches_per_step()
        # the same context with the persistent step: the list fill and every
        # gather pass of a step in one launch, each scene at its own pace
        # through the passes (pbf_set_persistent; its fixed launch shapes)
        g.set_persistent(True)
        g.upload(x0)
        g.step(steps)          # captures the steps-step graph (untimed)
        g.upload(x0)
        g.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        g.step(steps)
        e1.record(stream)
        e1.synchronize()
        tp = e0.elapsed_time(e1) / 1e3
        persistent = {"value": b.n * steps / tp, "ms_per_step": 1e3 * tp / steps, "graph_launches": 1,
                      "kernel_launches_per_step": g.launches_per_step(), "error_flags": g.stats()["error_flags"]}
    out.update({"value": b.n * steps / t, "unit": UNIT, "steps": steps, "ms_per_step": 1e3 * t / steps,
                "graph_launches": 1, "kernel_launches_per_step": launches, "tuning": tuning,
                "scene_mean_density_error": {"min": float(np.min(errs)), "max": float(np.max(errs))},
                "error_flags": flags})
    # the same scenes as independent contexts
    ctxs = []
    try:
        for sc in b.scenes:
            c = Particles(sc.params(), sc.n)
            c.set_tuning(tuning)
            c.upload(sc.positions())
            c.step(1)  # captures the one-step graph
            c.upload(sc.positions())
            ctxs.append(c)
        torch.cuda.synchronize()
        for c in ctxs:
            c.sync()
        s0 = torch.cuda.ExternalStream(ctxs[0].stream_handle())
        e0 = torch.cuda.Event(enable_timing=True)
        e0.record(s0)
        for c in ctxs:  # every context's stream starts after e0
            torch.cuda.ExternalStream(c.stream_handle()).wait_event(e0)
        for _ in range(steps):
            for c in ctxs:
                c.step(1)
        ends = []
        for c in ctxs:
            e = torch.cuda.Event(enable_timing=True)
            e.record(torch.cuda.ExternalStream(c.stream_handle()))
            ends.append(e)
        for e in ends:
            e.synchronize()
        ts = max(e0.elapsed_time(e) for e in ends) / 1e3
        out_ind = {"value": b.n * steps / ts, "ms_per_step": 1e3 * ts / steps,
                   "steps": steps, "graph_launches_per_step": len(b.scenes)}
        # the same contexts as one scene group: one graph launch of every scene's
        # `steps`-step chain, each scene at its own pace (pbf_group_step)
        from pbf_b200 import SceneGroup
        for c, sc in zip(ctxs, b.scenes):
            c.upload(sc.positions())
        with SceneGroup(ctxs) as grp:
            grp.step(steps)           # captures and instantiates the group's graph (untimed)
            grp.sync()
            for c, sc in zip(ctxs, b.scenes):
                c.upload(sc.positions())
            torch.cuda.synchronize()
            gs = torch.cuda.ExternalStream(grp.stream_handle())
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(gs)
            grp.step(steps)
            e1.record(gs)
            e1.synchronize()
            tg = e0.elapsed_time(e1) / 1e3
        group_flags = max(c.stats()["error_flags"] for c in ctxs)
    finally:
        for c in ctxs:
            c.close()
    one_context = {k: out[k] for k in ("value", "ms_per_step", "graph_launches", "kernel_launches_per_step",
                                       "scene_mean_density_error", "error_flags")}
    one_context["speedup_vs_independent"] = one_context["value"] / out_ind["value"]
    persistent["speedup_vs_independent"] = persistent["value"] / out_ind["value"]
    one_context["persistent_step"] = persistent
    res = {"workload": out["workload"], "mode": "scene group: one graph launch of every scene's step chain, "
                                                "each scene at its own pace (pbf_group_step)",
           "value": b.n * steps / tg, "unit": UNIT, "steps": steps, "ms_per_step": 1e3 * tg / steps,
           "graph_launches": 1, "tuning": tuning, "error_flags": group_flags,
           "independent_contexts": out_ind, "speedup_vs_independent": (b.n * steps / tg) / out_ind["value"],
           "one_context": one_context}
    return res


# ---------------------------------------------------------------- more workloads
def timed_steps(g, stream, steps: int) -> float:
    """Seconds of `steps` graph-replayed steps on the library's stream (CUDA events)."""
    import torch
    g.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        g.step(1)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / 1e3


def plain_run(scene, steps: int, warmup: int, tuning=None) -> dict:
    """particle-steps/s of `steps` graph-replayed steps of `scene` after
    `warmup` steps, with the given launch shapes (the 1M dam's autotuned ones)."""
    import torch
    from pbf_b200 import Particles
    with Particles(scene.params(), scene.n) as g:
        if tuning:
            g.set_tuning(tuning)
        stream = torch.cuda.ExternalStream(g.stream_handle())
        g.upload(scene.positions())
        for _ in range(warmup):
            g.step(1)
        t = timed_steps(g, stream, steps)
        st = g.stats()
    return {"workload": f"{scene.name}: {scene.n} particles, K = {scene.solve_steps}, cap {scene.neighbor_cap}, "
                        f"eps {scene.lambda_epsilon}, s_corr k = {scene.scorr[0]}",
            "value": scene.n * steps / t, "unit": UNIT, "ms_per_step": 1e3 * t / steps, "steps": steps,
            "warmup": warmup, "mean_density_error": st["mean_density_error"], "mean_neighbors": st["mean_neighbors"],
            "error_flags": st["error_flags"]}


def trajectory_run(scene, steps: int = 200, window: int = 50, tuning=None) -> dict:
    """The whole `steps`-step dam break from its initial state, timed in
    windows of `window` graph-replayed steps (the step cost grows as the
    dam collapses and the bins crowd)."""
    import torch
    from pbf_b200 import Particles
    with Particles(scene.params(), scene.n) as g:
        if tuning:
            g.set_tuning(tuning)
        stream = torch.cuda.ExternalStream(g.stream_handle())
        g.upload(scene.positions())
        g.step(1)                      # captures the one-step graph
        g.upload(scene.positions())    # back to the initial state
        ts, errs = [], []
        for _ in range(steps // window):
            ts.append(timed_steps(g, stream, window))
            errs.append(g.stats()["mean_density_error"])
    total = sum(ts)
    return {"workload": f"{scene.name}: steps 0..{steps} from the initial state, K = {scene.solve_steps}",
            "value": scene.n * steps / total, "unit": UNIT, "ms_per_step": 1e3 * total / steps,
            "windows": [{"steps": f"{i * window}..{(i + 1) * window}", "ms_per_step": 1e3 * t / window,
                         "mean_density_error_at_end": e} for i, (t, e) in enumerate(zip(ts, errs))]}


# ---------------------------------------------------------------- main
def main():
    args = parse_args()
    if args.impl == "reference":
        return reference_arm(args)
    if args.profile_training:
        import ctypes as C
        import torch
        from pbf_b200 import Particles
        from pbf_b200.learn import normalization, warm_start_scene
        sc = warm_start_scene(args.scene)
        with Particles(sc.params(), sc.n) as g:
            g.mlp_init(7)
            g.upload(sc.positions())
            g.step(3)
            g.set_recording(True)
            g.step(1)
            g.set_recording(False)
            f, lab = g.training_data()
            params, _ = g.mlp_get()
            g.mlp_set(params, normalization(f, lab))
            loss = C.c_float()
            for _ in range(2):  # the second call is timed
                g.sync()
                t0 = time.perf_counter()
                rc = g._lib.pbf_mlp_train(g.ctx, args.profile_training, 65536, C.c_float(1e-3), 5, C.byref(loss))
                dt = time.perf_counter() - t0
                assert rc == 0, g._lib.pbf_last_error(g.ctx)
        print(json.dumps({"ms_per_adam_update": 1e3 * dt / args.profile_training, "batch": 65536,
                          "loss": loss.value}), flush=True)
        return 0
    if args.profile_learned:
        from pbf_b200.learn import DEFAULT_MODEL, load_model, warm_start_scene
        params, norm, _ = load_model(DEFAULT_MODEL)
        sc = warm_start_scene(args.scene, seed=4242).with_(solver=1, residual_tol=0.01,
                                                           max_iterations=args.learned_iterations,
                                                           residual_sample=args.residual_sample)
        r = solver_run(sc, args.profile_learned, args.warmup, params, norm, autotune=False)
        print(json.dumps({"learned_ms_per_step": r["ms_per_step"], "iterations": r["mean_iterations"],
                          "kernel_ms_per_step": r["kernel_ms_per_step"]}), flush=True)
        return 0
    rank, world, local = dist_env()
    from pbf_b200 import make_scene
    scene = make_scene(args.scene, exact_math=1 if args.exact else 0)
    K, W = args.steps, args.warmup

    import numpy as np
    import torch
    torch.cuda.set_device(local)
    ranks = RankGroup(world)

    from pbf_b200 import Particles
    p = scene.params()
    x0 = scene.positions()
    g = Particles(p, scene.n)
    g.upload(x0)
    stream = torch.cuda.ExternalStream(g.stream_handle())

    def barrier():
        ranks.barrier()
        torch.cuda.synchronize()
        g.sync()

    max_over_ranks = ranks.max

    # warm-up: 3 steps, the autotuner (times each launch shape on 3 steps from
    # this state, then restores it), then W steps (the last captures the graph)
    for _ in range(3):
        g.step(1)
    tuning, tune_table = (None, None) if args.no_autotune else g.autotune(3)
    for _ in range(max(W, 3)):
        g.step(1)
    barrier()

    # ---- device-resident timed region: K graph replays ----
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier()
        e0.record(stream)
        for _ in range(K):
            g.step(1)
        e1.record(stream)
        e1.synchronize()
        barrier()
    t_dev = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    st = g.stats()
    nbar = st["mean_neighbors"]

    # ---- per-kernel times: the same K steps again (from the initial state, the
    # same warm-up count), eager, with CUDA events around each kernel ----
    g.upload(x0)
    for _ in range(3 + max(W, 3)):
        g.step(1)
    g.set_timing(True)
    g.reset_timing()
    g.step(K)
    kt = g.kernel_times()
    g.set_timing(False)
    total_kernel_ms = sum(v["total_ms"] for v in kt.values())
    dom = max(kt.items(), key=lambda kv: kv[1]["total_ms"])
    dom_name, dom_t = dom[0], dom[1]
    dom_avg_s = dom_t["total_ms"] / dom_t["launches"] / 1e3
    nbins = int(g._lib.pbf_num_bins(g.ctx))
    dom_bytes = kernel_bytes(dom_name, scene.n, nbar, scene.solve_steps, nbins)
    peaks = measured_peaks()
    achieved = dom_bytes / dom_avg_s / 1e9
    step_bytes = sum(kernel_bytes(k, scene.n, nbar, scene.solve_steps, nbins) * v["launches"] for k, v in kt.items()) / K
    kernels = {k: {"launches": v["launches"], "ms_per_launch": v["total_ms"] / v["launches"],
                   "share": v["total_ms"] / total_kernel_ms,
                   "gbs": kernel_bytes(k, scene.n, nbar, scene.solve_steps, nbins) / (v["total_ms"] / v["launches"] / 1e3) / 1e9}
               for k, v in sorted(kt.items(), key=lambda kv: -kv[1]["total_ms"])}

    # ---- end to end through the C ABI with pinned host buffers ----
    xh = torch.empty((scene.n, 3), dtype=torch.float32, pin_memory=True).numpy()
    vh = torch.empty((scene.n, 3), dtype=torch.float32, pin_memory=True).numpy()
    xh[:] = x0
    vh[:] = 0.0
    import ctypes as C
    lib = g._lib
    px, pv = xh.ctypes.data_as(C.c_void_p), vh.ctypes.data_as(C.c_void_p)
    for _ in range(2):
        assert lib.pbf_upload(g.ctx, px, pv, scene.n) == 0
        assert lib.pbf_step(g.ctx, 1) == 0
        assert lib.pbf_download(g.ctx, px, pv, None, None) == 0
    barrier()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(K):
        lib.pbf_upload(g.ctx, px, pv, scene.n)
        lib.pbf_step(g.ctx, 1)
        lib.pbf_download(g.ctx, px, pv, None, None)
    f1.record(stream)
    f1.synchronize()
    barrier()
    t_e2e = max_over_ranks(f0.elapsed_time(f1) / 1e3)

    ok = bool(np.isfinite(xh).all())
    launches = g.launches_per_step() * K

    learned = None
    if rank == 0 and world == 1 and not args.no_learned:
        try:
            learned = learned_comparison(args.scene, max(K, 20), 100, autotune=not args.no_autotune)
        except Exception as e:  # reported, never fatal for the GPU line
            learned = {"error": str(e)}

    batched = None
    if rank == 0 and world == 1 and not args.no_batched:
        try:
            batched = batched_run(autotune=not args.no_autotune)
        except Exception as e:  # reported, never fatal for the GPU line
            batched = {"error": str(e)}

    extra = None
    if rank == 0 and world == 1 and not args.no_extra:
        extra = {}
        shapes = g.tuning()
        for key, fn in (("dam_16m", lambda: plain_run(make_scene("dam_16m"), 10, 3, shapes)),
                        ("trajectory_200", lambda: trajectory_run(make_scene(args.scene), 200, 50, shapes)),
                        ("scorr_on", lambda: plain_run(make_scene(args.scene, scorr=(0.1, 4.0, 0.2)), K, max(W, 3),
                                                       shapes))):
            try:
                extra[key] = fn()
            except Exception as e:  # reported, never fatal for the GPU line
                extra[key] = {"error": str(e)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = run_reference_cpu(scene.name, 100, 1, args.cpu_seconds)
            one = run_reference_cpu(scene.name, 100, 0, args.cpu_seconds / 3, threads=1)
            cpu["one_thread"] = {k: one[k] for k in ("value", "cores", "sample")}
        except Exception as e:  # reported, never fatal for the GPU line
            cpu = {"error": str(e)}
    ranks.barrier()

    if rank == 0:
        value = scene.n * K * world / t_dev
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": max(W, 3),
            "ms_per_step": 1e3 * t_dev / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded jittered dam-break lattice, zero initial velocity)",
            "config": workload_config(scene.name, scene.n, scene.lattice, scene.box_max, scene.solve_steps,
                                      scene.lambda_epsilon, scene.neighbor_cap, world),
            "solver": {"exact_math": scene.exact_math, "tuning": g.tuning(), "autotuned": not args.no_autotune,
                       "neighbor_list_mb": scene.n * (4 * nbar + 4) / 1e6},
            "e2e": {"value": scene.n * K * world / t_e2e, "unit": UNIT, "h2d_bytes_per_step": scene.n * 24,
                    "d2h_bytes_per_step": scene.n * 24},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": achieved, "peak": peaks["hbm_gbs"],
                         "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
                         "traffic": ncu_traffic(dom_name, scene.name),
                         "algorithmic_bytes_per_launch": dom_bytes, "peak_source": peaks["source"],
                         "step_gbs": step_bytes / (t_dev / K) / 1e9},
            "kernels": kernels,
            "autotune_ms_per_step": None if tune_table is None else
            {f"{l}x{b}{'staged' if st else ''}": v for (l, b, st), v in tune_table.items()},
            "physics": {"mean_neighbors": nbar, "cap_hits": st["cap_hits"],
                        "mean_density_error": st["mean_density_error"], "error_flags": st["error_flags"],
                        "finite": ok},
            "clocks": clk.summary(),
            "learned_vs_plain": learned,
            "batched": batched,
            "extra": extra,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    g.close()
    ranks.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
