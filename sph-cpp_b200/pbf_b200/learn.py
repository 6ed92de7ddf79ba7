"""Learned warm start: training on the GPU and the plain-vs-learned comparison.

The network (include/pbf.h, pbf_mlp_*) is trained by the library's own
tensor-core forward/backward kernels and Adam, on data the plain solver
produces while it runs: with recording on, every fused step keeps each
particle's features at its first Jacobi iteration and, as label, the sum of
the lambdas the plain solver applied over its K iterations.  One Adam update
on a batch drawn from that step follows each step.

    python -m pbf_b200.learn --out model.npz [--scene dam_1m] [--trajectories 10] [--steps 200] [--runs 8]

Training reduces its weight gradients with atomics, so two runs of the same
recipe differ; on the 1M dam they have needed from 2.2 to 2.8 solver
iterations per step.  --runs R trains R weight initialisations and keeps the
network whose learned solver needs the fewest iterations on a validation
seed that neither training nor the plain-vs-learned comparison uses.

The warm start targets the regime where the plain solver reaches a mean
clamped density error near 1% of rest density: relaxation epsilon 1 (at the
reference's epsilon 600 the plain solver's error stays above 40%).
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

from . import _abi
from .scenes import Scene, make_scene

TRAIN_EPSILON = 1.0
# jitter seeds of the training trajectories (evaluation uses other seeds)
TRAIN_SEEDS = tuple(1000 + 17 * i for i in range(10))
# jitter seed of the validation run stored with a trained model: neither a
# training seed nor the seed of the plain-vs-learned comparison (4242)
VALIDATION_SEED = 5151
# initialisation seeds of the weights, one per training run (--runs)
INIT_SEEDS = (7, 11, 13, 17, 19, 23, 29, 31)
MODEL_DIR = Path(__file__).resolve().parent / "models"
DEFAULT_MODEL = MODEL_DIR / "warm_start_dam_eps1.npz"


def warm_start_scene(name: str = "dam_1m", **kw) -> Scene:
    return make_scene(name, lambda_epsilon=TRAIN_EPSILON, **kw)


def normalization(features: np.ndarray, labels: np.ndarray) -> np.ndarray:
    """mean[12], inv_std[12], label_scale (rms of the labels) of recorded samples."""
    f = features.astype(np.float64)
    mean = f.mean(axis=0)
    std = f.std(axis=0)
    inv = 1.0 / np.maximum(std, 1e-6)
    scale = float(np.sqrt(np.mean(labels.astype(np.float64) ** 2)))
    if not scale > 0.0:
        scale = 1.0
    return np.concatenate([mean, inv, [scale]]).astype(np.float32)


def record_samples(ctx, scene: Scene, seed: int, steps: int, every: int, per_step: int, rng) -> tuple:
    """Features and labels of `per_step` particles of every `every`-th of
    `steps` recorded plain steps of one trajectory."""
    ctx.upload(scene.with_(seed=seed).positions())
    fs, ls = [], []
    for st in range(steps):
        ctx.step(1)
        if st % every == every - 1:
            f, lab = ctx.training_data()
            idx = rng.choice(f.shape[0], min(per_step, f.shape[0]), replace=False)
            fs.append(f[idx])
            ls.append(lab[idx])
    return np.concatenate(fs), np.concatenate(ls)


def train(scene: Scene, seeds=TRAIN_SEEDS, steps: int = 200, adam_per_step: int = 1, batch: int = 65536,
          lr: float = 1e-3, init_seed: int = 7, log=None):
    """Train on len(seeds) trajectories of `steps` plain steps each; the
    normalisation comes from a first pass over the first trajectory.  Returns
    (params, norm, history); history rows are (trajectory, step, loss)."""
    from . import Particles
    p = scene.with_(solver=0, exact_math=0).params()
    history = []
    rng = np.random.default_rng(init_seed)
    with Particles(p, scene.n) as ctx:
        ctx.mlp_init(init_seed)
        ctx.set_recording(True)
        f, lab = record_samples(ctx, scene, seeds[0], steps, max(1, steps // 20), 20000, rng)
        params, _ = ctx.mlp_get()
        ctx.mlp_set(params, normalization(f, lab))
        for ti, seed in enumerate(seeds):
            ctx.upload(scene.with_(seed=seed).positions())
            for st in range(steps):
                ctx.step(1)
                loss = ctx.mlp_train(adam_per_step, batch, lr, seed=(seed << 20) + st)
                history.append((ti, st, loss))
                if log and st % 50 == 0:
                    log(f"trajectory {ti} step {st} loss {loss:.5f}")
        params, norm = ctx.mlp_get()
    return params, norm, np.array(history, np.float64)


def held_out_loss(scene: Scene, params: np.ndarray, norm: np.ndarray, seed: int, steps: int = 100,
                  every: int = 10, per_step: int = 500) -> float:
    """Mean squared error of the network on samples of a trajectory it was not
    trained on (network units)."""
    from . import Particles
    p = scene.with_(solver=0, exact_math=0).params()
    cap = max(scene.n, per_step * (steps // every) * 13 // 6 + 16)
    with Particles(p, cap) as ctx:
        ctx.set_recording(True)
        f, lab = record_samples(ctx, scene, seed, steps, every, per_step, np.random.default_rng(seed))
        ctx.mlp_set(params, norm)
        k = _abi.MLP_FEATURES
        x = (f - norm[:k]) * norm[k:2 * k]
        _, loss = ctx.mlp_gradients(x.astype(np.float32), (lab / norm[2 * k]).astype(np.float32))
    return loss


def save_model(path: Path, params: np.ndarray, norm: np.ndarray, meta: dict) -> None:
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(path, params=params.astype(np.float32), norm=norm.astype(np.float32),
                        meta=np.array(json.dumps(meta)))


def load_model(path: Path = DEFAULT_MODEL) -> tuple[np.ndarray, np.ndarray, dict]:
    d = np.load(Path(path))
    return d["params"], d["norm"], json.loads(str(d["meta"]))


def run_solver(scene: Scene, steps: int, params=None, norm=None, warmup: int = 0) -> dict:
    """Run `steps` fused steps (after `warmup`) and report the per-step
    residual (mean clamped density error after the step) and iterations."""
    from . import Particles
    p = scene.params()
    res, its = [], []
    with Particles(p, scene.n) as ctx:
        if scene.solver == 1:
            ctx.mlp_set(params, norm)
        ctx.upload(scene.positions())
        for _ in range(warmup):
            ctx.step(1)
        for _ in range(steps):
            ctx.step(1)
            st = ctx.stats()
            res.append(st["mean_density_error"])
            its.append(st["solver_iterations"])
    return {"residual": np.array(res), "iterations": np.array(its)}


def validate(scene_name: str, params: np.ndarray, norm: np.ndarray, seed: int = VALIDATION_SEED,
             steps: int = 20, warmup: int = 100) -> dict:
    """The learned solver with this network on a held-out seed, as the
    comparison runs it (residual_tol 1%, at most 10 iterations): mean
    iterations per step and mean clamped density error over `steps` steps
    after `warmup` steps.  The training loss alone does not predict the
    iteration count (networks of lower loss have needed more iterations)."""
    sc = warm_start_scene(scene_name, seed=seed, solver=1, residual_tol=0.01, max_iterations=10)
    r = run_solver(sc, steps, params, norm, warmup=warmup)
    return {"seed": seed, "steps": f"{warmup}..{warmup + steps}", "mean_iterations": float(r["iterations"].mean()),
            "mean_density_error": float(r["residual"].mean())}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", type=Path, default=DEFAULT_MODEL)
    ap.add_argument("--scene", default="dam_1m")
    ap.add_argument("--trajectories", type=int, default=len(TRAIN_SEEDS))
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--lr", type=float, default=1e-3)
    # four Adam updates per recorded step: fewer solver iterations on the
    # validation seed than one (2.0-2.2 against 2.45-2.6, two initialisations each)
    ap.add_argument("--adam-per-step", type=int, default=4)
    ap.add_argument("--no-validate", action="store_true", help="skip the held-out learned-solver run")
    ap.add_argument("--runs", type=int, default=1,
                    help="train this many initialisations and keep the one the validation run favours")
    args = ap.parse_args(argv)
    if args.runs > 1 and args.no_validate:
        ap.error("--runs > 1 selects by the validation run; drop --no-validate")
    scene = warm_start_scene(args.scene)
    best = None
    runs = []
    for r in range(args.runs):
        init = INIT_SEEDS[r % len(INIT_SEEDS)]
        t0 = time.time()
        params, norm, hist = train(scene, TRAIN_SEEDS[: args.trajectories], args.steps, args.adam_per_step,
                                   args.batch, args.lr, init_seed=init, log=lambda m: print(m, flush=True))
        seconds = time.time() - t0
        val = None if args.no_validate else validate(args.scene, params, norm)
        runs.append({"init_seed": init, "final_loss": float(hist[-1, 2]) if len(hist) else None,
                     "seconds": seconds, "validation": val})
        print(json.dumps(runs[-1]), flush=True)
        key = (val["mean_iterations"], val["mean_density_error"]) if val else (0.0, 0.0)
        if best is None or key < best[0]:
            best = (key, params, norm, runs[-1])
    _, params, norm, chosen = best
    meta = {"scene": scene.name, "lambda_epsilon": scene.lambda_epsilon, "solve_steps": scene.solve_steps,
            "trajectories": args.trajectories, "steps": args.steps, "batch": args.batch, "lr": args.lr,
            "adam_per_step": args.adam_per_step, "seeds": list(TRAIN_SEEDS[: args.trajectories]),
            "init_seed": chosen["init_seed"], "final_loss": chosen["final_loss"], "seconds": chosen["seconds"]}
    if chosen["validation"]:
        meta["validation"] = chosen["validation"]
    if args.runs > 1:
        meta["selection"] = {"criterion": "fewest mean iterations on the validation seed, then lower error",
                             "runs": runs}
    save_model(args.out, params, norm, meta)
    print(json.dumps(meta), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
