"""Learned warm start on the GPU: the tensor-core network against the float64
oracle (forward and gradients), training on the plain solver's own lambdas,
what the trained network gains over the plain first iteration, and the
residual-controlled iteration loop."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import mlp_oracle as MO
from pbf_b200 import Particles, _abi
from pbf_b200.learn import held_out_loss, normalization, run_solver, train, warm_start_scene

pytestmark = pytest.mark.gpu

# BF16 operands (8-bit mantissa), FP32 accumulation, two hidden layers.
Y_TOL = 0.03        # forward: max |y_gpu - y_oracle| relative to max |y|
GRAD_COS = 0.995    # gradient direction
GRAD_REL = 0.05     # gradient norm-wise relative error


def _ctx_with_net(seed=5):
    sc = warm_start_scene("dam_2k")
    g = Particles(sc.params(), 8192)  # staging room for 8192 * 6 / 13 host samples
    g.mlp_init(seed)
    return g


def test_forward_matches_float64_oracle():
    g = _ctx_with_net()
    params, norm = g.mlp_get()
    rng = np.random.default_rng(0)
    x = rng.normal(0, 1, (1000, _abi.MLP_FEATURES)).astype(np.float32)
    y = g.mlp_predict(x)
    ref, _ = MO.forward(params.astype(np.float64), x.astype(np.float64))
    assert np.abs(y - ref).max() <= Y_TOL * max(np.abs(ref).max(), 0.1)


def test_gradients_match_float64_oracle():
    g = _ctx_with_net(9)
    params, _ = g.mlp_get()
    rng = np.random.default_rng(1)
    x = rng.normal(0, 1, (1024, _abi.MLP_FEATURES)).astype(np.float32)
    t = rng.normal(0, 1, 1024).astype(np.float32)
    grad, loss = g.mlp_gradients(x, t)
    ref_loss, ref = MO.loss_and_grad(params.astype(np.float64), x, t)
    assert loss == pytest.approx(ref_loss, rel=0.02)
    cos = float(grad @ ref / (np.linalg.norm(grad) * np.linalg.norm(ref)))
    assert cos >= GRAD_COS, cos
    assert np.linalg.norm(grad - ref) <= GRAD_REL * np.linalg.norm(ref)
    # every parameter block gets its gradient (layer 1 weights, biases, layer 3)
    for a, b in ((MO.OFF_W1, MO.OFF_B1), (MO.OFF_B1, MO.OFF_W2), (MO.OFF_W2, MO.OFF_B2), (MO.OFF_W3, MO.OFF_B3)):
        blk, rb = grad[a:b], ref[a:b]
        assert np.linalg.norm(blk - rb) <= 0.1 * np.linalg.norm(rb) + 1e-7


@pytest.fixture(scope="module")
def trained_8k():
    sc = warm_start_scene("dam_8k")
    params, norm, hist = train(sc, seeds=(11, 12, 13, 14), steps=120, adam_per_step=4, batch=8192, lr=1e-3)
    return sc, params, norm, hist


def test_recorded_training_data_are_the_plain_solver_lambdas():
    sc = warm_start_scene("dam_2k")
    p = sc.params()
    g = Particles(p, sc.n)
    g.set_recording(True)
    g.upload(sc.positions())
    g.step(5)
    f, lab = g.training_data()
    assert np.isfinite(f).all() and np.isfinite(lab).all()
    assert (lab <= 0).all() and (lab < 0).any()           # lambdas are never positive
    assert np.allclose(f[:, 0] * 64, np.round(f[:, 0] * 64))     # neighbour counts
    assert (f[:, 1] >= 0).all() and np.allclose(np.maximum(f[:, 2], 0), f[:, 1], atol=1e-6)
    # the plain first-iteration lambda feature, -C/(S+eps)
    assert np.allclose(f[:, 4], -f[:, 1] / (f[:, 3] + p.lambda_epsilon), rtol=1e-5, atol=1e-12)
    norm = normalization(f, lab)
    assert norm.shape == (_abi.MLP_NORM,) and np.isfinite(norm).all()


def test_training_reduces_held_out_loss(trained_8k):
    """Trained on the plain solver's lambdas, the network predicts them on a
    trajectory it has not seen far better than it did untrained."""
    sc, params, norm, hist = trained_8k
    assert np.isfinite(hist[:, 2]).all()
    g = _ctx_with_net(7)  # the same initial network as train(init_seed=7)
    init_params, _ = g.mlp_get()
    before = held_out_loss(sc, init_params, norm, seed=97)
    after = held_out_loss(sc, params, norm, seed=97)
    assert after < 0.5 * before, (before, after)


def test_trained_warm_start_beats_plain_at_equal_iterations(trained_8k):
    """What the network gains: with two Jacobi iterations per step, the first
    seeded by the network's lambda, the density error is lower than with two
    plain iterations (held-out seed; the residual check never stops early)."""
    sc, params, norm, _ = trained_8k
    held = sc.with_(seed=99)
    plain2 = run_solver(held.with_(solve_steps=2), 60, warmup=20)
    learned2 = run_solver(held.with_(solver=1, max_iterations=2, residual_tol=0.0), 60, params, norm, warmup=20)
    assert (learned2["iterations"] == 2).all()
    assert learned2["residual"].mean() < plain2["residual"].mean(), (learned2["residual"].mean(),
                                                                     plain2["residual"].mean())


def test_residual_controlled_iterations(trained_8k):
    sc, params, norm, _ = trained_8k
    held = sc.with_(seed=98)
    never = run_solver(held.with_(solver=1, max_iterations=5, residual_tol=1e9), 10, params, norm)
    assert (never["iterations"] == 1).all()
    always = run_solver(held.with_(solver=1, max_iterations=5, residual_tol=0.0), 10, params, norm)
    assert (always["iterations"] == 5).all()
    plain3 = run_solver(held.with_(solve_steps=3), 40, warmup=20)
    tol = float(plain3["residual"].mean())
    from pbf_b200 import Particles as P
    p = held.with_(solver=1, max_iterations=6, residual_tol=tol).params()
    with P(p, held.n) as g:
        g.mlp_set(params, norm)
        g.upload(held.positions())
        g.step(20)
        for _ in range(40):
            g.step(1)
            st = g.stats()
            assert st["error_flags"] == 0
            if st["solver_iterations"] < 6:
                assert st["solver_residual"] <= tol
                assert st["mean_density_error"] <= tol * 1.02 + 1e-6


def test_network_kernel_gives_up_a_wait_and_the_context_stays_usable():
    """Failure detection without a GPU fault: the network kernel launched with
    nothing arriving on its completion barrier gives up its bounded waits,
    raises the timeout flag in its own status word and frees its tensor
    memory; the context's error flags stay clear and the next network call
    still matches the float64 oracle."""
    g = _ctx_with_net()
    flags = g.selftest_mlp_wait_timeout()
    assert flags & _abi.PBF_FLAG_WAIT_TIMEOUT
    params, _ = g.mlp_get()
    x = np.random.default_rng(1).normal(0, 1, (600, _abi.MLP_FEATURES)).astype(np.float32)
    y = g.mlp_predict(x)
    ref, _ = MO.forward(params.astype(np.float64), x.astype(np.float64))
    assert np.abs(y - ref).max() <= Y_TOL * max(np.abs(ref).max(), 0.1)
    g.upload(warm_start_scene("dam_2k").positions())
    g.step(1)
    assert g.stats()["error_flags"] == 0
    g2 = Particles(warm_start_scene("dam_2k").params(), 4096)
    with pytest.raises(RuntimeError, match="no network"):
        g2.selftest_mlp_wait_timeout()


@pytest.mark.parametrize("sample", [1, 8])
@pytest.mark.parametrize("tol", [1e-4, 0.005])
def test_captured_iteration_loop_matches_eager_launches(tol, sample):
    """In a captured step the learned solver's plain iterations are a WHILE
    node of the graph that the residual check ends; eager launches (per-kernel
    timing on) run the same iterations as a loop of launches that skip
    themselves.  Both give the same positions, velocities and iteration
    counts, bit for bit, with one step or four steps per graph.  Once the dam
    compresses, tol 1e-4 is never reached: those steps run the loop body three
    times and leave it at the iteration cap (4); at tol 0.005 the check inside
    the loop ends it."""
    from pbf_b200.learn import DEFAULT_MODEL, load_model
    params, norm, _ = load_model(DEFAULT_MODEL)
    sc = warm_start_scene("dam_8k", solver=1, residual_tol=tol, max_iterations=4, residual_sample=sample)
    runs = {}
    for mode in ("eager", "graph1", "graph4"):
        g = Particles(sc.params(), sc.n)
        g.mlp_set(params, norm)
        g.upload(sc.positions())
        g.set_timing(mode == "eager")
        its = []
        for k in range(18):  # 72 steps, the iteration counts of every fourth
            if mode == "graph4":
                g.step(4)
            else:
                for _ in range(4):
                    g.step(1)
            its.append(g.stats()["solver_iterations"])
        runs[mode] = (g.positions(), g.velocities(), its)
        assert g.stats()["error_flags"] == 0
    x, v, its = runs["eager"]
    if tol < 1e-3:  # the first steps (a falling lattice, no compression) converge at once
        assert its.count(4) >= 12, its
    for mode in ("graph1", "graph4"):
        assert np.array_equal(runs[mode][0], x), mode
        assert np.array_equal(runs[mode][1], v), mode
        assert runs[mode][2] == its, (mode, runs[mode][2], its)


def test_fixed_count_runs_the_checked_iterations_without_the_checks():
    """residual_tol <= 0 fixes the count at max_iterations with no residual
    checks.  From the same state, one step moves every particle exactly as the
    checked loop does when its tolerance is never met (each check's
    density/lambda pass is the plain one); the velocities differ only through
    the density XSPH divides by, which the fixed count takes from its last
    density pass, as the plain solver does (particles.h:436-447 after the last
    iteration), and the checked loop from its final check."""
    from pbf_b200.learn import DEFAULT_MODEL, load_model
    params, norm, _ = load_model(DEFAULT_MODEL)
    base = warm_start_scene("dam_8k", solver=1, residual_tol=1e-30, max_iterations=3)
    with Particles(base.params(), base.n) as w:
        w.mlp_set(params, norm)
        w.upload(base.positions())
        w.step(30)
        d = w.download()
    out = {}
    for tol in (1e-30, 0.0):
        sc = base.with_(residual_tol=tol)
        with Particles(sc.params(), sc.n) as g:
            g.mlp_set(params, norm)
            g.upload(d["x"], d["v"])
            g.set_timing(True)
            g.step(1)
            kt = g.kernel_times()
            g.set_timing(False)
            st = g.stats()
            assert st["error_flags"] == 0 and st["solver_iterations"] == 3
            assert sum(v["launches"] for v in kt.values()) == g.launches_per_step()
            out[tol] = (g.positions(), g.velocities(), kt)
    assert np.array_equal(out[0.0][0], out[1e-30][0])
    v0, v1 = out[0.0][1], out[1e-30][1]
    assert np.abs(v0 - v1).max() <= 1e-3 * np.abs(v1).max()
    assert "residual_check" not in out[0.0][2] and out[0.0][2]["density_lambda"]["launches"] == 2


def test_sampled_checks_keep_the_error_at_the_tolerance(trained_8k):
    """residual_sample = 8: each check estimates the mean clamped density
    error from every 8th run of 32 slots, and the plain density/lambda pass runs only
    when another iteration follows.  A step that stops before the cap has an
    estimate at or below the tolerance, and the true mean error over the window
    stays within a few per cent of it."""
    sc, params, norm, _ = trained_8k
    held = sc.with_(seed=98)
    plain3 = run_solver(held.with_(solve_steps=3), 40, warmup=20)
    tol = float(plain3["residual"].mean())
    p = held.with_(solver=1, max_iterations=6, residual_tol=tol, residual_sample=8).params()
    errs = []
    with Particles(p, held.n) as g:
        g.mlp_set(params, norm)
        g.upload(held.positions())
        g.step(20)
        for _ in range(40):
            g.step(1)
            st = g.stats()
            assert st["error_flags"] == 0
            if st["solver_iterations"] < 6:
                assert st["solver_residual"] <= tol
            errs.append(st["mean_density_error"])
    assert np.mean(errs) <= tol * 1.05 + 1e-6, (np.mean(errs), tol)


def test_timing_counts_every_learned_kernel():
    """Eager learned steps (per-kernel timing on) launch exactly what
    launches_per_step reports: the features and the network, then
    max_iterations residual checks and as many position updates, each
    skipping itself once the step has converged."""
    sc = warm_start_scene("dam_2k", solver=1, max_iterations=5)
    g = Particles(sc.params(), sc.n)
    g.mlp_init(3)
    g.upload(sc.positions())
    g.set_timing(True)
    g.step(2)
    t = g.kernel_times()
    g.set_timing(False)
    assert sum(v["launches"] for v in t.values()) == 2 * g.launches_per_step()
    assert t["warm_mlp"]["launches"] == 2 and t["warm_features"]["launches"] == 2
    assert t["residual_check"]["launches"] == 2 * 5 and t["dp_update"]["launches"] == 2 * 5


def test_hundred_learned_steps_in_one_graph():
    """A hundred learned steps captured in one graph (a hundred conditional
    loop nodes) give the same state as a hundred one-step graphs."""
    from pbf_b200.learn import DEFAULT_MODEL, load_model
    params, norm, _ = load_model(DEFAULT_MODEL)
    sc = warm_start_scene("dam_2k", solver=1, residual_tol=0.005, max_iterations=4)
    out = []
    for per_graph in (100, 1):
        g = Particles(sc.params(), sc.n)
        g.mlp_set(params, norm)
        g.upload(sc.positions())
        for _ in range(100 // per_graph):
            g.step(per_graph)
        out.append((g.positions(), g.velocities(), g.stats()))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    assert out[0][2]["solver_iterations"] == out[1][2]["solver_iterations"]
    assert out[0][2]["error_flags"] == 0
