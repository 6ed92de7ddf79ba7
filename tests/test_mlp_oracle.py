"""The float64 network oracle (oracle/mlp_oracle.py) checked against central
finite differences: its analytic gradient is what the GPU's tensor-core
backward pass is compared with."""
import numpy as np

from oracle import mlp_oracle as M


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = rng.normal(0, 0.3, M.N_PARAMS)
    x = rng.normal(0, 1, (17, M.N_IN))
    t = rng.normal(0, 1, 17)
    loss, g = M.loss_and_grad(p, x, t)
    idx = rng.choice(M.N_PARAMS, 60, replace=False)
    idx = np.concatenate([idx, [M.OFF_B3, M.OFF_W1, M.OFF_B1, M.OFF_W2 + 5, M.OFF_W3]])
    for i in idx:
        e = np.zeros(M.N_PARAMS)
        e[i] = 1e-6
        fd = (M.loss_and_grad(p + e, x, t)[0] - M.loss_and_grad(p - e, x, t)[0]) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(g[i]), (i, fd, g[i])


def test_oracle_gelu_is_the_erf_form():
    xs = np.array([-3.0, -1.0, 0.0, 0.5, 2.0])
    from math import erf, sqrt
    ref = np.array([0.5 * x * (1 + erf(x / sqrt(2))) for x in xs])
    assert np.allclose(M.gelu(xs), ref, rtol=0, atol=1e-15)


def test_training_cli_selection_needs_the_validation_run():
    """--runs R keeps the network the held-out validation run favours, so it
    cannot be combined with --no-validate (rejected before any device work);
    the validation seed is neither a training seed nor the comparison's."""
    import pytest
    from pbf_b200 import learn
    with pytest.raises(SystemExit):
        learn.main(["--runs", "2", "--no-validate"])
    assert learn.VALIDATION_SEED not in learn.TRAIN_SEEDS and learn.VALIDATION_SEED != 4242
    assert len(set(learn.INIT_SEEDS)) == len(learn.INIT_SEEDS)


def test_network_gelu_polynomial_against_erf():
    """The tensor-core network's GELU (pbf_mlp.cuh gelu2: erf from a fitted
    odd polynomial on the clamped argument) evaluated in float32 as the
    kernel does, against the exact GELU over the range bf16 activations
    take: erf within 3e-5, GELU within 7e-5 absolute."""
    import re
    from pathlib import Path

    import numpy as np
    from scipy.special import erf
    src = (Path(__file__).resolve().parents[1] / "sph-cpp_b200" / "csrc" / "pbf_mlp.cuh").read_text()
    body = src[src.index("float2 gelu2(float2 x)"):]
    coeffs = [float(v) for v in re.findall(r"(-?[0-9.]+e?-?[0-9]*)f", body[:body.index("};")])]
    assert len(coeffs) == 9
    f = np.float32
    c = [f(v) for v in coeffs]
    x = np.linspace(-40.0, 40.0, 800001).astype(f)
    u = np.clip((x * f(0.70710678118654752)).astype(f), f(-3.0), f(3.0))
    u2 = (u * u).astype(f)
    q = np.full_like(u, c[8])
    for k in range(7, -1, -1):
        q = (q * u2 + c[k]).astype(f)
    e = (q * u).astype(f)
    hx = (x * f(0.5)).astype(f)
    g = (hx * e + hx).astype(f)
    ux = x.astype(np.float64) / np.sqrt(2.0)
    inside = np.abs(ux) <= 3.0
    assert np.abs(e.astype(np.float64) - erf(u.astype(np.float64)))[inside].max() < 3e-5
    exact = 0.5 * x.astype(np.float64) * (1.0 + erf(ux))
    small = np.abs(x) <= 8.0  # activations of the trained network stay well inside
    assert np.abs(g - exact)[small].max() < 7e-5
