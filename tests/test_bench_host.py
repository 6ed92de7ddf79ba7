"""bench.py's host logic without a GPU: the compulsory-bytes model behind the
roofline and per-kernel GB/s covers every kernel the library times."""
from __future__ import annotations

import re
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_every_timed_kernel_has_a_byte_model():
    sys.path.insert(0, str(ROOT))
    import bench
    src = (ROOT / "sph-cpp_b200" / "csrc" / "pbf_cuda.cu").read_text()
    names = set(re.findall(r'Launch L\d*\(ctx, "([a-z_]+)"\)', src))
    assert {"fill_neighbors", "density_lambda", "dp_update", "warm_mlp"} <= names
    n, nbar, K, nbins = 1 << 20, 55.0, 3, 1 << 20
    missing = sorted(k for k in names if not bench.kernel_bytes(k, n, nbar, K, nbins) > 0.0)
    assert not missing, missing


def test_roofline_traffic_and_peak_come_from_committed_files():
    """The dominant kernel's DRAM traffic is read from its committed ncu
    summary and the denominator from the measured peaks (or the stated
    fallback), so the bench line's roofline is never left without them."""
    sys.path.insert(0, str(ROOT))
    import bench
    t = bench.ncu_traffic("fill_neighbors", "dam_1m")
    assert t is not None and 1e8 < t < 1e9
    for kernel in ("density_lambda", "dp_update", "viscosity_final"):
        assert bench.ncu_traffic(kernel, "dam_1m") > 0
    peaks = bench.measured_peaks()
    assert peaks["hbm_gbs"] > 1000 and peaks["source"] in ("measured", "fallback")


def test_training_normalisation():
    """Feature mean and 1/std per column (a constant column gets a finite
    scale), and the label scale is the labels' rms."""
    import numpy as np
    sys.path.insert(0, str(ROOT / "sph-cpp_b200"))
    from pbf_b200.learn import normalization
    rng = np.random.default_rng(3)
    f = rng.normal(2.0, 3.0, (5000, 12)).astype(np.float32)
    f[:, 5] = 7.0
    lab = rng.normal(0.0, 0.5, 5000).astype(np.float32)
    n = normalization(f, lab)
    assert n.shape == (25,)
    np.testing.assert_allclose(n[:12], f.mean(axis=0), rtol=1e-4, atol=1e-4)
    np.testing.assert_allclose(n[12:24][[0, 1, 2]], 1.0 / f[:, [0, 1, 2]].std(axis=0), rtol=1e-3)
    assert np.isfinite(n[12 + 5]) and n[12 + 5] > 0
    assert abs(n[24] - np.sqrt(np.mean(lab.astype(np.float64) ** 2))) < 1e-6
