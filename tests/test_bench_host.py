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
