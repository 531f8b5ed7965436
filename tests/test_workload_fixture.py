"""The committed edge set of the benchmark workload equals the generator's output (CPU)."""
from __future__ import annotations

import numpy as np

from conftest import GOLDEN


def test_chunglu18k_fixture_matches_generator(dm):
    from dumato_b200 import workloads

    z = np.load(GOLDEN / "chunglu18k_s1.npz")
    u, v = workloads.make("chunglu18k", 1).edges()
    assert np.array_equal(z["u"], u) and np.array_equal(z["v"], v)
    assert z["u"].size == 198_000
