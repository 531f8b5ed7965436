"""Writes the edge set of the benchmark's Chung-Lu workload (18,700 vertices, 198,000
undirected edges, exponent 2.1, max degree 500, seed 1) to tests/golden/chunglu18k_s1.npz
as (u < v) pairs, so that processes which must not load this library (the CPU reference
arm of bench.py) read the very graph the GPU arm counts. tests/test_workload_fixture.py
checks that the file still equals the generator's output.

    python tests/golden/make_workload_fixture.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
OUT = ROOT / "tests" / "golden" / "chunglu18k_s1.npz"


def main() -> None:
    sys.path.insert(0, str(ROOT))
    from dumato_b200 import workloads

    u, v = workloads.make("chunglu18k", 1).edges()
    np.savez_compressed(OUT, u=u.astype(np.int32), v=v.astype(np.int32))
    print(OUT, u.size)


if __name__ == "__main__":
    main()
