"""Host-side checks of the batched entry point (argument validation needs no GPU)."""
from __future__ import annotations

import pytest


def test_batch_rejects_bad_queries(dm):
    g = dm.Graph.from_edges([0, 1, 2], [1, 2, 0])
    with pytest.raises(dm.DMError, match="clique k must be in"):
        dm.Batch([dm.Query(dm.QUERY_CLIQUE, 9, g)])
    with pytest.raises(ValueError, match="needs its k-vertex dictionary"):
        dm.Batch([dm.Query(dm.QUERY_MOTIF, 4, g)])
    d3 = dm.Dictionary.generate(3)
    with pytest.raises(dm.DMError, match="needs the k-vertex dictionary"):
        dm.Batch([dm.Query(dm.QUERY_MOTIF, 4, g, d3)])
    with pytest.raises(dm.DMError, match="vwarp"):
        dm.Batch([dm.Query(dm.QUERY_CLIQUE, 3, g, vwarp=12)])
    with pytest.raises(dm.DMError, match="autotune"):
        dm.Batch([dm.Query(dm.QUERY_CLIQUE, 3, g)], autotune=7)


def test_batched_workload_shape(dm):
    from dumato_b200 import workloads

    specs = workloads.batch_specs(seed=1, n_graphs=256)
    assert len(specs) == 256
    assert all(50 <= s["n"] <= 5000 and 2.0 <= s["gamma"] <= 2.5 for s in specs)
    assert {(s["query"], s["k"]) for s in specs} == set(workloads.BATCH_QUERIES)
    assert all(2 * s["m"] / s["n"] <= 40.0 + 1e-9 for s in specs)
