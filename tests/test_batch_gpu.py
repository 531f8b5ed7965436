"""Batched mining (one persistent, CUDA-graph-captured launch over many graphs and queries)
against the CPU oracle and the single-query entry points."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _small_batch(dm, seed, n_graphs=24, nmax=400):
    """Chung-Lu graphs small enough for the oracle, one query each (cliques k = 3..6, motifs
    k = 3..5), in the shape of the batched workload."""
    rng = np.random.default_rng(seed)
    kinds = [(dm.QUERY_CLIQUE, 3), (dm.QUERY_CLIQUE, 4), (dm.QUERY_CLIQUE, 5), (dm.QUERY_CLIQUE, 6),
             (dm.QUERY_MOTIF, 3), (dm.QUERY_MOTIF, 4), (dm.QUERY_MOTIF, 5)]
    dicts = {k: dm.Dictionary.generate(k) for k in (3, 4, 5)}
    queries = []
    for i in range(n_graphs):
        n = int(rng.integers(50, nmax))
        avg = float(min(rng.uniform(4, 12), (n - 1) / 4))
        g = dm.Graph.generate(dm.GEN_CHUNG_LU, n, int(n * avg / 2), seed=1000 * seed + i,
                              gamma=float(rng.uniform(2.0, 2.5)), dmax=float(min(n - 1, 10 * avg)))
        kind, k = kinds[i % len(kinds)]
        queries.append(dm.Query(kind, k, g, dicts[k] if kind == dm.QUERY_MOTIF else None))
    return queries, dicts


def _oracle(dm, orc, q):
    og = orc.OracleGraph.from_pairs(*q.graph.edges())
    if q.kind == dm.QUERY_CLIQUE:
        return orc.clique_dfs(og, q.k)
    q2c = q.dictionary.tables()[0]
    return orc.motifs(og, q.k, q2c, q.dictionary.n_classes)


def _same(a, b):
    return a == b if isinstance(a, int) else np.array_equal(a, b)


def test_batch_matches_oracle_and_replays(dm, orc, gpu):
    queries, _ = _small_batch(dm, seed=1)
    want = [_oracle(dm, orc, q) for q in queries]
    b = dm.Batch(queries)
    for _ in range(3):  # the captured launch replays with fresh counters
        got, st = b.run()
        assert all(_same(g, w) for g, w in zip(got, want))
        assert st.kernel_launches == 1 and st.kernel_ms > 0
    b.close()


@pytest.mark.parametrize("vwarp", [8, 16, 32])
def test_batch_forced_settings(dm, orc, gpu, vwarp):
    queries, _ = _small_batch(dm, seed=2, n_graphs=14)
    want = [_oracle(dm, orc, q) for q in queries]
    for mode in (dm.MODE_LIST, dm.MODE_BITMAP):
        for thr in (0, 100):
            qs = [dm.Query(q.kind, q.k, q.graph, q.dictionary, vwarp=vwarp, threshold=thr, mode=mode) for q in queries]
            b = dm.Batch(qs, opts=dm.Options(test_flags=dm.TEST_EAGER_DONATION))
            got, _ = b.run()
            assert all(_same(g, w) for g, w in zip(got, want)), (vwarp, mode, thr)
            for i, q in enumerate(qs):
                t = b.tuning(i)
                assert t.threshold == thr
                if q.kind == dm.QUERY_MOTIF:
                    assert t.vwarp == vwarp
                else:
                    assert t.mode == mode
            b.close()


def test_batch_measured_autotune(dm, orc, gpu):
    queries, _ = _small_batch(dm, seed=3, n_graphs=7)
    want = [_oracle(dm, orc, q) for q in queries]
    b = dm.Batch(queries, autotune=dm.AUTOTUNE_MEASURE)
    got, _ = b.run()
    assert all(_same(g, w) for g, w in zip(got, want))
    for i, q in enumerate(queries):
        t = b.tuning(i)
        assert t.tune_ms > 0
        assert t.vwarp in (8, 16, 32) and t.threshold in (0, 100)


def test_batched_workload_matches_single_queries(dm, gpu):
    """A slice of the 256-graph batched workload: every query's result equals the
    single-graph entry point's (which the other tests pin to the oracle)."""
    from dumato_b200 import workloads

    queries, _graphs, _dicts = workloads.make_batch(seed=1, n_graphs=40)
    b = dm.Batch(queries)
    got, st = b.run()
    for q, g in zip(queries, got):
        if q.kind == dm.QUERY_CLIQUE:
            w, _ = dm.count_cliques(q.graph, q.k)
        else:
            w, _ = dm.count_motifs(q.graph, q.k, q.dictionary)
        assert _same(g, w)
