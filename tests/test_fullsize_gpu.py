"""Parity at the benchmark configurations' full sizes (GPU against the CPU oracle).

- Large skewed R-MAT graph (~321k vertices, 1.05M edges): k-cliques k = 3..7 in both
  intersection modes against the oracle's DAG enumerator.
- Mid-size R-MAT graph (~98.6k vertices, 1.08M edges): triangles against the oracle; the
  whole-graph 3- and 4-vertex motif histograms (5.9e11 connected 4-subgraphs, beyond any
  enumerator on a CPU) against closed-form counts computed by the oracle without
  enumeration; 4- and 5-vertex motifs per class on single-root shards of the full graph
  against the enumerating oracle (which restates the reference's extend + canonical filter
  + quick-code aggregation) for the same roots.
- The full 256-graph batched workload: every query against the single-query entry points,
  clique queries against the oracle, 3- and 4-vertex motif queries against closed forms.
Counts are exact integers: the tolerance is zero everywhere.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHARD_WORLD = 1 << 24  # a shard of this world holds exactly one root (its plan index)


@pytest.fixture(scope="module")
def rmat317k(dm, orc):
    from dumato_b200 import workloads

    g = workloads.make("rmat317k", 1)
    return g, orc.OracleGraph.from_pairs(*g.edges())


@pytest.fixture(scope="module")
def rmat100k(dm, orc):
    from dumato_b200 import workloads

    g = workloads.make("rmat100k", 1)
    return g, orc.OracleGraph.from_pairs(*g.edges())


@pytest.mark.parametrize("k", [3, 4, 5, 6, 7])
def test_rmat317k_cliques_vs_oracle(dm, orc, gpu, rmat317k, k):
    g, og = rmat317k
    want, _ = orc.clique_dag_bytes(og, k)
    assert want > 0
    for mode in (dm.MODE_AUTO, dm.MODE_LIST):
        got, _ = dm.count_cliques(g, k, dm.Options(mode=mode))
        assert got == want, (mode, got, want)


def test_rmat100k_triangles_vs_oracle(dm, orc, gpu, rmat100k):
    g, og = rmat100k
    want, _ = orc.clique_dag_bytes(og, 3)
    for mode in (dm.MODE_AUTO, dm.MODE_LIST):
        assert dm.count_cliques(g, 3, dm.Options(mode=mode))[0] == want


def _types(orc, d):
    q2c, _ = d.tables()
    return orc.class_types4(q2c, d.n_classes)


def _by_type(types, hist):
    out = {}
    for c, t in enumerate(types):
        if t is not None:
            out[t] = out.get(t, 0) + int(hist[c])
        else:
            assert int(hist[c]) == 0
    return out


def _closed_form_k3(orc, og, g):
    off, _ = g.csr()
    deg = np.diff(off).astype(np.int64)
    tri, _ = orc.clique_dag_bytes(og, 3)
    return int((deg * (deg - 1) // 2).sum()) - 3 * tri, tri  # open wedges, triangles


def _check_k3(dm, orc, g, og, hist, d):
    wedges, tri = _closed_form_k3(orc, og, g)
    _, code = d.tables()
    tri_cls = int(np.where(code == 7)[0][0])
    assert int(hist[tri_cls]) == tri
    assert int(hist.sum()) - tri == wedges


@pytest.mark.parametrize("name", ["rmat100k", "rmat317k"])
def test_full_size_motifs_k3_closed_form(dm, orc, gpu, request, name):
    g, og = request.getfixturevalue(name)
    d = dm.Dictionary.generate(3)
    hist, _ = dm.count_motifs(g, 3, d)
    _check_k3(dm, orc, g, og, hist, d)


@pytest.mark.parametrize("name", ["rmat100k", "rmat317k"])
def test_full_size_motifs_k4_closed_form(dm, orc, gpu, request, name):
    """Every connected 4-vertex class of the whole graph against the oracle's closed form."""
    g, og = request.getfixturevalue(name)
    d = dm.Dictionary.generate(4)
    hist, _ = dm.count_motifs(g, 4, d)
    assert _by_type(_types(orc, d), hist) == orc.graphlet4(og)


@pytest.mark.parametrize("k,index", [(4, 20000), (4, 60000), (5, 65000), (5, 73000)])
def test_rmat100k_motif_root_shards_vs_oracle(dm, orc, gpu, rmat100k, k, index):
    """Single-root shards of the full graph (the root at a fixed position of the plan), per
    class against the enumerating oracle for the same root."""
    g, og = rmat100k
    d = dm.Dictionary.generate(k)
    q2c, _ = d.tables()
    opts = dm.Options(rank=index, world_size=SHARD_WORLD)
    roots, _ = dm.plan_roots(g, k, clique=False, opts=opts)
    assert roots.size == 1
    got, st = dm.count_motifs(g, k, d, opts)
    want = orc.motifs_roots(og, k, q2c, d.n_classes, roots)
    assert int(want.sum()) > 0
    assert np.array_equal(got, want)


def test_full_batched_workload(dm, orc, gpu):
    """All 256 queries of the batched workload in one replay: each against the single-query
    entry point, clique queries against the oracle's DAG enumerator, 3- and 4-vertex motif
    queries against the closed forms."""
    from dumato_b200 import workloads

    queries, _graphs, _dicts = workloads.make_batch(seed=1, n_graphs=256)
    b = dm.Batch(queries)
    got, st = b.run()
    assert st.kernel_launches == 1
    checked = {"single": 0, "oracle": 0, "closed_form": 0}
    for q, res in zip(queries, got):
        og = orc.OracleGraph.from_pairs(*q.graph.edges())
        if q.kind == dm.QUERY_CLIQUE:
            single, _ = dm.count_cliques(q.graph, q.k)
            assert res == single
            assert res == orc.clique_dag_bytes(og, q.k)[0]
            checked["oracle"] += 1
        else:
            single, _ = dm.count_motifs(q.graph, q.k, q.dictionary)
            assert np.array_equal(res, single)
            if q.k == 3:
                _check_k3(dm, orc, q.graph, og, res, q.dictionary)
                checked["closed_form"] += 1
            elif q.k == 4:
                assert _by_type(_types(orc, q.dictionary), res) == orc.graphlet4(og)
                checked["closed_form"] += 1
        checked["single"] += 1
    assert checked["single"] == 256 and checked["oracle"] > 0 and checked["closed_form"] > 0
    b.close()
