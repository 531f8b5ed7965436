"""k-clique counting on the clique index (per-root local bitmaps built once per device copy
of the graph) against the CPU oracle, with both ways of staging a root's block into shared
memory (bulk asynchronous copies and 16-byte loads), and against the per-launch rebuild.
Counts are exact: zero tolerance."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

STAGINGS = ("tma", "loads")


def _opts(dm, staging, **kw):
    return dm.Options(staging=dm.STAGE_TMA if staging == "tma" else dm.STAGE_LOADS, **kw)


def _og(orc, g):
    return orc.OracleGraph.from_pairs(*g.edges())


def _dense_core(dm, seed=3, core=110, p=0.75, n=4000, extra=30000):
    """A near-clique of `core` vertices inside a sparse graph: DAG out-degrees up to ~80 (two
    words per bitmap row) and items whose candidate sets hold dozens of vertices."""
    rng = np.random.default_rng(seed)
    ids = rng.choice(n, core, replace=False)
    iu = np.triu_indices(core, 1)
    keep = rng.random(iu[0].size) < p
    s = np.concatenate([ids[iu[0][keep]], rng.integers(0, n, extra)])
    t = np.concatenate([ids[iu[1][keep]], rng.integers(0, n, extra)])
    return dm.Graph.from_edges(s, t)


@pytest.mark.parametrize("staging", STAGINGS)
def test_index_small_graphs(dm, orc, gpu, staging):
    g = dm.Graph.load_edgelist(GOLDEN / "citeseer.edgelist")
    og = _og(orc, g)
    for k in range(3, 9):
        got, st = dm.count_cliques(g, k, _opts(dm, staging))
        assert got == orc.clique_dag_bytes(og, k)[0], k
        assert st.mode_used == dm.MODE_BITMAP
    g = dm.Graph.load_edgelist(GOLDEN / "test.edgelist")
    assert dm.count_cliques(g, 3, _opts(dm, staging))[0] == 2


@pytest.mark.parametrize("staging", STAGINGS)
@pytest.mark.parametrize("name", ["chunglu18k", "rmat100k"])
def test_index_workloads(dm, orc, gpu, staging, name):
    from dumato_b200 import workloads

    g = workloads.make(name, 1)
    og = _og(orc, g)
    for k in (3, 4, 5, 6, 7, 8):
        want = orc.clique_dag_bytes(og, k)[0]
        got, st = dm.count_cliques(g, k, _opts(dm, staging))
        assert got == want, (name, k)
        assert st.mode_used == dm.MODE_BITMAP
        assert dm.count_cliques(g, k, dm.Options(mode=dm.MODE_REBUILD))[0] == want


@pytest.mark.parametrize("staging", STAGINGS)
def test_index_dense_core_level1_donations(dm, orc, gpu, staging):
    """Heavy items (candidate sets of 24+ vertices at k >= 6) run as position ranges that
    hungry warps take over: donations below the first level, and exact counts."""
    g = _dense_core(dm)
    og = _og(orc, g)
    assert g.info().max_out_degree > 64
    for k in (6, 7, 8):
        want = orc.clique_dag_bytes(og, k)[0]
        assert want > 0
        got, st = dm.count_cliques(g, k, _opts(dm, staging, test_flags=dm.TEST_EAGER_DONATION))
        assert got == want, k
        assert st.prefix_donations > 0
        off, _ = dm.count_cliques(g, k, _opts(dm, staging, threshold=100))
        assert off == want


@pytest.mark.parametrize("staging", STAGINGS)
def test_index_list_roots_beside_index_roots(dm, orc, gpu, staging):
    """Roots above 256 out-neighbours take the list path inside the index kernel, next to
    roots counted from their index blocks."""
    g = _dense_core(dm, seed=9, core=300, p=0.95, n=3000, extra=20000)
    og = _og(orc, g)
    assert g.info().max_out_degree > 256
    for k in (3, 4):
        got, st = dm.count_cliques(g, k, _opts(dm, staging))
        assert got == orc.clique_dag_bytes(og, k)[0], k
        assert st.mode_used == dm.MODE_BITMAP


@pytest.mark.parametrize("staging", STAGINGS)
def test_index_schedules_shards_and_logger(dm, orc, gpu, staging):
    from dumato_b200 import workloads

    g = workloads.make("chunglu18k", 2)
    og = _og(orc, g)
    k = 5
    want = orc.clique_dag_bytes(og, k)[0]
    assert dm.count_cliques(g, k, _opts(dm, staging, scheduler=dm.SCHED_ID))[0] == want
    parts = [dm.count_cliques(g, k, _opts(dm, staging, rank=r, world_size=3))[0] for r in range(3)]
    assert sum(parts) == want
    per = np.zeros(g.info().n_vertices, np.uint64)
    total, _ = dm.count_cliques(g, k, _opts(dm, staging, subtree_counts=per))
    assert total == want
    assert np.array_equal(per, orc.clique_per_root(og, k))


def test_index_rebuilt_after_release(dm, orc, gpu):
    from dumato_b200 import workloads

    g = workloads.make("er2k", 3)
    want = orc.clique_dag_bytes(_og(orc, g), 3)[0]
    for _ in range(3):
        assert dm.count_cliques(g, 3)[0] == want
        g.release_device()


def test_live_reports_during_a_count(dm, orc, gpu):
    """A report function set in the options is called every report_ms while the counting
    kernel runs, with the warps' occupancy and the tasks dealt so far; counts are unchanged."""
    from dumato_b200 import workloads

    g = workloads.make("rmat100k", 1)
    want = orc.clique_dag_bytes(_og(orc, g), 7)[0]
    samples = []
    got, st = dm.count_cliques(g, 7, dm.Options(threshold=100, report=samples.append, report_ms=2))
    assert got == want
    assert len(samples) >= 2, (len(samples), st.kernel_ms)
    assert all(0 <= s["hungry_warps"] <= s["warps"] and s["roots_claimed"] <= s["roots_total"] for s in samples)
    claimed = [s["roots_claimed"] for s in samples]
    assert claimed == sorted(claimed)
    assert [s["elapsed_ms"] for s in samples] == sorted(s["elapsed_ms"] for s in samples)


@pytest.mark.parametrize("name", ["citeseer", "chunglu18k", "rmat100k", "rmat317k", "dense"])
def test_fused_counts_every_size(dm, orc, gpu, name):
    """One launch counts every clique size 3..8, each equal to the oracle's count, with and
    without eager donation (level-0 and level-1 donations carry the fused counts too)."""
    from dumato_b200 import workloads

    if name == "citeseer":
        g = dm.Graph.load_edgelist(GOLDEN / "citeseer.edgelist")
    elif name == "dense":
        g = _dense_core(dm)
    else:
        g = workloads.make(name, 1)
    og = _og(orc, g)
    want = {k: orc.clique_dag_bytes(og, k)[0] for k in range(3, 9)}
    first, st = dm.count_cliques_upto(g, 8)  # also builds the graph's clique index (a second launch)
    assert first == want and st.kernel_launches <= 2
    for flags in (0, dm.TEST_EAGER_DONATION):
        got, st = dm.count_cliques_upto(g, 8, dm.Options(test_flags=flags))
        assert got == want, (name, flags)
        assert st.kernel_launches == 1
    got6, _ = dm.count_cliques_upto(g, 6)
    assert got6 == {k: want[k] for k in range(3, 7)}


def test_fused_counts_fall_back_per_size(dm, orc, gpu):
    """Where the fused walk cannot run (roots above 256 out-neighbours, list mode), the counts
    come from one launch per size and are the same."""
    g = _dense_core(dm, seed=9, core=300, p=0.95, n=3000, extra=20000)
    og = _og(orc, g)
    want = {k: orc.clique_dag_bytes(og, k)[0] for k in (3, 4)}
    got, st = dm.count_cliques_upto(g, 4)
    assert got == want and st.kernel_launches >= 2
    g2 = dm.Graph.load_edgelist(GOLDEN / "citeseer.edgelist")
    og2 = _og(orc, g2)
    got2, _ = dm.count_cliques_upto(g2, 5, dm.Options(mode=dm.MODE_LIST))
    assert got2 == {k: orc.clique_dag_bytes(og2, k)[0] for k in range(3, 6)}
