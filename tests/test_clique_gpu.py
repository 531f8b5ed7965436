"""GPU k-clique counts against the CPU oracle (bit-exact uint64)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _oracle_graph(orc, g):
    u, v = g.edges()
    return orc.OracleGraph.from_pairs(u, v)


def test_toy_graph_known_answers(dm, gpu):
    g = dm.Graph.load_edgelist(GOLDEN / "test.edgelist")
    assert dm.count_cliques(g, 3)[0] == 2
    assert dm.count_cliques(g, 4)[0] == 0
    assert dm.count_cliques(g, 2)[0] == 6


@pytest.mark.parametrize("k", [3, 4, 5, 6, 7])
def test_citeseer_vs_oracle(dm, orc, gpu, k):
    g = dm.Graph.load_edgelist(GOLDEN / "citeseer.edgelist")
    og = orc.OracleGraph.load(GOLDEN / "citeseer.edgelist")
    assert dm.count_cliques(g, k)[0] == orc.clique_dfs(og, k)


@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("k", [3, 4])
def test_er2k_vs_plain_dfs(dm, orc, gpu, seed, k):
    from dumato_b200 import workloads

    g = workloads.make("er2k", seed)
    og = _oracle_graph(orc, g)
    assert dm.count_cliques(g, k)[0] == orc.clique_dfs(og, k)


@pytest.mark.parametrize("k", [4, 5, 6, 7])
def test_chunglu18k_vs_oracle(dm, orc, gpu, k):
    from dumato_b200 import workloads

    g = workloads.make("chunglu18k", 1)
    og = _oracle_graph(orc, g)
    want = orc.clique_dfs(og, k)
    assert want == orc.clique_dag_bytes(og, k)[0]
    for mode in (dm.MODE_AUTO, dm.MODE_LIST):
        got, st = dm.count_cliques(g, k, dm.Options(mode=mode))
        assert got == want, (mode, got, want)


@pytest.mark.parametrize("k", [4, 5, 6])
def test_rmat100k_vs_oracle(dm, orc, gpu, k):
    from dumato_b200 import workloads

    g = workloads.make("rmat100k", 1)
    og = _oracle_graph(orc, g)
    want, _ = orc.clique_dag_bytes(og, k)
    got, _ = dm.count_cliques(g, k)
    assert got == want
    got_list, _ = dm.count_cliques(g, k, dm.Options(mode=dm.MODE_LIST))
    assert got_list == want


def test_sharded_roots_sum_to_total(dm, gpu):
    from dumato_b200 import workloads

    g = workloads.make("chunglu18k", 2)
    total = dm.count_cliques(g, 4)[0]
    parts = [dm.count_cliques(g, 4, dm.Options(rank=r, world_size=3))[0] for r in range(3)]
    assert sum(parts) == total and all(p > 0 for p in parts)


def test_reference_launch_shape_arguments(dm, gpu):
    # the reference's recommended "102400 256" threads/blockSize pair
    from dumato_b200 import workloads

    g = workloads.make("er2k", 1)
    a = dm.count_cliques(g, 3)[0]
    b = dm.count_cliques(g, 3, dm.Options(threads=102400, block_size=256))[0]
    assert a == b


def test_dense_roots_use_warp_and_list_modes(dm, orc, gpu):
    # a graph whose top roots have out-degree > 128 and > 2048 exercises warp and list mode
    rng = np.random.default_rng(7)
    n = 3000
    core = rng.choice(n, 300, replace=False)
    src, dst = [], []
    for i in range(len(core)):
        for j in range(i + 1, len(core)):
            if rng.random() < 0.6:
                src.append(core[i]); dst.append(core[j])
    s2 = rng.integers(0, n, 20000); d2 = rng.integers(0, n, 20000)
    src = np.concatenate([np.array(src), s2]); dst = np.concatenate([np.array(dst), d2])
    g = dm.Graph.from_edges(src, dst)
    og = orc.OracleGraph.from_pairs(src, dst)
    assert g.info().max_out_degree > 128
    for k in (3, 4, 5):
        want = orc.clique_dag_bytes(og, k)[0]
        assert dm.count_cliques(g, k)[0] == want
        assert dm.count_cliques(g, k, dm.Options(mode=dm.MODE_LIST))[0] == want


@pytest.mark.parametrize("k", [3, 5])
def test_subtree_logger_matches_oracle(dm, orc, gpu, k):
    from dumato_b200 import workloads

    g = workloads.make("chunglu18k", 1)
    og = _oracle_graph(orc, g)
    per = np.zeros(g.info().n_vertices, np.uint64)
    total, _ = dm.count_cliques(g, k, dm.Options(subtree_counts=per))
    want = orc.clique_per_root(og, k)
    assert int(per.sum()) == total
    assert np.array_equal(per, want)


def test_donations_happen_and_stay_exact(dm, orc, gpu):
    from dumato_b200 import workloads

    g = workloads.make("rmat100k", 1)
    og = _oracle_graph(orc, g)
    want, _ = orc.clique_dag_bytes(og, 5)
    got, st = dm.count_cliques(g, 5, dm.Options(threshold=0))
    assert got == want
    assert st.donations > 0
    off, _ = dm.count_cliques(g, 5, dm.Options(threshold=100))
    assert off == want


@pytest.mark.parametrize("vwarp", [8, 16, 32])
def test_list_path_virtual_warps(dm, orc, gpu, vwarp):
    """The list path with groups of 8, 16 or 32 lanes per first-level candidate (the
    reference's DM_WCV clique variant) gives the oracle's counts, with donations on."""
    from dumato_b200 import workloads

    for g in (dm.Graph.load_edgelist(GOLDEN / "citeseer.edgelist"), workloads.make("rmat100k", 1)):
        og = _oracle_graph(orc, g)
        for k in (3, 4, 5, 6):
            want = orc.clique_dag_bytes(og, k)[0]
            got, st = dm.count_cliques(g, k, dm.Options(mode=dm.MODE_LIST, vwarp=vwarp,
                                                        test_flags=dm.TEST_EAGER_DONATION))
            assert got == want, (vwarp, k)
            assert st.vwarp_used == vwarp
