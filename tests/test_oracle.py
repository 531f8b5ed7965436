"""The CPU oracle against the reference's known answers and against brute force (CPU)."""
from __future__ import annotations

import json

import numpy as np
import pytest

from conftest import GOLDEN


def test_toy_graph_known_answers(dm, orc):
    g = orc.OracleGraph.load(GOLDEN / "test.edgelist")
    assert (g.n, g.m) == (5, 6)
    assert orc.clique_dfs(g, 3) == 2 and orc.clique_dfs(g, 4) == 0
    for k, total in ((3, 7), (4, 4)):
        d = dm.Dictionary.generate(k)
        q2c, _ = d.tables()
        h = orc.motifs(g, k, q2c, d.n_classes)
        assert int(h[d.connected()].sum()) == total and int(h[~d.connected()].sum()) == 0


def test_citeseer_stats(orc):
    g = orc.OracleGraph.load(GOLDEN / "citeseer.edgelist")
    assert (g.n, g.m, g.maxdeg) == (3264, 4536, 99)


@pytest.mark.parametrize("seed", range(6))
def test_dfs_matches_brute_force(dm, orc, seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(8, 15))
    m = int(rng.integers(n, n * (n - 1) // 2))
    s, t = rng.integers(0, n, m), rng.integers(0, n, m)  # includes self-loops and repeats
    g = orc.OracleGraph.from_pairs(s, t)
    for k in (3, 4, 5):
        assert orc.clique_dfs(g, k) == orc.clique_brute(g, k) == orc.clique_dag_bytes(g, k)[0]
        d = dm.Dictionary.generate(k)
        q2c, _ = d.tables()
        assert np.array_equal(orc.motifs(g, k, q2c, d.n_classes), orc.motifs_brute(g, k, q2c, d.n_classes))


def test_per_root_sums_to_total(orc, dm):
    from dumato_b200 import workloads

    u, v = workloads.make("er2k", 2).edges()
    g = orc.OracleGraph.from_pairs(u, v)
    assert int(orc.clique_per_root(g, 4).sum()) == orc.clique_dfs(g, 4)


def test_oracle_matches_reference_binaries(dm, orc):
    """Counts printed by the reference's own clique_PA / motifs_DM_WCLB on a B200
    (tests/golden/ref_counts.json, made by run_reference_binaries.py)."""
    path = GOLDEN / "ref_counts.json"
    if not path.exists():
        pytest.skip("reference counts fixture not generated")
    ref = json.loads(path.read_text())
    from dumato_b200 import workloads

    graphs = {"test": lambda: orc.OracleGraph.load(GOLDEN / "test.edgelist"),
              "citeseer": lambda: orc.OracleGraph.load(GOLDEN / "citeseer.edgelist"),
              "er2k_s1": lambda: orc.OracleGraph.from_pairs(*workloads.make("er2k", 1).edges()),
              "rmat2k_s3": lambda: orc.OracleGraph.from_pairs(*dm.Graph.generate(dm.GEN_RMAT, 2000, 8000, seed=3).edges())}
    for name, entry in ref.items():
        g = graphs[name]()
        for k, c in entry["clique"].items():
            assert orc.clique_dfs(g, int(k)) == c, (name, k)
        for k, mot in entry["motifs"].items():
            k = int(k)
            rq2c = np.load(GOLDEN / f"ref_dict_{k}.npz")["quick_to_class"]
            h = orc.motifs(g, k, rq2c, int(rq2c.max()) + 1)
            want = np.zeros_like(h)
            for cls, cnt in mot["classes"].items():
                want[int(cls)] = cnt
            assert np.array_equal(h, want), (name, k)
