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


LARGE_REF_GRAPHS = {"chunglu18k_s1": ("chunglu18k", 1), "rmat317k_s1": ("rmat317k", 1)}


def _ref_motif_check(orc, g, k, mot, large):
    """The reference's per-class counts (its own class ids) against the enumerating oracle,
    or on graphs too large to enumerate on a CPU, against the closed forms (k = 3, 4)."""
    rq2c = np.load(GOLDEN / f"ref_dict_{k}.npz")["quick_to_class"]
    ncls = int(rq2c.max()) + 1
    want = np.zeros(ncls, np.uint64)
    for cls, cnt in mot["classes"].items():
        want[int(cls)] = cnt
    if not large:
        return np.array_equal(orc.motifs(g, k, rq2c, ncls), want)
    if k == 4:
        types = orc.class_types4(rq2c, ncls)
        got = {}
        for c, t in enumerate(types):
            if t is not None:
                got[t] = got.get(t, 0) + int(want[c])
        return got == orc.graphlet4(g)
    tri, _ = orc.clique_dag_bytes(g, 3)
    return sorted(int(x) for x in want if x) == sorted([tri, int(mot["total"]) - tri])


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
    for name, (w, seed) in LARGE_REF_GRAPHS.items():
        graphs[name] = lambda w=w, seed=seed: orc.OracleGraph.from_pairs(*workloads.make(w, seed).edges())
    for name, entry in ref.items():
        g = graphs[name]()
        large = name in LARGE_REF_GRAPHS
        for key in ("clique", "clique_lb_threshold30"):
            for k, c in entry.get(key, {}).items():
                got = orc.clique_dag_bytes(g, int(k))[0] if large else orc.clique_dfs(g, int(k))
                assert got == c, (name, key, k)
        for k, mot in entry["motifs"].items():
            assert _ref_motif_check(orc, g, int(k), mot, large), (name, k)
        for q, c in entry.get("near", {}).items():
            assert orc.near_cliques(g, int(q)) == c, (name, "q", q)


def _by_type(orc, dm, og):
    d = dm.Dictionary.generate(4)
    q2c, _ = d.tables()
    types = orc.class_types4(q2c, d.n_classes)
    h = orc.motifs(og, 4, q2c, d.n_classes)
    out = {t: 0 for t in orc.GRAPHLET4_TYPES}
    for c, t in enumerate(types):
        if t is not None:
            out[t] += int(h[c])
    return out


@pytest.mark.parametrize("seed", range(4))
def test_graphlet4_closed_form_matches_enumeration(dm, orc, seed):
    """The closed-form 4-graphlet checker (used at full size, where no enumerator finishes)
    agrees with the enumerating motif oracle on random graphs with self-loops and repeats."""
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(20, 60))
    m = int(rng.integers(n, 4 * n))
    s, t = rng.integers(0, n, m), rng.integers(0, n, m)
    og = orc.OracleGraph.from_pairs(s, t)
    assert orc.graphlet4(og) == _by_type(orc, dm, og)


@pytest.mark.parametrize("name", ["citeseer", "rmat2k"])
def test_graphlet4_closed_form_on_skewed_graphs(dm, orc, name):
    if name == "citeseer":
        og = orc.OracleGraph.load(GOLDEN / "citeseer.edgelist")
    else:
        u, v = dm.Graph.generate(dm.GEN_RMAT, 2000, 8000, seed=3).edges()
        og = orc.OracleGraph.from_pairs(u, v)
    assert orc.graphlet4(og) == _by_type(orc, dm, og)


def test_class_types_of_the_reference_dictionary(dm, orc):
    """Every connected class of the k = 4 dictionary gets a distinct graphlet type."""
    d = dm.Dictionary.generate(4)
    q2c, _ = d.tables()
    types = orc.class_types4(q2c, d.n_classes)
    conn = d.connected()
    assert sorted(t for t, c in zip(types, conn) if c) == sorted(orc.GRAPHLET4_TYPES)
    assert all(t is None for t, c in zip(types, conn) if not c)


@pytest.mark.parametrize("seed", range(4))
def test_near_cliques_match_brute_force(orc, seed):
    """q_n (K_n minus one edge, non-induced) from the (n-2)-clique formula equals brute force."""
    rng = np.random.default_rng(200 + seed)
    n = int(rng.integers(10, 16))
    m = int(rng.integers(2 * n, n * (n - 1) // 2))
    s, t = rng.integers(0, n, m), rng.integers(0, n, m)
    g = orc.OracleGraph.from_pairs(s, t)
    for q in (4, 5, 6):
        assert orc.near_cliques(g, q) == orc.near_cliques_brute(g, q), q


def test_q4_is_the_diamond_subgraph_count(orc):
    """q4 counts non-induced diamonds: the closed-form checker's diamond + 6 x 4-clique total."""
    g = orc.OracleGraph.load(GOLDEN / "citeseer.edgelist")
    gl = orc.graphlet4(g)
    assert orc.near_cliques(g, 4) == gl["diamond"] + 6 * gl["clique"]
