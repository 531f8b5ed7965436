"""GPU motif counts (per class, uint64) against the CPU oracle and the reference's tables."""
from __future__ import annotations

import json

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _dict(dm, k):
    d = dm.Dictionary.generate(k)
    return d, d.tables()[0]


def test_toy_graph_known_answers(dm, gpu):
    g = dm.Graph.load_edgelist(GOLDEN / "test.edgelist")
    for k, total in ((3, 7), (4, 4)):
        d, _ = _dict(dm, k)
        h, _ = dm.count_motifs(g, k, d)
        assert int(h.sum()) == total and int(h[~d.connected()].sum()) == 0


@pytest.mark.parametrize("k", [3, 4, 5])
def test_citeseer_vs_oracle(dm, orc, gpu, k):
    g = dm.Graph.load_edgelist(GOLDEN / "citeseer.edgelist")
    og = orc.OracleGraph.load(GOLDEN / "citeseer.edgelist")
    d, q2c = _dict(dm, k)
    got, _ = dm.count_motifs(g, k, d)
    assert np.array_equal(got, orc.motifs(og, k, q2c, d.n_classes))


@pytest.mark.parametrize("k", [3, 4, 5, 6])
def test_er2k_vs_oracle(dm, orc, gpu, k):
    from dumato_b200 import workloads

    g = workloads.make("er2k", 1)
    og = orc.OracleGraph.from_pairs(*g.edges())
    d, q2c = _dict(dm, k)
    got, st = dm.count_motifs(g, k, d)
    assert np.array_equal(got, orc.motifs(og, k, q2c, d.n_classes))


@pytest.mark.parametrize("k", [3, 4])
def test_skewed_rmat_vs_oracle(dm, orc, gpu, k):
    g = dm.Graph.generate(dm.GEN_RMAT, 2000, 8000, seed=3)
    og = orc.OracleGraph.from_pairs(*g.edges())
    d, q2c = _dict(dm, k)
    got, _ = dm.count_motifs(g, k, d)
    assert np.array_equal(got, orc.motifs(og, k, q2c, d.n_classes))


def test_k7_small_graph_vs_brute_force(dm, orc, gpu):
    rng = np.random.default_rng(11)
    n = 14
    s, t = rng.integers(0, n, 45), rng.integers(0, n, 45)
    g = dm.Graph.from_edges(s, t)
    og = orc.OracleGraph.from_pairs(s, t)
    for k in (6, 7):
        d, q2c = _dict(dm, k)
        got, _ = dm.count_motifs(g, k, d)
        assert np.array_equal(got, orc.motifs_brute(og, k, q2c, d.n_classes))


@pytest.mark.parametrize("k", [3, 4, 5, 6])
def test_reference_dictionary_gives_reference_class_ids(dm, orc, gpu, tmp_path, k):
    z = np.load(GOLDEN / f"ref_dict_{k}.npz")
    rq2c, rcode = z["quick_to_class"], z["class_code"]
    p = tmp_path / f"{k}.csv"
    with open(p, "w") as f:
        f.write(f"#quick,cg_local\n{rq2c.size}\n" + "".join(f"{q},{c}\n" for q, c in enumerate(rq2c)))
        f.write(f"#cg_local,cg_global\n{rcode.size}\n" + "".join(f"{c},{int(x)}\n" for c, x in enumerate(rcode)))
    ref_d = dm.Dictionary.load_csv(p)
    g = dm.Graph.load_edgelist(GOLDEN / "citeseer.edgelist")
    og = orc.OracleGraph.load(GOLDEN / "citeseer.edgelist")
    got, _ = dm.count_motifs(g, k, ref_d)
    assert np.array_equal(got, orc.motifs(og, k, rq2c, rcode.size))
    # same multiset as with the self-generated dictionary
    mine, _ = dm.count_motifs(g, k, dm.Dictionary.generate(k))
    assert sorted(got.tolist()) == sorted(mine.tolist())


def test_sharding_and_subtree_log(dm, gpu):
    from dumato_b200 import workloads

    g = workloads.make("er2k", 2)
    d, _ = _dict(dm, 4)
    total, _ = dm.count_motifs(g, 4, d)
    parts = [dm.count_motifs(g, 4, d, dm.Options(rank=r, world_size=3))[0] for r in range(3)]
    assert np.array_equal(sum(parts), total)
    per = np.zeros(g.info().n_vertices, np.uint64)
    got, _ = dm.count_motifs(g, 4, d, dm.Options(subtree_counts=per))
    assert int(per.sum()) == int(total.sum())


def test_full_size_rmat100k_k3_closed_form(dm, gpu):
    """Connected 3-subgraphs = open wedges + triangles = sum C(d,2) - 2T."""
    from dumato_b200 import workloads

    g = workloads.make("rmat100k", 1)
    off, _ = g.csr()
    deg = np.diff(off).astype(np.int64)
    tri, _ = dm.count_cliques(g, 3)
    d, _ = _dict(dm, 3)
    h, _ = dm.count_motifs(g, 3, d)
    assert int(h.sum()) == int((deg * (deg - 1) // 2).sum()) - 2 * tri
    # the triangle class is the complete-graph class (code 7)
    q2c, code = d.tables()
    assert int(h[int(np.where(code == 7)[0][0])]) == tri


def test_matches_reference_binaries(dm, gpu, tmp_path):
    path = GOLDEN / "ref_counts.json"
    if not path.exists():
        pytest.skip("reference counts fixture not generated")
    ref = json.loads(path.read_text())
    from dumato_b200 import workloads

    graphs = {"test": lambda: dm.Graph.load_edgelist(GOLDEN / "test.edgelist"),
              "citeseer": lambda: dm.Graph.load_edgelist(GOLDEN / "citeseer.edgelist"),
              "er2k_s1": lambda: workloads.make("er2k", 1),
              "rmat2k_s3": lambda: dm.Graph.generate(dm.GEN_RMAT, 2000, 8000, seed=3),
              "chunglu18k_s1": lambda: workloads.make("chunglu18k", 1),
              "rmat317k_s1": lambda: workloads.make("rmat317k", 1)}
    for name, entry in ref.items():
        g = graphs[name]()
        for key in ("clique", "clique_lb_threshold30"):
            for k, c in entry.get(key, {}).items():
                assert dm.count_cliques(g, int(k))[0] == c, (name, key, k)
        for k, mot in entry["motifs"].items():
            k = int(k)
            z = np.load(GOLDEN / f"ref_dict_{k}.npz")
            p = tmp_path / f"{name}_{k}.csv"
            with open(p, "w") as f:
                q, c = z["quick_to_class"], z["class_code"]
                f.write(f"#quick,cg_local\n{q.size}\n" + "".join(f"{i},{x}\n" for i, x in enumerate(q)))
                f.write(f"#cg_local,cg_global\n{c.size}\n" + "".join(f"{i},{int(x)}\n" for i, x in enumerate(c)))
            got, _ = dm.count_motifs(g, k, dm.Dictionary.load_csv(p))
            want = np.zeros_like(got)
            for cls, cnt in mot["classes"].items():
                want[int(cls)] = cnt
            assert np.array_equal(got, want), (name, k)


def _hub_graph(hub_deg, seed):
    """Vertex 0 (the lowest id, so a root) is adjacent to hub 1 and a few others; the hub has
    `hub_deg` neighbours, so the item (root 0, second vertex 1) holds most of the work."""
    rng = np.random.default_rng(seed)
    n = 600
    src = [0] * 11 + [1] * hub_deg
    dst = [1] + list(rng.choice(np.arange(2, n), 10, replace=False)) + list(rng.choice(np.arange(2, n), hub_deg, replace=False))
    s, t = rng.integers(2, n, 1500), rng.integers(2, n, 1500)
    return np.concatenate([np.array(src), s]), np.concatenate([np.array(dst), t])


@pytest.mark.parametrize("k,hub_deg", [(4, 250), (5, 120), (6, 60), (7, 36)])
def test_hub_item_split_by_prefix_donation(dm, orc, gpu, k, hub_deg):
    """Donated DFS prefixes (path replay on the receiving warp) give the oracle's counts."""
    src, dst = _hub_graph(hub_deg, seed=k)
    g = dm.Graph.from_edges(src, dst)
    og = orc.OracleGraph.from_pairs(*g.edges())
    d, q2c = _dict(dm, k)
    want = orc.motifs(og, k, q2c, d.n_classes)
    plain, _ = dm.count_motifs(g, k, d)
    assert np.array_equal(plain, want)
    for _ in range(2):
        eager, st = dm.count_motifs(g, k, d, dm.Options(test_flags=dm.TEST_EAGER_DONATION))
        assert np.array_equal(eager, want)
        assert st.prefix_donations > 0 and st.donations >= st.prefix_donations


@pytest.mark.parametrize("vwarp", [8, 16])
@pytest.mark.parametrize("k", [3, 4, 5, 6])
def test_virtual_warps_vs_oracle(dm, orc, gpu, vwarp, k):
    """Groups of 8 or 16 lanes sharing a task's second vertices give the oracle's counts."""
    from dumato_b200 import workloads

    g = workloads.make("er2k", 2)
    og = orc.OracleGraph.from_pairs(*g.edges())
    d, q2c = _dict(dm, k)
    want = orc.motifs(og, k, q2c, d.n_classes)
    got, st = dm.count_motifs(g, k, d, dm.Options(vwarp=vwarp))
    assert st.vwarp_used == vwarp
    assert np.array_equal(got, want)


@pytest.mark.parametrize("vwarp", [8, 16])
def test_virtual_warps_with_prefix_donation(dm, orc, gpu, vwarp):
    src, dst = _hub_graph(120, seed=5)
    g = dm.Graph.from_edges(src, dst)
    og = orc.OracleGraph.from_pairs(*g.edges())
    d, q2c = _dict(dm, 5)
    want = orc.motifs(og, 5, q2c, d.n_classes)
    got, st = dm.count_motifs(g, 5, d, dm.Options(vwarp=vwarp, test_flags=dm.TEST_EAGER_DONATION))
    assert np.array_equal(got, want)
    assert st.prefix_donations > 0
