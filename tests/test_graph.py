"""Host-side graph store: reader semantics, generators, CSR and orientation (CPU)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN


def test_reader_semantics(dm, tmp_path):
    p = tmp_path / "g.edgelist"
    # duplicate, reverse duplicate, self-loop, isolated id 6 (only reachable through max id)
    p.write_text("0 1\n1 0\n0 1\n2 2\n1 2\n3 6\n")
    g = dm.Graph.load_edgelist(p)
    i = g.info()
    assert (i.n_vertices, i.n_edges, i.n_self_loops, i.n_input_pairs) == (7, 3, 1, 6)
    u, v = g.edges()
    assert list(zip(u.tolist(), v.tolist())) == [(0, 1), (1, 2), (3, 6)]
    off, adj = g.csr()
    assert off.tolist() == [0, 1, 3, 4, 5, 5, 5, 6] and adj.tolist() == [1, 0, 2, 1, 6, 3]


@pytest.mark.parametrize("text,status", [("0 1\n2\n", -3), ("0 -1\n", -3), ("0 x\n", -3)])
def test_reader_rejects_malformed(dm, tmp_path, text, status):
    p = tmp_path / "bad.edgelist"
    p.write_text(text)
    with pytest.raises(dm.DMError) as e:
        dm.Graph.load_edgelist(p)
    assert e.value.status == status


def test_missing_file(dm, tmp_path):
    with pytest.raises(dm.DMError) as e:
        dm.Graph.load_edgelist(tmp_path / "nope")
    assert e.value.status == -2


def test_matches_oracle_reader(dm, orc):
    g = dm.Graph.load_edgelist(GOLDEN / "citeseer.edgelist")
    og = orc.OracleGraph.load(GOLDEN / "citeseer.edgelist")
    i = g.info()
    assert (i.n_vertices, i.n_edges, i.max_degree) == (og.n, og.m, og.maxdeg)


def test_generators_deterministic_and_sized(dm):
    from dumato_b200 import workloads

    for name in ("er2k", "chunglu18k"):
        a, b = workloads.make(name, 5), workloads.make(name, 5)
        assert all(np.array_equal(x, y) for x, y in zip(a.edges(), b.edges()))
        assert a.info().n_edges == workloads.CONFIGS[name]["m"]
    c = workloads.make("chunglu18k", 1).info()
    assert c.n_vertices == 18_700 and 400 <= c.max_degree <= 500
    assert not all(np.array_equal(x, y) for x, y in zip(workloads.make("er2k", 1).edges(),
                                                          workloads.make("er2k", 2).edges()))


def test_rmat_compact_relabel(dm):
    g = dm.Graph.generate(dm.GEN_RMAT, 4000, 20_000, seed=9)
    i = g.info()
    off, _ = g.csr()
    assert i.n_edges == 20_000 and (np.diff(off) > 0).all()  # every id touched


def test_round_trip_through_edgelist(dm, tmp_path):
    from dumato_b200 import workloads

    g = workloads.make("er2k", 3)
    p = tmp_path / "e.edgelist"
    g.write_edgelist(p)
    h = dm.Graph.load_edgelist(p)
    assert all(np.array_equal(x, y) for x, y in zip(g.edges(), h.edges()))


@pytest.mark.parametrize("k", [3, 5, 7])
def test_work_model_matches_oracle(dm, orc, k):
    from dumato_b200 import workloads

    g = workloads.make("chunglu18k", 1)
    og = orc.OracleGraph.from_pairs(*g.edges())
    assert dm.clique_work_model(g, k)[1] == orc.clique_dag_bytes(og, k)[1]


def test_generator_argument_errors(dm):
    with pytest.raises(dm.DMError):
        dm.Graph.generate(dm.GEN_ER, 10, 100, seed=1)
    with pytest.raises(dm.DMError):
        dm.Graph.generate(7, 10, 10, seed=1)


@pytest.mark.parametrize("k", [3, 4, 5])
def test_motif_work_model_matches_oracle_bytes(dm, orc, k):
    """The host work model walks only the internal prefixes, yet its byte total equals the
    oracle's, which charges every extension and leaf while enumerating."""
    rng = np.random.default_rng(40 + k)
    graphs = [dm.Graph.load_edgelist(GOLDEN / "citeseer.edgelist")] if k < 5 else []
    for _ in range(3):
        n = int(rng.integers(30, 90))
        s, t = rng.integers(0, n, 4 * n), rng.integers(0, n, 4 * n)
        graphs.append(dm.Graph.from_edges(s, t))
    for g in graphs:
        og = orc.OracleGraph.from_pairs(*g.edges())
        d = dm.Dictionary.generate(k)
        q2c, _ = d.tables()
        _, want = orc.motifs(og, k, q2c, d.n_classes, with_bytes=True)
        assert dm.motif_work_model(g, k)[1] == want
