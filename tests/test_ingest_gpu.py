"""Edgelist ingest on the GPU against the host reader: the same graph (CSR, orientation,
counts, statistics) and the same format errors."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _same_graph(dm, a, b):
    ia, ib = a.info(), b.info()
    for f in ("n_vertices", "n_edges", "max_degree", "max_out_degree", "n_self_loops", "n_input_pairs"):
        assert getattr(ia, f) == getattr(ib, f), f
    oa, xa = a.csr()
    ob, xb = b.csr()
    assert np.array_equal(oa, ob) and np.array_equal(xa, xb)
    ua, va = a.edges()
    ub, vb = b.edges()
    assert np.array_equal(ua, ub) and np.array_equal(va, vb)


@pytest.mark.parametrize("name", ["test", "citeseer"])
def test_device_ingest_reference_files(dm, gpu, name):
    path = GOLDEN / f"{name}.edgelist"
    g, ms = dm.Graph.load_edgelist_device(path)
    assert ms > 0
    _same_graph(dm, g, dm.Graph.load_edgelist(path))


@pytest.mark.parametrize("name", ["er2k", "chunglu18k", "rmat100k"])
def test_device_ingest_workloads(dm, orc, gpu, tmp_path, name):
    from dumato_b200 import workloads

    src = workloads.make(name, 1)
    path = tmp_path / f"{name}.edgelist"
    src.write_edgelist(path)
    g, _ = dm.Graph.load_edgelist_device(path)
    h = dm.Graph.load_edgelist(path)
    _same_graph(dm, g, h)
    for k in (3, 4):  # the orientation drives the clique engine
        assert dm.count_cliques(g, k)[0] == dm.count_cliques(h, k)[0]


def test_device_ingest_separators_comments_duplicates(dm, gpu, tmp_path):
    text = ("# a comment line\n0 1\r\n1 0\n2,3\n3 3\n% another comment\n4 2 # trailing comment 9 9\n"
            "1\t2\n\n0 1\n7 5\n")
    path = tmp_path / "mixed.edgelist"
    path.write_text(text)
    g, _ = dm.Graph.load_edgelist_device(path)
    h = dm.Graph.load_edgelist(path)
    _same_graph(dm, g, h)
    info = g.info()
    assert (info.n_vertices, info.n_edges, info.n_self_loops, info.n_input_pairs) == (8, 5, 1, 8)


@pytest.mark.parametrize("text", ["0 1\n2 -3\n", "0 1\n2 x\n", "0 1 2\n", "0 4294967296\n"])
def test_device_ingest_format_errors(dm, gpu, tmp_path, text):
    path = tmp_path / "bad.edgelist"
    path.write_text(text)
    with pytest.raises(dm.DMError) as host_err:
        dm.Graph.load_edgelist(path)
    with pytest.raises(dm.DMError) as dev_err:
        dm.Graph.load_edgelist_device(path)
    assert dev_err.value.status == host_err.value.status == -3


def test_device_ingest_empty_file(dm, gpu, tmp_path):
    path = tmp_path / "empty.edgelist"
    path.write_text("")
    g, _ = dm.Graph.load_edgelist_device(path)
    assert g.info().n_vertices == 0 and g.info().n_edges == 0
