"""dm_count_cliques_noalloc: clique counts from a caller-held device DAG, with the scratch
taken from the library's fixed device array instead of cudaMalloc.

Callers that cannot allocate GPU memory (code inside another framework's memory pool, an
allocator-free runtime, or a hook that must leave the device's allocations untouched)
use this entry point. The test builds an id-oriented DAG in device memory (allocated here
by torch, as such a caller's host framework would), calls the entry point twice in a row
through the C ABI and checks both exact counts against dm_count_cliques. Counts are
integers, so the tolerance is zero. This file is collected last on purpose.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _id_dag(g):
    """Out-neighbours above each vertex id, as (row start, degree, adjacency) arrays."""
    off, adj = g.csr()
    n = off.size - 1
    src = np.repeat(np.arange(n, dtype=np.int64), np.diff(off))
    keep = adj > src
    out_adj = adj[keep].astype(np.int32)
    deg = np.bincount(src[keep], minlength=n).astype(np.int32)
    row = np.zeros(n, np.int32)
    row[1:] = np.cumsum(deg)[:-1]
    return row, deg, out_adj


def _noalloc(dm, torch, row, deg, adj, k, max_deg=None):
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    d_row, d_deg, d_adj = dev(row), dev(deg), dev(adj if adj.size else np.zeros(1, np.int32))
    roots = np.nonzero(deg >= k - 1)[0].astype(np.int32)
    d_roots = dev(roots if roots.size else np.zeros(1, np.int32))
    out = ctypes.c_uint64()
    stream = torch.cuda.current_stream().cuda_stream
    rc = dm.lib().dm_count_cliques_noalloc(
        ctypes.c_void_p(d_row.data_ptr()), ctypes.c_void_p(d_deg.data_ptr()), ctypes.c_void_p(d_adj.data_ptr()),
        int(row.size), ctypes.c_void_p(d_roots.data_ptr()), int(roots.size),
        int(deg.max() if max_deg is None else max_deg), int(k), stream, ctypes.byref(out))
    torch.cuda.synchronize()
    return rc, out.value


@pytest.mark.parametrize("source", ["citeseer", "er2k"])
def test_noalloc_matches_dm_count_cliques_twice(dm, gpu, source):
    import torch

    from dumato_b200 import workloads

    g = dm.Graph.load_edgelist(GOLDEN / "citeseer.edgelist") if source == "citeseer" else workloads.make("er2k", 1)
    row, deg, adj = _id_dag(g)
    assert int(deg.max()) <= 256
    for k in (3, 4, 5):
        want, _ = dm.count_cliques(g, k)
        for _ in range(2):  # the fixed scratch keeps the last call's contents
            rc, got = _noalloc(dm, torch, row, deg, adj, k)
            assert rc == 0, dm.lib().dm_last_error()
            assert got == want


def test_noalloc_rejects_out_degree_beyond_limit(dm, gpu):
    import torch

    g = dm.Graph.load_edgelist(GOLDEN / "test.edgelist")
    row, deg, adj = _id_dag(g)
    rc, _ = _noalloc(dm, torch, row, deg, adj, 3, max_deg=300)
    assert rc == -1
    assert b"256" in dm.lib().dm_last_error()


def test_noalloc_leaves_device_memory_untouched(dm, gpu):
    """The device's free memory is the same before and after warmed-up calls: the entry
    point reserves nothing (a cudaMalloc would take at least one 2 MB page)."""
    import torch

    from dumato_b200 import workloads

    g = workloads.make("er2k", 2)
    row, deg, adj = _id_dag(g)
    want, _ = dm.count_cliques(g, 4)
    rc, got = _noalloc(dm, torch, row, deg, adj, 4)  # warm-up: module and kernels loaded
    assert rc == 0 and got == want
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    d_row, d_deg, d_adj = dev(row), dev(deg), dev(adj)
    roots = np.nonzero(deg >= 3)[0].astype(np.int32)
    d_roots = dev(roots)
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        out = ctypes.c_uint64()
        rc = dm.lib().dm_count_cliques_noalloc(
            ctypes.c_void_p(d_row.data_ptr()), ctypes.c_void_p(d_deg.data_ptr()), ctypes.c_void_p(d_adj.data_ptr()),
            int(row.size), ctypes.c_void_p(d_roots.data_ptr()), int(roots.size), int(deg.max()), 4, stream,
            ctypes.byref(out))
        assert rc == 0 and out.value == want
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after >= free_before


def test_noalloc_overflow_then_next_call_is_exact(dm, gpu):
    """An understated max_out_degree sends the largest root to a path that needs scratch the
    entry point does not hold: the call returns DM_EOVERFLOW, and the next correct call
    (whose set-up rebuilds the shared queue) matches dm_count_cliques."""
    import torch

    rng = np.random.default_rng(11)
    hub = np.zeros(100, np.int32)
    spokes = np.arange(1, 101, dtype=np.int32)
    a = rng.integers(1, 101, 1500).astype(np.int32)
    b = rng.integers(1, 101, 1500).astype(np.int32)
    g = dm.Graph.from_edges(np.concatenate([hub, a]), np.concatenate([spokes, b]))
    row, deg, adj = _id_dag(g)
    assert int(deg.max()) == 100
    want, _ = dm.count_cliques(g, 4)
    rc, _ = _noalloc(dm, torch, row, deg, adj, 4, max_deg=32)
    assert rc == -8, dm.lib().dm_last_error()
    for _ in range(2):
        rc, got = _noalloc(dm, torch, row, deg, adj, 4)
        assert rc == 0, dm.lib().dm_last_error()
        assert got == want
