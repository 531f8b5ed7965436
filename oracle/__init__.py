"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline / reference legs, never by the dumato_b200 package.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path
from typing import Optional

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
_lib: Optional[ctypes.CDLL] = None
_P = ctypes.c_void_p


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE), "liboracle.so"], check=True)
    return LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(LIB_PATH))
        sig = {
            "oracle_graph_from_pairs": (_P, [_P, _P, ctypes.c_int64]),
            "oracle_graph_load": (_P, [ctypes.c_char_p]),
            "oracle_graph_free": (None, [_P]),
            "oracle_graph_n": (ctypes.c_int32, [_P]),
            "oracle_graph_m": (ctypes.c_int64, [_P]),
            "oracle_graph_maxdeg": (ctypes.c_int32, [_P]),
            "oracle_clique_dfs": (ctypes.c_uint64, [_P, ctypes.c_int, ctypes.c_int]),
            "oracle_clique_dfs_range": (ctypes.c_uint64, [_P, ctypes.c_int, ctypes.c_int32, ctypes.c_int32, ctypes.c_int]),
            "oracle_clique_dfs_roots": (ctypes.c_uint64, [_P, ctypes.c_int, _P, ctypes.c_int64, ctypes.c_int]),
            "oracle_clique_brute": (ctypes.c_uint64, [_P, ctypes.c_int]),
            "oracle_clique_dag_bytes": (ctypes.c_uint64, [_P, ctypes.c_int, _P, ctypes.c_int]),
            "oracle_clique_dag_per_root": (None, [_P, ctypes.c_int, _P, ctypes.c_int]),
            "oracle_motifs": (ctypes.c_int, [_P, ctypes.c_int, _P, ctypes.c_int32, _P, ctypes.c_int]),
            "oracle_motifs_range": (ctypes.c_int, [_P, ctypes.c_int, _P, ctypes.c_int32, _P, ctypes.c_int32,
                                                   ctypes.c_int32, ctypes.c_int, _P]),
            "oracle_motifs_roots": (ctypes.c_int, [_P, ctypes.c_int, _P, ctypes.c_int32, _P, _P, ctypes.c_int64,
                                                   ctypes.c_int]),
            "oracle_motifs_brute": (ctypes.c_int, [_P, ctypes.c_int, _P, ctypes.c_int32, _P]),
            "oracle_graphlet4": (ctypes.c_int, [_P, _P, ctypes.c_int]),
            "oracle_near_cliques": (ctypes.c_uint64, [_P, ctypes.c_int, ctypes.c_int]),
            "oracle_near_cliques_brute": (ctypes.c_uint64, [_P, ctypes.c_int]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class OracleGraph:
    """The reference reader's view of a graph (set adjacency, self-loops kept)."""

    def __init__(self, h):
        if not h:
            raise ValueError("oracle could not read the graph")
        self.h = h

    @classmethod
    def from_pairs(cls, src, dst) -> "OracleGraph":
        s = np.ascontiguousarray(src, dtype=np.int32)
        d = np.ascontiguousarray(dst, dtype=np.int32)
        return cls(lib().oracle_graph_from_pairs(s.ctypes.data, d.ctypes.data, s.size))

    @classmethod
    def load(cls, path) -> "OracleGraph":
        return cls(lib().oracle_graph_load(str(path).encode()))

    @property
    def n(self) -> int:
        return lib().oracle_graph_n(self.h)

    @property
    def m(self) -> int:
        return lib().oracle_graph_m(self.h)

    @property
    def maxdeg(self) -> int:
        return lib().oracle_graph_maxdeg(self.h)

    def __del__(self):
        try:
            lib().oracle_graph_free(self.h)
        except Exception:
            pass


def clique_dfs(g: OracleGraph, k: int, threads: int = 0, root_begin: int = 0, root_end: int = -1) -> int:
    if root_end < 0:
        root_end = g.n
    return lib().oracle_clique_dfs_range(g.h, k, root_begin, root_end, threads)


def clique_dfs_roots(g: OracleGraph, k: int, roots, threads: int = 0) -> int:
    r = np.ascontiguousarray(roots, dtype=np.int32)
    return lib().oracle_clique_dfs_roots(g.h, k, r.ctypes.data, r.size, threads)


def clique_brute(g: OracleGraph, k: int) -> int:
    return lib().oracle_clique_brute(g.h, k)


def clique_dag_bytes(g: OracleGraph, k: int, threads: int = 0) -> tuple[int, int]:
    b = ctypes.c_uint64()
    c = lib().oracle_clique_dag_bytes(g.h, k, ctypes.byref(b), threads)
    return c, b.value


def clique_per_root(g: OracleGraph, k: int, threads: int = 0) -> np.ndarray:
    """k-cliques per root vertex (the clique's lowest (degree, id)-ranked vertex)."""
    out = np.zeros(g.n, np.uint64)
    lib().oracle_clique_dag_per_root(g.h, k, out.ctypes.data, threads)
    return out


def motifs(g: OracleGraph, k: int, q2c: np.ndarray, n_classes: int, threads: int = 0,
           root_begin: int = 0, root_end: int = -1, with_bytes: bool = False):
    q = np.ascontiguousarray(q2c, dtype=np.int32)
    hist = np.zeros(n_classes, np.uint64)
    if root_end < 0:
        root_end = g.n
    b = ctypes.c_uint64()
    rc = lib().oracle_motifs_range(g.h, k, q.ctypes.data, n_classes, hist.ctypes.data, root_begin, root_end, threads,
                                   ctypes.byref(b) if with_bytes else None)
    if rc != 0:
        raise RuntimeError(f"oracle_motifs failed ({rc})")
    return (hist, b.value) if with_bytes else hist


def motifs_roots(g: OracleGraph, k: int, q2c: np.ndarray, n_classes: int, roots, threads: int = 0) -> np.ndarray:
    q = np.ascontiguousarray(q2c, dtype=np.int32)
    r = np.ascontiguousarray(roots, dtype=np.int32)
    hist = np.zeros(n_classes, np.uint64)
    if lib().oracle_motifs_roots(g.h, k, q.ctypes.data, n_classes, hist.ctypes.data, r.ctypes.data, r.size, threads):
        raise RuntimeError("oracle_motifs_roots failed")
    return hist


def motifs_brute(g: OracleGraph, k: int, q2c: np.ndarray, n_classes: int) -> np.ndarray:
    q = np.ascontiguousarray(q2c, dtype=np.int32)
    hist = np.zeros(n_classes, np.uint64)
    lib().oracle_motifs_brute(g.h, k, q.ctypes.data, n_classes, hist.ctypes.data)
    return hist


GRAPHLET4_TYPES = ("path", "claw", "cycle", "paw", "diamond", "clique")


def graphlet4(g: OracleGraph, threads: int = 0) -> dict:
    """Connected induced 4-vertex subgraphs of the whole graph by type, from closed-form
    subgraph counts (no enumeration): {"path", "claw", "cycle", "paw", "diamond", "clique"}."""
    out = np.zeros(6, np.uint64)
    lib().oracle_graphlet4(g.h, out.ctypes.data, threads)
    return {t: int(c) for t, c in zip(GRAPHLET4_TYPES, out)}


def quick_edges(q: int, k: int) -> list[tuple[int, int]]:
    """Edges of the k-vertex pattern whose quick code is q: the edge (v0, v1) is implicit and
    vertex p >= 2 owns bits [(p-2)(p+1)/2, +p), bit j meaning the edge (v_j, v_p)
    (src/main/DuMatoGPU.cu:858,932)."""
    edges = [(0, 1)]
    for p in range(2, k):
        base = (p - 2) * (p + 1) // 2
        for j in range(p):
            if (q >> (base + j)) & 1:
                edges.append((j, p))
    return edges


def graphlet4_type(edges) -> Optional[str]:
    """Type of a 4-vertex pattern given by its edges (None when it is disconnected)."""
    deg = [0] * 4
    for a, b in edges:
        deg[a] += 1
        deg[b] += 1
    # connectivity by a small union-find
    par = list(range(4))

    def find(x):
        while par[x] != x:
            x = par[x]
        return x

    for a, b in edges:
        par[find(a)] = find(b)
    if len({find(x) for x in range(4)}) != 1:
        return None
    ds = tuple(sorted(deg))
    return {(1, 1, 2, 2): "path", (1, 1, 1, 3): "claw", (2, 2, 2, 2): "cycle", (1, 2, 2, 3): "paw",
            (2, 2, 3, 3): "diamond", (3, 3, 3, 3): "clique"}[ds]


def class_types4(q2c: np.ndarray, n_classes: int) -> list:
    """Graphlet type of every class of a k = 4 dictionary (None for disconnected classes)."""
    types = [None] * n_classes
    for q, c in enumerate(np.asarray(q2c)):
        if 0 <= c < n_classes and types[c] is None:
            types[c] = graphlet4_type(quick_edges(q, 4)) or "disconnected"
    return [None if t == "disconnected" else t for t in types]


def near_cliques(g: OracleGraph, n: int, threads: int = 0) -> int:
    """The reference's pattern-aware query q_n: non-induced copies of K_n minus one edge."""
    return lib().oracle_near_cliques(g.h, n, threads)


def near_cliques_brute(g: OracleGraph, n: int) -> int:
    """q_n by brute force over all n-subsets (tiny graphs, n <= 8)."""
    return lib().oracle_near_cliques_brute(g.h, n)
