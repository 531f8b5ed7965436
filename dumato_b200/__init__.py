"""dumato_b200 - B200-native warp-centric subgraph enumeration (k-clique and k-motif counting).

Python binding of the C ABI in include/dumato_b200.h (libdmb200.so, built in-tree by
``python -m dumato_b200.build``). The binding is a thin ctypes layer: every counting call
runs the library's sm_100a kernels; there is no CPU path, and a missing library or device
raises instead of falling back.

Reference correspondence (DuMato project root):
    Graph.load_edgelist   - Graph::Graph(const char*)            src/main/Graph.cpp:17-54
    count_cliques         - clique driver + outputAggregateCounter src/main/clique_PA.cu:34-130
    count_motifs          - motif driver + outputAggregatePattern  src/main/motifs_DM_WCLB.cu:38-140
    Dictionary.load_csv   - QuickMapping::QuickMapping(int k)      src/main/QuickMapping.cpp:5-45
    Options(threads, block_size, donations_per_warp, threshold)
                          - argv[3..6] of both drivers             src/main/clique_PA.cu:54-63
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field
from pathlib import Path
from typing import Optional, Sequence

import numpy as np

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libdmb200.so"

DM_OK = 0
STATUS_NAMES = {
    -1: "DM_EINVAL", -2: "DM_EIO", -3: "DM_EFORMAT", -4: "DM_ENOMEM", -5: "DM_ENODEVICE",
    -6: "DM_ECUDA", -7: "DM_ETIMEOUT", -8: "DM_EOVERFLOW", -9: "DM_EINTERNAL",
}

GEN_ER, GEN_CHUNG_LU, GEN_RMAT = 0, 1, 2
MODE_AUTO, MODE_LIST, MODE_BITMAP, MODE_REBUILD = 0, 1, 2, 3
STAGE_AUTO, STAGE_LOADS, STAGE_TMA = 0, 1, 2
FLAG_L2_PERSIST = 1
QUERY_CLIQUE, QUERY_MOTIF = 0, 1
AUTOTUNE_MODEL, AUTOTUNE_MEASURE = 0, 1
SCHED_PLAIN, SCHED_LEARNED, SCHED_ID = 0, 1, 2


class DMError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class _GenParams(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("n", ctypes.c_int32), ("m", ctypes.c_int64),
                ("gamma", ctypes.c_double), ("dmax", ctypes.c_double), ("a", ctypes.c_double),
                ("b", ctypes.c_double), ("c", ctypes.c_double), ("seed", ctypes.c_uint64)]


class _GraphInfo(ctypes.Structure):
    _fields_ = [("n_vertices", ctypes.c_int32), ("n_edges", ctypes.c_int64), ("max_degree", ctypes.c_int32),
                ("max_out_degree", ctypes.c_int32), ("n_self_loops", ctypes.c_int64),
                ("n_input_pairs", ctypes.c_int64)]


class _Report(ctypes.Structure):
    _fields_ = [("elapsed_ms", ctypes.c_double), ("warps", ctypes.c_int32), ("hungry_warps", ctypes.c_int32),
                ("roots_claimed", ctypes.c_int64), ("roots_total", ctypes.c_int64), ("pending", ctypes.c_int64),
                ("donations", ctypes.c_uint64), ("progress", ctypes.c_uint64)]


_REPORT_FN = ctypes.CFUNCTYPE(None, ctypes.POINTER(_Report), ctypes.c_void_p)


class _Opts(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_int32), ("device", ctypes.c_int32), ("stream", ctypes.c_uint64),
                ("threads", ctypes.c_int32), ("block_size", ctypes.c_int32),
                ("donations_per_warp", ctypes.c_int32), ("threshold", ctypes.c_int32),
                ("vwarp", ctypes.c_int32), ("mode", ctypes.c_int32), ("scheduler", ctypes.c_int32),
                ("rank", ctypes.c_int32), ("world_size", ctypes.c_int32), ("timeout_ms", ctypes.c_int32),
                ("predictor", ctypes.c_void_p), ("subtree_counts", ctypes.c_void_p),
                ("test_flags", ctypes.c_int32), ("staging", ctypes.c_int32), ("flags", ctypes.c_int32),
                ("report_ms", ctypes.c_int32), ("report", _REPORT_FN), ("report_user", ctypes.c_void_p)]


class _Stats(ctypes.Structure):
    _fields_ = [("kernel_ms", ctypes.c_double), ("prep_ms", ctypes.c_double), ("tasks", ctypes.c_uint64),
                ("donations", ctypes.c_uint64), ("idle_polls", ctypes.c_uint64), ("nodes", ctypes.c_uint64),
                ("mode_used", ctypes.c_int32), ("vwarp_used", ctypes.c_int32), ("grid", ctypes.c_int32),
                ("block", ctypes.c_int32), ("kernel_launches", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("idle_warp_fraction", ctypes.c_double), ("max_task_ms", ctypes.c_double),
                ("max_task_root", ctypes.c_int32), ("prefix_donations", ctypes.c_int32)]


class _Query(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("k", ctypes.c_int32), ("graph", ctypes.c_void_p),
                ("dict", ctypes.c_void_p), ("vwarp", ctypes.c_int32), ("threshold", ctypes.c_int32),
                ("mode", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class _QueryTuning(ctypes.Structure):
    _fields_ = [("vwarp", ctypes.c_int32), ("threshold", ctypes.c_int32), ("mode", ctypes.c_int32),
                ("n_results", ctypes.c_int32), ("result_offset", ctypes.c_int64), ("tune_ms", ctypes.c_double),
                ("est_cost", ctypes.c_double)]


_P = ctypes.c_void_p
_SIGNATURES = {
    "dm_abi_version": (ctypes.c_int, []),
    "dm_last_error": (ctypes.c_char_p, []),
    "dm_device_count": (ctypes.c_int, []),
    "dm_graph_load_edgelist": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(_P)]),
    "dm_graph_load_edgelist_device": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(_Opts), ctypes.POINTER(_P),
                                                     ctypes.POINTER(ctypes.c_double)]),
    "dm_graph_from_edges": (ctypes.c_int, [_P, _P, ctypes.c_int64, ctypes.c_int32, ctypes.POINTER(_P)]),
    "dm_graph_generate": (ctypes.c_int, [ctypes.POINTER(_GenParams), ctypes.POINTER(_P)]),
    "dm_graph_info_get": (ctypes.c_int, [_P, ctypes.POINTER(_GraphInfo)]),
    "dm_graph_edges": (ctypes.c_int, [_P, _P, _P]),
    "dm_graph_csr": (ctypes.c_int, [_P, _P, _P]),
    "dm_graph_write_edgelist": (ctypes.c_int, [_P, ctypes.c_char_p]),
    "dm_graph_free": (None, [_P]),
    "dm_graph_release_device": (ctypes.c_int, [_P]),
    "dm_dictionary_generate": (ctypes.c_int, [ctypes.c_int32, ctypes.POINTER(_P)]),
    "dm_dictionary_load_csv": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(_P)]),
    "dm_dictionary_write_csv": (ctypes.c_int, [_P, ctypes.c_char_p]),
    "dm_dictionary_shape": (ctypes.c_int, [_P, _P, _P, _P]),
    "dm_dictionary_tables": (ctypes.c_int, [_P, _P, _P]),
    "dm_dictionary_connected": (ctypes.c_int, [_P, _P]),
    "dm_dictionary_free": (None, [_P]),
    "dm_clique_work_model": (ctypes.c_int, [_P, ctypes.c_int32, _P, _P]),
    "dm_motif_work_model": (ctypes.c_int, [_P, ctypes.c_int32, _P, _P]),
    "dm_plan_roots": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(_Opts), _P, _P, ctypes.c_int64,
                                     ctypes.POINTER(ctypes.c_int64)]),
    "dm_predictor_create": (ctypes.c_int, [ctypes.c_uint64, ctypes.POINTER(_P)]),
    "dm_predictor_free": (None, [_P]),
    "dm_predictor_num_params": (ctypes.c_int, []),
    "dm_predictor_get_params": (ctypes.c_int, [_P, _P]),
    "dm_predictor_set_params": (ctypes.c_int, [_P, _P]),
    "dm_predictor_features": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32, _P]),
    "dm_predictor_predict": (ctypes.c_int, [_P, _P, ctypes.c_int64, _P]),
    "dm_predictor_gradients": (ctypes.c_int, [_P, _P, _P, ctypes.c_int64, _P, _P]),
    "dm_predictor_train": (ctypes.c_int, [_P, _P, _P, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32,
                                          ctypes.c_float, _P]),
    "dm_count_cliques_noalloc": (ctypes.c_int, [_P, _P, _P, ctypes.c_int32, _P, ctypes.c_int32, ctypes.c_int32,
                                                ctypes.c_int32, ctypes.c_uint64, _P]),
    "dm_count_cliques": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.POINTER(_Opts), _P, ctypes.POINTER(_Stats)]),
    "dm_count_cliques_upto": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.POINTER(_Opts), _P, ctypes.POINTER(_Stats)]),
    "dm_count_near_cliques": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.POINTER(_Opts), _P, ctypes.POINTER(_Stats)]),
    "dm_count_motifs": (ctypes.c_int, [_P, ctypes.c_int32, _P, ctypes.POINTER(_Opts), _P, ctypes.POINTER(_Stats)]),
    "dm_batch_create": (ctypes.c_int, [ctypes.POINTER(_Query), ctypes.c_int32, ctypes.POINTER(_Opts), ctypes.c_int32,
                                       ctypes.POINTER(_P)]),
    "dm_batch_num_results": (ctypes.c_int64, [_P]),
    "dm_batch_tuning": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.POINTER(_QueryTuning)]),
    "dm_batch_run": (ctypes.c_int, [_P, _P, ctypes.c_int64, ctypes.POINTER(_Stats)]),
    "dm_batch_free": (None, [_P]),
}

_lib: Optional[ctypes.CDLL] = None


def lib() -> ctypes.CDLL:
    """Loads libdmb200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: run `python -m dumato_b200.build` first")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_symbols() -> list[str]:
    return list(_SIGNATURES)


def _check(rc: int) -> None:
    if rc != DM_OK:
        msg = lib().dm_last_error()
        raise DMError(rc, msg.decode() if msg else "")


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


def device_count() -> int:
    return lib().dm_device_count()


@dataclass
class GraphInfo:
    n_vertices: int
    n_edges: int
    max_degree: int
    max_out_degree: int
    n_self_loops: int
    n_input_pairs: int


class Graph:
    """An undirected, unlabeled graph (ids in [0, V-1], duplicates merged, self-loops dropped)."""

    def __init__(self, handle: ctypes.c_void_p):
        self._h = handle

    @classmethod
    def load_edgelist(cls, path: str | os.PathLike) -> "Graph":
        h = _P()
        _check(lib().dm_graph_load_edgelist(str(path).encode(), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def load_edgelist_device(cls, path: str | os.PathLike, opts: "Optional[Options]" = None) -> "tuple[Graph, float]":
        """The edgelist reader on the GPU (parse, dedup, symmetrise, orient on the device);
        returns the graph and the device time in ms."""
        h = _P()
        ms = ctypes.c_double()
        o = (opts or Options()).to_c()
        _check(lib().dm_graph_load_edgelist_device(str(path).encode(), ctypes.byref(o), ctypes.byref(h),
                                                   ctypes.byref(ms)))
        return cls(h), ms.value

    @classmethod
    def from_edges(cls, src: Sequence[int], dst: Sequence[int], n_vertices: int = 0) -> "Graph":
        s = np.ascontiguousarray(src, dtype=np.int32)
        d = np.ascontiguousarray(dst, dtype=np.int32)
        if s.shape != d.shape:
            raise ValueError("src and dst differ in length")
        h = _P()
        _check(lib().dm_graph_from_edges(_ptr(s), _ptr(d), s.size, int(n_vertices), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def generate(cls, kind: int, n: int, m: int, seed: int, gamma: float = 2.1, dmax: float = 500.0,
                 a: float = 0.57, b: float = 0.19, c: float = 0.19) -> "Graph":
        p = _GenParams(kind=kind, n=n, m=m, gamma=gamma, dmax=dmax, a=a, b=b, c=c, seed=seed)
        h = _P()
        _check(lib().dm_graph_generate(ctypes.byref(p), ctypes.byref(h)))
        return cls(h)

    @property
    def handle(self) -> ctypes.c_void_p:
        if self._h is None:
            raise ValueError("graph was freed")
        return self._h

    def info(self) -> GraphInfo:
        i = _GraphInfo()
        _check(lib().dm_graph_info_get(self.handle, ctypes.byref(i)))
        return GraphInfo(i.n_vertices, i.n_edges, i.max_degree, i.max_out_degree, i.n_self_loops, i.n_input_pairs)

    def edges(self) -> tuple[np.ndarray, np.ndarray]:
        m = self.info().n_edges
        u = np.empty(m, np.int32)
        v = np.empty(m, np.int32)
        _check(lib().dm_graph_edges(self.handle, _ptr(u), _ptr(v)))
        return u, v

    def csr(self) -> tuple[np.ndarray, np.ndarray]:
        inf = self.info()
        off = np.empty(inf.n_vertices + 1, np.int64)
        adj = np.empty(2 * inf.n_edges, np.int32)
        _check(lib().dm_graph_csr(self.handle, _ptr(off), _ptr(adj)))
        return off, adj

    def write_edgelist(self, path: str | os.PathLike) -> None:
        _check(lib().dm_graph_write_edgelist(self.handle, str(path).encode()))

    def release_device(self) -> None:
        _check(lib().dm_graph_release_device(self.handle))

    def free(self) -> None:
        if self._h is not None:
            lib().dm_graph_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Dictionary:
    """quick code -> canonical class table for k-vertex motifs (k in 3..7)."""

    def __init__(self, handle: ctypes.c_void_p):
        self._h = handle

    @classmethod
    def generate(cls, k: int) -> "Dictionary":
        h = _P()
        _check(lib().dm_dictionary_generate(int(k), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def load_csv(cls, path: str | os.PathLike) -> "Dictionary":
        h = _P()
        _check(lib().dm_dictionary_load_csv(str(path).encode(), ctypes.byref(h)))
        return cls(h)

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def shape(self) -> tuple[int, int, int]:
        k = ctypes.c_int32()
        nq = ctypes.c_int64()
        nc = ctypes.c_int32()
        _check(lib().dm_dictionary_shape(self._h, ctypes.byref(k), ctypes.byref(nq), ctypes.byref(nc)))
        return k.value, nq.value, nc.value

    @property
    def k(self) -> int:
        return self.shape()[0]

    @property
    def n_classes(self) -> int:
        return self.shape()[2]

    def tables(self) -> tuple[np.ndarray, np.ndarray]:
        _, nq, nc = self.shape()
        q2c = np.empty(nq, np.int32)
        code = np.empty(nc, np.uint64)
        _check(lib().dm_dictionary_tables(self._h, _ptr(q2c), _ptr(code)))
        return q2c, code

    def connected(self) -> np.ndarray:
        nc = self.n_classes
        out = np.empty(nc, np.uint8)
        _check(lib().dm_dictionary_connected(self._h, _ptr(out)))
        return out.astype(bool)

    def write_csv(self, path: str | os.PathLike) -> None:
        _check(lib().dm_dictionary_write_csv(self._h, str(path).encode()))

    def __del__(self):
        try:
            if self._h is not None:
                lib().dm_dictionary_free(self._h)
                self._h = None
        except Exception:
            pass


class Predictor:
    """Learned work predictor: an 8 -> 32 -> 32 -> 1 FP32 MLP over root-task features,
    trained and evaluated by the library's CUDA kernels (log(1 + subtree size) target)."""

    N_FEATURES = 8

    def __init__(self, seed: int = 0):
        h = _P()
        _check(lib().dm_predictor_create(int(seed), ctypes.byref(h)))
        self._h = h

    @property
    def handle(self) -> int:
        return self._h.value

    @property
    def n_params(self) -> int:
        return lib().dm_predictor_num_params()

    def get_params(self) -> np.ndarray:
        p = np.empty(self.n_params, np.float32)
        _check(lib().dm_predictor_get_params(self._h, _ptr(p)))
        return p

    def set_params(self, params: np.ndarray) -> None:
        p = np.ascontiguousarray(params, dtype=np.float32)
        if p.size != self.n_params:
            raise ValueError(f"expected {self.n_params} parameters")
        _check(lib().dm_predictor_set_params(self._h, _ptr(p)))

    @staticmethod
    def features(g: "Graph", k: int, clique: bool = True) -> np.ndarray:
        X = np.empty((g.info().n_vertices, Predictor.N_FEATURES), np.float32)
        _check(lib().dm_predictor_features(g.handle, int(k), 1 if clique else 0, _ptr(X)))
        return X

    def predict(self, X: np.ndarray) -> np.ndarray:
        X = np.ascontiguousarray(X, dtype=np.float32)
        y = np.empty(X.shape[0], np.float32)
        _check(lib().dm_predictor_predict(self._h, _ptr(X), X.shape[0], _ptr(y)))
        return y

    def gradients(self, X: np.ndarray, T: np.ndarray) -> tuple[np.ndarray, float]:
        X = np.ascontiguousarray(X, dtype=np.float32)
        T = np.ascontiguousarray(T, dtype=np.float32)
        g = np.empty(self.n_params, np.float32)
        loss = ctypes.c_float()
        _check(lib().dm_predictor_gradients(self._h, _ptr(X), _ptr(T), X.shape[0], _ptr(g), ctypes.byref(loss)))
        return g, loss.value

    def train(self, X: np.ndarray, T: np.ndarray, epochs: int = 60, batch: int = 256, lr: float = 3e-3) -> float:
        X = np.ascontiguousarray(X, dtype=np.float32)
        T = np.ascontiguousarray(T, dtype=np.float32)
        loss = ctypes.c_float()
        _check(lib().dm_predictor_train(self._h, _ptr(X), _ptr(T), X.shape[0], int(epochs), int(batch),
                                        float(lr), ctypes.byref(loss)))
        return loss.value

    def __del__(self):
        try:
            if self._h:
                lib().dm_predictor_free(self._h)
                self._h = None
        except Exception:
            pass


def subtree_log(g: "Graph", k: int, clique: bool = True, dictionary: "Optional[Dictionary]" = None):
    """Per-root subtree sizes logged by the plain engine: (features[n, 8], log1p(size)[n],
    roots mask). Roots that start no task are masked out."""
    n = g.info().n_vertices
    per = np.zeros(n, np.uint64)
    opts = Options(subtree_counts=per)
    if clique:
        count_cliques(g, k, opts)
    else:
        count_motifs(g, k, dictionary, opts)
    X = Predictor.features(g, k, clique)
    if clique:
        mask = np.expm1(X[:, 5]).round() >= k - 1        # DAG out-degree >= k-1
    else:
        mask = np.expm1(X[:, 2]).round() >= 1            # a neighbour above v
    return X, np.log1p(per.astype(np.float64)).astype(np.float32), mask


@dataclass
class Options:
    """Engine options; threads/block_size/donations_per_warp/threshold are the reference's
    positional CLI arguments 3..6 (src/main/clique_PA.cu:54-63)."""
    device: int = -1
    stream: int = 0
    threads: int = 0
    block_size: int = 0
    donations_per_warp: int = 0
    threshold: int = 0
    vwarp: int = 0
    mode: int = MODE_AUTO
    scheduler: int = SCHED_PLAIN
    rank: int = 0
    world_size: int = 1
    timeout_ms: int = 0
    predictor: Optional[int] = None
    subtree_counts: Optional[np.ndarray] = None   # uint64[n_vertices], filled per root
    test_flags: int = 0
    staging: int = STAGE_AUTO
    flags: int = 0
    report: Optional[object] = None   # callable(dict), called every report_ms while a kernel runs
    report_ms: int = 0

    def __setattr__(self, name, value):
        object.__setattr__(self, name, value)
        if name != "_c_cache":
            object.__setattr__(self, "_c_cache", None)  # any change rebuilds the C struct

    def to_c(self) -> _Opts:
        c = self.__dict__.get("_c_cache")
        if c is not None:
            return c
        c = self._build_c()
        object.__setattr__(self, "_c_cache", c)
        return c

    def _build_c(self) -> _Opts:
        st = None
        if self.subtree_counts is not None:
            if self.subtree_counts.dtype != np.uint64 or not self.subtree_counts.flags.c_contiguous:
                raise ValueError("subtree_counts must be a contiguous uint64 array")
            st = self.subtree_counts.ctypes.data
        return _Opts(struct_size=ctypes.sizeof(_Opts), device=self.device, stream=self.stream,
                     threads=self.threads, block_size=self.block_size,
                     donations_per_warp=self.donations_per_warp, threshold=self.threshold, vwarp=self.vwarp,
                     mode=self.mode, scheduler=self.scheduler, rank=self.rank, world_size=self.world_size,
                     timeout_ms=self.timeout_ms, predictor=self.predictor, subtree_counts=st,
                     test_flags=self.test_flags, staging=self.staging, flags=self.flags,
                     report_ms=self.report_ms if self.report else 0, report=self._report_fn(),
                     report_user=None)

    def _report_fn(self):
        if self.report is None:
            return _REPORT_FN()
        user = self.report

        def cb(sample, _user):
            r = sample.contents
            user({f: getattr(r, f) for f, _ in _Report._fields_})

        fn = _REPORT_FN(cb)
        # the C function pointer must outlive the call: keep it with the options
        object.__setattr__(self, "_report_keep", fn)
        return fn


@dataclass
class Stats:
    kernel_ms: float = 0.0
    prep_ms: float = 0.0
    tasks: int = 0
    donations: int = 0
    idle_polls: int = 0
    nodes: int = 0
    mode_used: int = 0
    vwarp_used: int = 0
    grid: int = 0
    block: int = 0
    kernel_launches: int = 0
    idle_warp_fraction: float = 0.0
    max_task_ms: float = 0.0
    max_task_root: int = -1
    prefix_donations: int = 0

    @classmethod
    def from_c(cls, s: _Stats) -> "Stats":
        return cls(s.kernel_ms, s.prep_ms, s.tasks, s.donations, s.idle_polls, s.nodes, s.mode_used,
                   s.vwarp_used, s.grid, s.block, s.kernel_launches, s.idle_warp_fraction, s.max_task_ms,
                   s.max_task_root, s.prefix_donations)


def motif_work_model(g: Graph, k: int) -> tuple[int, int]:
    """(DFS prefixes, algorithmic bytes) of k-motif counting on g: the byte model behind the
    motif roofline figures (host-side accounting, not a counting path)."""
    n = ctypes.c_uint64()
    b = ctypes.c_uint64()
    _check(lib().dm_motif_work_model(g.handle, int(k), ctypes.byref(n), ctypes.byref(b)))
    return n.value, b.value


def clique_work_model(g: Graph, k: int) -> tuple[int, int]:
    """(DFS nodes, algorithmic bytes) of k-clique counting on g's degree-ordered DAG; the
    byte model behind the roofline figures (host-side accounting, not a counting path)."""
    n = ctypes.c_uint64()
    b = ctypes.c_uint64()
    _check(lib().dm_clique_work_model(g.handle, int(k), ctypes.byref(n), ctypes.byref(b)))
    return n.value, b.value


TEST_STALL_AT_EXIT = 1
TEST_EAGER_DONATION = 2


def plan_roots(g: Graph, k: int, clique: bool = True, opts: Optional[Options] = None) -> tuple[np.ndarray, np.ndarray]:
    """The ordered root tasks (original ids, part words) this shard would run (host only)."""
    o = (opts or Options()).to_c()
    n = ctypes.c_int64()
    _check(lib().dm_plan_roots(g.handle, int(k), 1 if clique else 0, ctypes.byref(o), None, None, 0, ctypes.byref(n)))
    roots = np.empty(n.value, np.int32)
    parts = np.empty(n.value, np.int32)
    _check(lib().dm_plan_roots(g.handle, int(k), 1 if clique else 0, ctypes.byref(o), _ptr(roots), _ptr(parts),
                               n.value, ctypes.byref(n)))
    return roots, parts


def count_cliques(g: Graph, k: int, opts: Optional[Options] = None) -> tuple[int, Stats]:
    """Number of k-cliques of g (exact uint64), computed on the GPU."""
    o = (opts or Options()).to_c()
    out = ctypes.c_uint64()
    st = _Stats()
    _check(lib().dm_count_cliques(g.handle, int(k), ctypes.byref(o), ctypes.byref(out), ctypes.byref(st)))
    return out.value, Stats.from_c(st)


def count_cliques_upto(g: Graph, kmax: int, opts: Optional[Options] = None) -> tuple[dict, Stats]:
    """Clique counts of every size 3..kmax from one traversal: ({k: count}, stats)."""
    o = (opts or Options()).to_c()
    out = np.zeros(kmax - 2, np.uint64)
    st = _Stats()
    _check(lib().dm_count_cliques_upto(g.handle, int(kmax), ctypes.byref(o), _ptr(out), ctypes.byref(st)))
    return {k: int(out[k - 3]) for k in range(3, kmax + 1)}, Stats.from_c(st)


def count_near_cliques(g: Graph, n: int, opts: Optional[Options] = None) -> tuple[int, Stats]:
    """The reference's pattern-aware query q_n (n = 4..13): non-induced copies of K_n minus
    one edge (src/main/q4_PA.cu .. q13_PA.cu)."""
    o = (opts or Options()).to_c()
    out = ctypes.c_uint64()
    st = _Stats()
    _check(lib().dm_count_near_cliques(g.handle, int(n), ctypes.byref(o), ctypes.byref(out), ctypes.byref(st)))
    return out.value, Stats.from_c(st)


def count_motifs(g: Graph, k: int, dictionary: Optional[Dictionary] = None,
                 opts: Optional[Options] = None) -> tuple[np.ndarray, Stats]:
    """Connected induced k-subgraph counts per dictionary class (uint64[n_classes])."""
    d = dictionary or Dictionary.generate(k)
    if d.k != k:
        raise ValueError(f"dictionary is for k={d.k}, asked for k={k}")
    o = (opts or Options()).to_c()
    out = np.zeros(d.n_classes, np.uint64)
    st = _Stats()
    _check(lib().dm_count_motifs(g.handle, int(k), d.handle, ctypes.byref(o), _ptr(out), ctypes.byref(st)))
    return out, Stats.from_c(st)


@dataclass
class Query:
    """One (graph, query) pair of a batch: k-cliques (kind QUERY_CLIQUE, k in 2..6) or motif
    class counts (QUERY_MOTIF, k in 3..5). vwarp / threshold / mode left at 0 / -1 / MODE_AUTO
    are chosen by the autotuner."""
    kind: int
    k: int
    graph: Graph
    dictionary: Optional[Dictionary] = None
    vwarp: int = 0
    threshold: int = -1
    mode: int = MODE_AUTO


@dataclass
class QueryTuning:
    vwarp: int
    threshold: int
    mode: int
    n_results: int
    result_offset: int
    tune_ms: float
    est_cost: float


class Batch:
    """Many (graph, query) pairs counted by one persistent, CUDA-graph-captured launch.

    Built once (union graph upload, autotuning, capture); run() replays the launch and returns
    one result per query: an int (k-cliques) or a uint64 array of class counts (motifs)."""

    def __init__(self, queries: Sequence[Query], autotune: int = AUTOTUNE_MODEL, opts: Optional[Options] = None):
        self._queries = list(queries)
        arr = (_Query * max(1, len(self._queries)))()
        for i, q in enumerate(self._queries):
            if q.kind == QUERY_MOTIF and q.dictionary is None:
                raise ValueError(f"query {i}: a motif query needs its k-vertex dictionary")
            arr[i] = _Query(kind=q.kind, k=q.k, graph=q.graph.handle,
                            dict=q.dictionary.handle if q.dictionary is not None else None,
                            vwarp=q.vwarp, threshold=q.threshold, mode=q.mode)
        o = (opts or Options()).to_c()
        h = _P()
        _check(lib().dm_batch_create(arr, len(self._queries), ctypes.byref(o), int(autotune), ctypes.byref(h)))
        self._h = h
        self.n_results = int(lib().dm_batch_num_results(h))

    def tuning(self, i: int) -> QueryTuning:
        t = _QueryTuning()
        _check(lib().dm_batch_tuning(self._h, int(i), ctypes.byref(t)))
        return QueryTuning(t.vwarp, t.threshold, t.mode, t.n_results, t.result_offset, t.tune_ms, t.est_cost)

    def run_raw(self, out: Optional[np.ndarray] = None) -> tuple[np.ndarray, Stats]:
        """All result words (uint64[n_results]) of one replay, and its stats."""
        if out is None:
            out = np.zeros(max(1, self.n_results), np.uint64)
        st = _Stats()
        _check(lib().dm_batch_run(self._h, _ptr(out), out.size, ctypes.byref(st)))
        return out, Stats.from_c(st)

    def run(self) -> tuple[list, Stats]:
        raw, st = self.run_raw()
        res = []
        for i, q in enumerate(self._queries):
            t = self.tuning(i)
            part = raw[t.result_offset:t.result_offset + t.n_results]
            res.append(int(part[0]) if q.kind == QUERY_CLIQUE else part.copy())
        return res, st

    def close(self) -> None:
        if getattr(self, "_h", None) is not None:
            lib().dm_batch_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
