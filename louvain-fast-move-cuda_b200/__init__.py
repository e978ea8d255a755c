"""B200 Louvain engine: Python mirror of the reference's host API over the C ABI.

The reference exposes ``ModularityAlgorithms::Louvain(GraphHost&, MODE)`` returning a
``Community`` (modularityAlgorithms.h:8-10, community.h:15-26). This package keeps those
names and argument meanings and calls the engine's shared library
(``liblouvain_b200.so``, C ABI declared in include/louvain_b200.h) through ctypes:

    lv = importlib.import_module("louvain-fast-move-cuda_b200")
    g = lv.GraphHost("graph.edge", False, 0)          # graphHost.cuh:17
    C = lv.ModularityAlgorithms.Louvain(g, lv.MODE.SORT)
    C.best_communities, C.n_of_best_communities, C.modularity

There is no CPU fallback: if the library is missing or no CUDA device is present the calls
raise ``LouvainError``.
"""
from __future__ import annotations

import ctypes
import enum
import os
import weakref
from typing import Optional, Sequence

import numpy as np

from . import graphs as graphs  # noqa: F401
from .graphs import CSRGraph

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liblouvain_b200.so")
_lib = None


class LouvainError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{message} (status {status})")
        self.status = status


class MODE(enum.IntEnum):
    """constants.h:13"""
    HASH = 0
    SORT = 1
    ADAPTIVE_SPEED = 2
    ADAPTIVE_MEMORY = 3


MEM_HOST, MEM_DEVICE = 0, 1
WEIGHTS_AUTO, WEIGHTS_INTEGER, WEIGHTS_FLOAT = 0, 1, 2


class Config(ctypes.Structure):
    _fields_ = [
        ("mode", ctypes.c_int32), ("fast_first", ctypes.c_int32),
        ("max_iterations", ctypes.c_int32), ("max_levels", ctypes.c_int32),
        ("threshold", ctypes.c_double), ("chunk_edges", ctypes.c_int64),
        ("weight_mode", ctypes.c_int32), ("validate", ctypes.c_int32),
        ("use_graphs", ctypes.c_int32), ("refine", ctypes.c_int32),
        ("refine_passes", ctypes.c_int32), ("reserved_i", ctypes.c_int32 * 5),
        ("bin_max_degree", ctypes.c_int32 * 8), ("refine_tolerance", ctypes.c_double),
        ("reserved_d", ctypes.c_double * 3),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("modularity", ctypes.c_double), ("n", ctypes.c_int64), ("m", ctypes.c_int64),
        ("levels", ctypes.c_int32), ("iterations", ctypes.c_int32),
        ("n_communities", ctypes.c_int32), ("reserved0", ctypes.c_int32),
        ("ms_total", ctypes.c_float), ("ms_window", ctypes.c_float),
        ("ms_optimization", ctypes.c_float), ("ms_aggregation", ctypes.c_float),
        ("ms_first_optimization", ctypes.c_float), ("ms_first_aggregation", ctypes.c_float),
        ("bytes_optimization", ctypes.c_double), ("ms_optimization_kernels", ctypes.c_float),
        ("reserved1", ctypes.c_int32), ("kernel_launches", ctypes.c_int64),
        ("active_entries", ctypes.c_int64), ("active_vertices", ctypes.c_int64),
        ("graph_launches", ctypes.c_int64), ("refine_passes", ctypes.c_int64),
        ("reserved", ctypes.c_int64 * 1),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if not k.startswith("reserved")}


class CommunityInfo(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int64), ("E", ctypes.c_int64), ("n0", ctypes.c_int64),
        ("level", ctypes.c_int32), ("iteration", ctypes.c_int32),
        ("modularity", ctypes.c_double), ("internal", ctypes.c_double),
        ("sum_a2", ctypes.c_double), ("total_weight", ctypes.c_double),
        ("n_best", ctypes.c_int64), ("weights_integer", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


TRACE_DTYPE = np.dtype([
    ("level", np.int32), ("iteration", np.int32), ("n_moved", np.int32), ("reserved", np.int32),
    ("internal", np.float64), ("sum_a2", np.float64), ("modularity", np.float64),
    ("delta", np.float64),
])

# Every entry point the header declares; tests check that the library exports all of them.
EXPORTS = (
    "lv_config_default", "lv_create", "lv_destroy", "lv_last_error", "lv_status_string",
    "lv_abi_version", "lv_run_csr", "lv_run_batch", "lv_autotune", "lv_community_create",
    "lv_community_destroy", "lv_community_resume", "lv_optimization_step", "lv_optimization_run",
    "lv_aggregation_run", "lv_louvain", "lv_community_info_get", "lv_community_get_partition",
    "lv_community_get_best", "lv_community_get_graph", "lv_community_get_trace",
    "lv_server_create", "lv_server_destroy", "lv_server_submit", "lv_server_submit_borrowed",
    "lv_server_progress", "lv_server_poll", "lv_server_drain",
    "lv_ingest_edge_list", "lv_ingest_info", "lv_ingest_copy_csr", "lv_ingest_run", "lv_ingest_destroy",
)


def load_library(path: Optional[str] = None):
    """Load liblouvain_b200.so (built by ``make -C louvain-fast-move-cuda_b200/csrc``)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise LouvainError(-1, f"engine library not built: {p} is missing "
                               "(run `make -C louvain-fast-move-cuda_b200/csrc` or __graft_entry__.build())")
    L = ctypes.CDLL(p)
    vp, i32, i64, dbl = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double
    P = ctypes.POINTER
    sig = {
        "lv_config_default": (None, [P(Config)]),
        "lv_create": (i32, [i32, P(Config), P(vp)]),
        "lv_destroy": (i32, [vp]),
        "lv_last_error": (ctypes.c_char_p, [vp]),
        "lv_status_string": (ctypes.c_char_p, [i32]),
        "lv_abi_version": (i32, []),
        "lv_run_csr": (i32, [vp, i64, vp, vp, vp, i32, vp, i32, P(dbl), P(Stats)]),
        "lv_run_batch": (i32, [vp, i32, vp, vp, vp, vp, i32, vp, i32, vp, vp, P(Stats)]),
        "lv_autotune": (i32, [vp, i32, vp, vp, vp, vp, i32, i32, P(Config), P(dbl)]),
        "lv_community_create": (i32, [vp, i64, vp, vp, vp, i32, P(vp)]),
        "lv_community_destroy": (i32, [vp]),
        "lv_community_resume": (i32, [vp, i64, vp, i32, i32, i64, vp, vp, vp, i32, P(vp)]),
        "lv_optimization_step": (i32, [vp, P(dbl), P(i64)]),
        "lv_optimization_run": (i32, [vp, P(i32)]),
        "lv_aggregation_run": (i32, [vp, i32]),
        "lv_louvain": (i32, [vp, P(Stats)]),
        "lv_community_info_get": (i32, [vp, P(CommunityInfo)]),
        "lv_community_get_partition": (i32, [vp, vp, vp]),
        "lv_community_get_best": (i32, [vp, vp]),
        "lv_community_get_graph": (i32, [vp, vp, vp, vp, vp]),
        "lv_community_get_trace": (i32, [vp, vp, i32, P(i32)]),
        "lv_server_create": (i32, [vp, i64, i32, P(vp)]),
        "lv_server_destroy": (i32, [vp]),
        "lv_server_submit": (i32, [vp, i64, vp, vp, vp, P(i64)]),
        "lv_server_submit_borrowed": (i32, [vp, i64, vp, vp, vp, P(i64)]),
        "lv_server_progress": (i32, [vp, P(i64), P(i64), P(i64)]),
        "lv_server_poll": (i32, [vp, i64, vp, P(dbl), P(dbl), P(i32)]),
        "lv_server_drain": (i32, [vp]),
        "lv_ingest_edge_list": (i32, [vp, vp, i64, i32, i32, P(vp)]),
        "lv_ingest_info": (i32, [vp, P(i64), P(i64), P(i64), P(i64)]),
        "lv_ingest_copy_csr": (i32, [vp, vp, vp, i32]),
        "lv_ingest_run": (i32, [vp, vp, i32, P(dbl), P(Stats)]),
        "lv_ingest_destroy": (i32, [vp]),
    }
    missing = []
    for name, (res, args) in sig.items():
        try:
            fn = getattr(L, name)
        except AttributeError:
            missing.append(name)
            continue
        fn.restype = res
        fn.argtypes = args
    L.missing_exports = tuple(missing)
    if path is None:
        _lib = L
    return L


def _ptr(a) -> Optional[int]:
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return int(a.data_ptr())  # torch tensor


def _is_device(a) -> bool:
    return a is not None and not isinstance(a, np.ndarray) and getattr(a, "is_cuda", False)


def config(mode: int = MODE.SORT, threshold: float = 1e-3, fast_first: bool = True,
           chunk_edges: int = 50_000_000, max_iterations: int = 1_000_000_000,
           max_levels: int = 0, weight_mode: int = WEIGHTS_AUTO,
           bin_max_degree: Optional[Sequence[int]] = None, use_graphs: bool = True,
           refine: bool = False, refine_passes: int = 0,
           refine_tolerance: Optional[float] = None) -> Config:
    c = Config()
    load_library().lv_config_default(ctypes.byref(c))
    c.mode = int(mode)
    c.threshold = float(threshold)
    c.fast_first = int(bool(fast_first))
    c.chunk_edges = int(chunk_edges)
    c.max_iterations = int(max_iterations)
    c.max_levels = int(max_levels)
    c.weight_mode = int(weight_mode)
    c.use_graphs = int(bool(use_graphs))
    c.refine = int(bool(refine))
    c.refine_passes = int(refine_passes)
    if refine_tolerance is not None:
        c.refine_tolerance = float(refine_tolerance)
    if bin_max_degree is not None:
        for i, d in enumerate(bin_max_degree[:8]):
            c.bin_max_degree[i] = int(d)
    return c


class Engine:
    """An lv_context: one device, its stream and reusable state."""

    def __init__(self, device: int = 0, cfg: Optional[Config] = None, **kw):
        self._L = load_library()
        self._deps = weakref.WeakSet()
        self.cfg = cfg if cfg is not None else config(**kw)
        h = ctypes.c_void_p()
        st = self._L.lv_create(int(device), ctypes.byref(self.cfg), ctypes.byref(h))
        if st != 0:
            raise LouvainError(st, "lv_create failed: " + self._L.lv_status_string(st).decode())
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            # communities, ingested graphs and servers use the context: they go first
            for d in list(getattr(self, "_deps", ())):
                d.close()
            self._L.lv_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def check(self, st: int, what: str):
        if st != 0:
            msg = self._L.lv_last_error(self._h).decode() or self._L.lv_status_string(st).decode()
            raise LouvainError(st, f"{what}: {msg}")

    # -- one-shot --------------------------------------------------------------------------
    def run_csr(self, n: int, row_ptr, col, w=None, out=None, stats: bool = True):
        """lv_run_csr on numpy (host) or torch CUDA (device) arrays. Returns
        (communities, modularity, Stats)."""
        dev = _is_device(row_ptr)
        if not dev:
            row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int64)
            col = np.ascontiguousarray(col, dtype=np.int32)
            w = None if w is None else np.ascontiguousarray(w, dtype=np.float32)
        if out is None:
            out = np.empty(n, dtype=np.int32)
        q = ctypes.c_double(0)
        s = Stats()
        st = self._L.lv_run_csr(self._h, int(n), _ptr(row_ptr), _ptr(col), _ptr(w),
                                MEM_DEVICE if dev else MEM_HOST, _ptr(out),
                                MEM_DEVICE if _is_device(out) else MEM_HOST,
                                ctypes.byref(q), ctypes.byref(s) if stats else None)
        self.check(st, "lv_run_csr")
        return out, q.value, s

    def run_graph(self, g: CSRGraph):
        return self.run_csr(g.n, g.row_ptr, g.col, g.w)

    def run_batch(self, vtx_offsets, row_ptr, col, w=None, out=None):
        """lv_run_batch: returns (communities, modularity[G], n_communities[G], Stats)."""
        dev = _is_device(row_ptr)
        if not dev:
            vtx_offsets = np.ascontiguousarray(vtx_offsets, dtype=np.int64)
            row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int64)
            col = np.ascontiguousarray(col, dtype=np.int32)
            w = None if w is None else np.ascontiguousarray(w, dtype=np.float32)
            G = vtx_offsets.size - 1
            n = int(vtx_offsets[-1])
        else:
            G = int(vtx_offsets.numel()) - 1
            n = int(vtx_offsets[-1].item())
        if out is None:
            out = np.empty(n, dtype=np.int32)
        qs = np.empty(G, dtype=np.float64)
        ks = np.empty(G, dtype=np.int32)
        s = Stats()
        st = self._L.lv_run_batch(self._h, G, _ptr(vtx_offsets), _ptr(row_ptr), _ptr(col), _ptr(w),
                                  MEM_DEVICE if dev else MEM_HOST, _ptr(out),
                                  MEM_DEVICE if _is_device(out) else MEM_HOST,
                                  qs.ctypes.data, ks.ctypes.data, ctypes.byref(s))
        self.check(st, "lv_run_batch")
        return out, qs, ks, s

    def autotune(self, vtx_offsets, row_ptr, col, w=None, trials: int = 2):
        """lv_autotune on a sample (a packed batch, or one graph with vtx_offsets = [0, n]):
        installs the fastest degree-bin table in this engine. Returns (bins[8], best_ms)."""
        dev = _is_device(row_ptr)
        if not dev:
            vtx_offsets = np.ascontiguousarray(vtx_offsets, dtype=np.int64)
            row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int64)
            col = np.ascontiguousarray(col, dtype=np.int32)
            w = None if w is None else np.ascontiguousarray(w, dtype=np.float32)
            G = vtx_offsets.size - 1
        else:
            G = int(vtx_offsets.numel()) - 1
        out = Config()
        ms = ctypes.c_double(0)
        self.check(self._L.lv_autotune(self._h, G, _ptr(vtx_offsets), _ptr(row_ptr), _ptr(col), _ptr(w),
                                       MEM_DEVICE if dev else MEM_HOST, int(trials), ctypes.byref(out),
                                       ctypes.byref(ms)), "lv_autotune")
        self.cfg = out
        return list(out.bin_max_degree), ms.value

    def ingest(self, source, skip_line: int = 0) -> "Ingest":
        """lv_ingest_edge_list: an edge-list file (path) or its bytes parsed into a CSR on the
        GPU with the reference's GraphHost rules (graph.cu:17-87)."""
        return Ingest(self, source, skip_line)

    def resume(self, ckpt: dict) -> "CommunityState":
        """lv_community_resume from CommunityState.checkpoint()'s dict."""
        row = np.ascontiguousarray(ckpt["row_ptr"], dtype=np.int64)
        col = np.ascontiguousarray(ckpt["col"], dtype=np.int32)
        w = np.ascontiguousarray(ckpt["w"], dtype=np.float64)
        best = np.ascontiguousarray(ckpt["best"], dtype=np.int32)
        h = ctypes.c_void_p()
        self.check(self._L.lv_community_resume(self._h, int(ckpt["n0"]), best.ctypes.data,
                                               int(ckpt["level"]), int(ckpt["iterations"]),
                                               row.size - 1, row.ctypes.data, col.ctypes.data,
                                               w.ctypes.data, int(ckpt["weights_integer"]),
                                               ctypes.byref(h)), "lv_community_resume")
        return CommunityState(self, None, _handle=h, _n0=int(ckpt["n0"]))

    def community(self, g: CSRGraph) -> "CommunityState":
        return CommunityState(self, g)


class CommunityState:
    """Phase-level handle (lv_community): the reference's Community plus the phase calls
    OptimizationPhase::run / AggregationPhase::run that modularity_routine makes."""

    def __init__(self, engine: Engine, g: Optional[CSRGraph], _handle=None, _n0: int = 0):
        self.e = engine
        if _handle is not None:  # built by Engine.resume
            self._h = _handle
            self.n0 = _n0
            engine._deps.add(self)
            return
        self._row = np.ascontiguousarray(g.row_ptr, dtype=np.int64)
        self._col = np.ascontiguousarray(g.col, dtype=np.int32)
        self._w = None if g.w is None else np.ascontiguousarray(g.w, dtype=np.float32)
        h = ctypes.c_void_p()
        st = engine._L.lv_community_create(engine._h, g.n, _ptr(self._row), _ptr(self._col),
                                           _ptr(self._w), MEM_HOST, ctypes.byref(h))
        engine.check(st, "lv_community_create")
        self._h = h
        self.n0 = g.n
        engine._deps.add(self)

    def close(self):
        # (a context already destroyed took this object's device memory with it)
        if getattr(self, "_h", None) and getattr(self.e, "_h", None):
            self.e._L.lv_community_destroy(self._h)
        self._h = None

    def __del__(self):
        self.close()

    def checkpoint(self) -> dict:
        """The run's state at a level start (call after aggregation_run(True), before the
        next optimisation): enough for Engine.resume to continue it anywhere."""
        info = self.info()
        tr = self.trace()
        row, col, w, _ = self.graph()
        return {"n0": int(info.n0), "level": int(info.level), "iterations": int(len(tr)),
                "weights_integer": int(info.weights_integer), "row_ptr": row, "col": col,
                "w": np.asarray(w, dtype=np.float64), "best": self.best().astype(np.int32)}

    def optimization_step(self):
        d = ctypes.c_double(0)
        mv = ctypes.c_int64(0)
        self.e.check(self.e._L.lv_optimization_step(self._h, ctypes.byref(d), ctypes.byref(mv)),
                     "lv_optimization_step")
        return int(mv.value), d.value

    def optimization_run(self) -> int:
        it = ctypes.c_int32(0)
        self.e.check(self.e._L.lv_optimization_run(self._h, ctypes.byref(it)), "lv_optimization_run")
        return it.value

    def aggregation_run(self, aggregate: bool) -> None:
        self.e.check(self.e._L.lv_aggregation_run(self._h, int(bool(aggregate))), "lv_aggregation_run")

    def louvain(self) -> Stats:
        s = Stats()
        self.e.check(self.e._L.lv_louvain(self._h, ctypes.byref(s)), "lv_louvain")
        return s

    def info(self) -> CommunityInfo:
        i = CommunityInfo()
        self.e.check(self.e._L.lv_community_info_get(self._h, ctypes.byref(i)), "lv_community_info_get")
        return i

    def partition(self):
        n = self.info().n
        comm = np.empty(n, dtype=np.int32)
        tot = np.empty(n, dtype=np.float64)
        self.e.check(self.e._L.lv_community_get_partition(self._h, comm.ctypes.data, tot.ctypes.data),
                     "lv_community_get_partition")
        return comm, tot

    def best(self) -> np.ndarray:
        out = np.empty(self.n0, dtype=np.int32)
        self.e.check(self.e._L.lv_community_get_best(self._h, out.ctypes.data), "lv_community_get_best")
        return out

    def graph(self):
        i = self.info()
        row = np.empty(i.n + 1, dtype=np.int64)
        col = np.empty(max(i.E, 1), dtype=np.int32)
        w = np.empty(max(i.E, 1), dtype=np.float64)
        k = np.empty(max(i.n, 1), dtype=np.float64)
        self.e.check(self.e._L.lv_community_get_graph(self._h, row.ctypes.data, col.ctypes.data,
                                                      w.ctypes.data, k.ctypes.data),
                     "lv_community_get_graph")
        return row, col[: i.E], w[: i.E], k[: i.n]

    def trace(self) -> np.ndarray:
        cap = 4096
        out = np.empty(cap, dtype=TRACE_DTYPE)
        ln = ctypes.c_int32(0)
        self.e.check(self.e._L.lv_community_get_trace(self._h, out.ctypes.data, cap, ctypes.byref(ln)),
                     "lv_community_get_trace")
        return out[: min(ln.value, cap)]


class Ingest:
    """A graph read on the GPU from edge-list text (lv_ingest_*): n_nodes, n_links, min_id,
    the CSR (``csr()``) and Louvain on it without leaving the device (``run()``)."""

    def __init__(self, engine: Engine, source, skip_line: int = 0):
        self.e = engine
        if isinstance(source, np.ndarray):  # the bytes in a uint8 array (read in place)
            data = np.ascontiguousarray(source, dtype=np.uint8)
            ptr, size = data.ctypes.data, data.size
        else:
            if isinstance(source, (bytes, bytearray, memoryview)):
                raw = bytes(source)
            else:
                with open(source, "rb") as f:
                    raw = f.read()
            data = ctypes.create_string_buffer(raw, len(raw))
            ptr, size = ctypes.addressof(data), len(raw)
        h = ctypes.c_void_p()
        engine.check(engine._L.lv_ingest_edge_list(engine._h, ptr, size, int(skip_line), MEM_HOST,
                                                   ctypes.byref(h)), "lv_ingest_edge_list")
        self._h = h
        engine._deps.add(self)
        n, m, E, mn = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        engine._L.lv_ingest_info(h, ctypes.byref(n), ctypes.byref(m), ctypes.byref(E), ctypes.byref(mn))
        self.n_nodes, self.n_links, self.entries, self.min_id = n.value, m.value, E.value, mn.value

    def close(self):
        if getattr(self, "_h", None) and getattr(self.e, "_h", None):
            self.e._L.lv_ingest_destroy(self._h)
        self._h = None

    def __del__(self):
        self.close()

    def csr(self) -> CSRGraph:
        row = np.empty(self.n_nodes + 1, dtype=np.int64)
        col = np.empty(self.entries, dtype=np.int32)
        self.e.check(self.e._L.lv_ingest_copy_csr(self._h, row.ctypes.data, col.ctypes.data, MEM_HOST),
                     "lv_ingest_copy_csr")
        return CSRGraph(n=self.n_nodes, row_ptr=row, col=col, w=None, name="ingested")

    def run(self):
        """(communities, modularity, Stats) of a Louvain run on the ingested graph."""
        out = np.empty(self.n_nodes, dtype=np.int32)
        q = ctypes.c_double(0)
        st = Stats()
        self.e.check(self.e._L.lv_ingest_run(self._h, out.ctypes.data, MEM_HOST, ctypes.byref(q),
                                             ctypes.byref(st)), "lv_ingest_run")
        return out, q.value, st


class Server:
    """lv_server_*: requests admitted under a device-memory budget into `slots` concurrent
    streams of one Engine's device; each request is one single-graph Louvain run."""

    def __init__(self, engine: Engine, budget_bytes: int, slots: int = 8):
        self.e = engine
        h = ctypes.c_void_p()
        engine.check(engine._L.lv_server_create(engine._h, int(budget_bytes), int(slots), ctypes.byref(h)),
                     "lv_server_create")
        self._h = h
        self.n_of = {}
        self._held = {}
        engine._deps.add(self)

    def close(self):
        if getattr(self, "_h", None) and getattr(self.e, "_h", None):
            self.e._L.lv_server_destroy(self._h)  # joins the workers: borrowed buffers are free after
        self._h = None
        self._held = {}

    def __del__(self):
        self.close()

    def submit(self, g: CSRGraph, borrow: bool = False) -> int:
        """Queues host CSR `g` and returns the request id. borrow=False copies the arrays at
        submit; borrow=True hands them to the server as they are (lv_server_submit_borrowed),
        and this object keeps them referenced until the request is polled done."""
        row = np.ascontiguousarray(g.row_ptr, dtype=np.int64)
        col = np.ascontiguousarray(g.col, dtype=np.int32)
        w = None if g.w is None else np.ascontiguousarray(g.w, dtype=np.float32)
        rid = ctypes.c_int64(0)
        fn = self.e._L.lv_server_submit_borrowed if borrow else self.e._L.lv_server_submit
        self.e.check(fn(self._h, int(g.n), row.ctypes.data, col.ctypes.data,
                        None if w is None else w.ctypes.data, ctypes.byref(rid)),
                     "lv_server_submit")
        self.n_of[rid.value] = int(g.n)
        if borrow:
            self._held[rid.value] = (row, col, w)
        return rid.value

    def progress(self):
        """(finished, running, queued) request counts."""
        d, r, q = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        self.e.check(self.e._L.lv_server_progress(self._h, ctypes.byref(d), ctypes.byref(r), ctypes.byref(q)),
                     "lv_server_progress")
        return d.value, r.value, q.value

    def poll(self, rid: int):
        """None while request `rid` runs; then (communities, modularity, latency_ms)."""
        out = np.empty(self.n_of[rid], dtype=np.int32)
        q, lat, done = ctypes.c_double(), ctypes.c_double(), ctypes.c_int32(0)
        st = self.e._L.lv_server_poll(self._h, int(rid), out.ctypes.data, ctypes.byref(q),
                                      ctypes.byref(lat), ctypes.byref(done))
        if done.value or st != 0:
            self._held.pop(rid, None)
        self.e.check(st, "lv_server_poll")
        return (out, q.value, lat.value) if done.value else None

    def drain(self):
        self.e.check(self.e._L.lv_server_drain(self._h), "lv_server_drain")


# ---- the reference's own names -------------------------------------------------------------------
class GraphHost:
    """graphHost.cuh:7-18. ``GraphHost(name, weighted, skip_line)`` parses an ``a b`` edge list
    like graph.cu:17-87; ``GraphHost.from_csr(g)`` wraps an in-memory CSRGraph."""

    def __init__(self, name: Optional[str] = None, weighted: bool = False, skip_line: int = 0,
                 csr: Optional[CSRGraph] = None):
        if csr is None:
            if weighted:
                raise LouvainError(2, "weighted edge lists are not parsed (the reference's "
                                      "weighted branch is a TODO, graph.cu:32-34); pass a CSRGraph")
            csr = graphs.read_edge_list(name, skip_line)
        self.csr = csr
        self.n_nodes = csr.n
        self.n_links = csr.m
        self.total_weight = float(csr.weights_or_ones.sum()) / 2.0
        self.min_id = 0

    @classmethod
    def from_csr(cls, g: CSRGraph) -> "GraphHost":
        return cls(csr=g)


class Community:
    """community.h:15-26: the result of a Louvain run."""

    def __init__(self, best, n_best: int, modularity: float, stats: Optional[Stats] = None):
        self.best_communities = best
        self.n_of_best_communities = int(n_best)
        self.modularity = float(modularity)
        self.stats = stats


_engines = {}


def _engine_for(mode: int, **kw) -> Engine:
    key = (int(mode), tuple(sorted(kw.items())))
    if key not in _engines:
        _engines[key] = Engine(0, mode=mode, **kw)
    return _engines[key]


class ModularityAlgorithms:
    """modularityAlgorithms.h:7-82."""

    @staticmethod
    def Louvain(graph: GraphHost, fastLocalMoveEnable: int = MODE.SORT, **kw) -> Community:
        g = graph.csr if isinstance(graph, GraphHost) else graph
        e = _engine_for(int(fastLocalMoveEnable), **kw)
        best, q, s = e.run_graph(g)
        return Community(best, s.n_communities, q, s)
