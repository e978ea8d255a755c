"""ctypes wrapper of the CPU oracle (liblouvain_oracle.so).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline leg / CPU reference arm, always as the checker or the timed CPU baseline.
The product path (the CUDA engine) never imports this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liblouvain_oracle.so")
_lib = None

HASH, SORT = 0, 1


class OrcConfig(ctypes.Structure):
    _fields_ = [
        ("mode", ctypes.c_int32),
        ("fast_first", ctypes.c_int32),
        ("max_iterations", ctypes.c_int32),
        ("max_levels", ctypes.c_int32),
        ("threshold", ctypes.c_double),
        ("chunk_edges", ctypes.c_int64),
        ("nthreads", ctypes.c_int32),
        ("integer_weights", ctypes.c_int32),
        ("refine", ctypes.c_int32),
        ("refine_passes", ctypes.c_int32),
        ("refine_tolerance", ctypes.c_double),
    ]


TRACE_DTYPE = np.dtype([
    ("level", np.int32), ("iteration", np.int32), ("n_considered", np.int32),
    ("n_moved", np.int32), ("internal", np.float64), ("sum_a2", np.float64),
    ("modularity", np.float64), ("delta", np.float64),
    ("n_pairs", np.int64), ("n_internal", np.int64),
])


def build() -> str:
    """Compile the oracle in place (make -C oracle)."""
    subprocess.run(["make", "-s", "-C", _HERE, "liblouvain_oracle.so"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        vp = ctypes.c_void_p
        L.orc_create.restype = vp
        L.orc_create.argtypes = [ctypes.c_int64, vp, vp, vp, ctypes.POINTER(OrcConfig),
                                 ctypes.POINTER(ctypes.c_int32)]
        L.orc_destroy.argtypes = [vp]
        for name in ("orc_louvain", "orc_optimization_run"):
            getattr(L, name).restype = ctypes.c_int32
            getattr(L, name).argtypes = [vp]
        L.orc_aggregation_run.restype = ctypes.c_int32
        L.orc_aggregation_run.argtypes = [vp, ctypes.c_int32]
        L.orc_optimization_step.restype = ctypes.c_int32
        L.orc_optimization_step.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
        for name in ("orc_n", "orc_E", "orc_n_best", "orc_trace_len", "orc_overrun_events",
                     "orc_refine_passes"):
            getattr(L, name).restype = ctypes.c_int64
            getattr(L, name).argtypes = [vp]
        L.orc_level.restype = ctypes.c_int32
        L.orc_level.argtypes = [vp]
        for name in ("orc_modularity", "orc_internal", "orc_sum_a2", "orc_total_weight"):
            getattr(L, name).restype = ctypes.c_double
            getattr(L, name).argtypes = [vp]
        for name in ("orc_get_best", "orc_get_comm", "orc_get_totals", "orc_get_k", "orc_get_trace"):
            getattr(L, name).restype = None
            getattr(L, name).argtypes = [vp, vp]
        L.orc_get_graph.restype = None
        L.orc_get_graph.argtypes = [vp, vp, vp, vp]
        L.orc_record_size.restype = ctypes.c_int32
        assert L.orc_record_size() == TRACE_DTYPE.itemsize
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


class Oracle:
    """One Louvain run on the CPU oracle, with the reference's phase granularity."""

    def __init__(self, graph, mode: int = SORT, threshold: float = 1e-3,
                 fast_first: bool = True, chunk_edges: int = 50_000_000,
                 max_iterations: int = 1_000_000_000, max_levels: int = 0,
                 nthreads: int = 1, integer_weights: Optional[bool] = None,
                 refine: bool = False, refine_passes: int = 0,
                 refine_tolerance: float = 0.95):
        L = lib()
        self._row = np.ascontiguousarray(graph.row_ptr, dtype=np.int64)
        self._col = np.ascontiguousarray(graph.col, dtype=np.int32)
        w = graph.w
        if integer_weights is None:
            integer_weights = w is None or bool(np.all(np.floor(w) == w))
        self._w = None if w is None else np.ascontiguousarray(w, dtype=np.float32)
        cfg = OrcConfig(mode, int(fast_first), max_iterations, max_levels, threshold,
                        chunk_edges, nthreads, int(integer_weights), int(refine), refine_passes,
                        refine_tolerance)
        err = ctypes.c_int32(0)
        self._h = L.orc_create(graph.n, _ptr(self._row), _ptr(self._col),
                               None if self._w is None else _ptr(self._w),
                               ctypes.byref(cfg), ctypes.byref(err))
        if not self._h:
            raise ValueError(f"oracle rejected the graph (code {err.value})")
        self.n0 = graph.n

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().orc_destroy(h)
            self._h = None

    # phases ------------------------------------------------------------------------
    def louvain(self) -> int:
        r = lib().orc_louvain(self._h)
        if r < 0:
            raise RuntimeError(f"oracle aggregation failed ({-r})")
        return r

    def optimization_run(self) -> int:
        return lib().orc_optimization_run(self._h)

    def optimization_step(self):
        d = ctypes.c_double(0)
        moved = lib().orc_optimization_step(self._h, ctypes.byref(d))
        return moved, d.value

    def aggregation_run(self, aggregate: bool) -> None:
        r = lib().orc_aggregation_run(self._h, int(aggregate))
        if r != 0:
            raise RuntimeError(f"oracle aggregation failed ({r})")

    # state -------------------------------------------------------------------------
    @property
    def n(self) -> int:
        return lib().orc_n(self._h)

    @property
    def E(self) -> int:
        return lib().orc_E(self._h)

    @property
    def level(self) -> int:
        return lib().orc_level(self._h)

    @property
    def modularity(self) -> float:
        return lib().orc_modularity(self._h)

    @property
    def internal(self) -> float:
        return lib().orc_internal(self._h)

    @property
    def sum_a2(self) -> float:
        return lib().orc_sum_a2(self._h)

    @property
    def total_weight(self) -> float:
        return lib().orc_total_weight(self._h)

    @property
    def overrun_events(self) -> int:
        """Times the reference's modularity scratch (community.h:69,85) would be too short."""
        return lib().orc_overrun_events(self._h)

    @property
    def refine_passes(self) -> int:
        """Refinement passes run so far (refine=True)."""
        return lib().orc_refine_passes(self._h)

    @property
    def n_best(self) -> int:
        return lib().orc_n_best(self._h)

    def best(self) -> np.ndarray:
        out = np.empty(self.n0, dtype=np.int32)
        lib().orc_get_best(self._h, _ptr(out))
        return out

    def comm(self) -> np.ndarray:
        out = np.empty(self.n, dtype=np.int32)
        lib().orc_get_comm(self._h, _ptr(out))
        return out

    def totals(self) -> np.ndarray:
        out = np.empty(self.n, dtype=np.float64)
        lib().orc_get_totals(self._h, _ptr(out))
        return out

    def k(self) -> np.ndarray:
        out = np.empty(self.n, dtype=np.float64)
        lib().orc_get_k(self._h, _ptr(out))
        return out

    def graph(self):
        n, E = self.n, self.E
        row = np.empty(n + 1, dtype=np.int64)
        col = np.empty(max(E, 1), dtype=np.int32)
        w = np.empty(max(E, 1), dtype=np.float64)
        lib().orc_get_graph(self._h, _ptr(row), _ptr(col), _ptr(w))
        return row, col[:E], w[:E]

    def trace(self) -> np.ndarray:
        n = lib().orc_trace_len(self._h)
        out = np.empty(n, dtype=TRACE_DTYPE)
        if n:
            lib().orc_get_trace(self._h, _ptr(out))
        return out


def louvain(graph, **kw):
    """Full run; returns (best, n_best, modularity, trace)."""
    o = Oracle(graph, **kw)
    o.louvain()
    return o.best(), o.n_best, o.modularity, o.trace()
