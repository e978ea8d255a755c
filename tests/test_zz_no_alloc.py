"""lv_modularity_noalloc: the modularity entry point for callers that cannot allocate.

Some callers may not allocate device memory at the moment they ask for a result -- for
example a framework that has reserved all of HBM for its own pool, or a serving loop that
must never wait on cudaMalloc. lv_modularity_noalloc evaluates the modularity of a partition
using only the caller's buffers and one fixed scratch array inside the library. These tests
check it against the modularity that lv_run_csr (the existing entry point) reports for the
partition it returns, within the tolerance the other parity tests use (1e-12), on two calls
in a row, and check that a graph larger than the fixed scratch is refused up front.

This file is named to be collected last, so that a run stopping at its first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

Q_TOL = 1e-12
LV_ERR_RANGE = 3
MAX_VERTICES = 1048576  # LV_NOALLOC_MAX_VERTICES in include/louvain_b200.h


def _entry(lv):
    L = lv.load_library()
    f = L.lv_modularity_noalloc
    f.restype = ctypes.c_int32
    f.argtypes = [ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p]
    return f


def _noalloc_q(f, g, comm, weights_integer):
    import torch
    row = torch.from_numpy(np.ascontiguousarray(g.row_ptr, dtype=np.int64)).cuda()
    col = torch.from_numpy(np.ascontiguousarray(g.col, dtype=np.int32)).cuda()
    w = None if g.w is None else torch.from_numpy(g.w).cuda()
    lab = torch.from_numpy(np.ascontiguousarray(comm, dtype=np.int32)).cuda()
    out = torch.full((4,), -1.0, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    st = f(g.n, row.data_ptr(), col.data_ptr(), None if w is None else w.data_ptr(),
           lab.data_ptr(), int(weights_integer), out.data_ptr(), None)
    assert st == 0
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_noalloc_matches_run_csr_on_consecutive_calls(lv, golden, graphs):
    f = _entry(lv)
    fixture = golden.load_fixture()
    other = graphs.rmat(14, 16, seed=9)
    e = lv.Engine(0)
    best_a, q_a, _ = e.run_graph(fixture)
    best_b, q_b, _ = e.run_graph(other)
    e.close()
    # two calls in a row on the same input, then a different graph, then the first again:
    # the shared scratch keeps the previous call's values and each call must clear them
    r1 = _noalloc_q(f, fixture, best_a, True)
    r2 = _noalloc_q(f, fixture, best_a, True)
    assert abs(r1[0] - q_a) <= Q_TOL
    assert abs(r2[0] - q_a) <= Q_TOL
    assert r1[3] == fixture.m
    rb = _noalloc_q(f, other, best_b, True)
    assert abs(rb[0] - q_b) <= Q_TOL
    r3 = _noalloc_q(f, fixture, best_a, True)
    assert abs(r3[0] - q_a) <= Q_TOL


def test_noalloc_fp32_weights(lv, graphs):
    """fp32 weights (double accumulation on both sides). lv_run_csr reports Q on its last
    contracted level, whose weights are fp32 sums; weights that are multiples of 0.5 keep
    every such sum exact, so both entry points evaluate the same quantity."""
    f = _entry(lv)
    g = graphs.planted_partition(n=3000, n_comm=30, smin=20, smax=300, mean_degree=10, seed=4)
    g.w = np.maximum(np.round(g.w * 2.0) / 2.0, 0.5).astype(np.float32)
    assert not np.all(np.floor(g.w) == g.w)
    e = lv.Engine(0)
    best, q, _ = e.run_graph(g)
    e.close()
    for _ in range(2):
        r = _noalloc_q(f, g, best, False)
        assert abs(r[0] - q) <= Q_TOL


def test_noalloc_allocates_nothing(lv, golden):
    """The point of the entry point: once its module is loaded on the device (the first call),
    a call leaves the device's free memory and torch's reserved pool exactly as they were."""
    import torch
    f = _entry(lv)
    g = golden.load_fixture()
    row = torch.from_numpy(np.ascontiguousarray(g.row_ptr, dtype=np.int64)).cuda()
    col = torch.from_numpy(np.ascontiguousarray(g.col, dtype=np.int32)).cuda()
    lab = torch.arange(g.n, dtype=torch.int32, device="cuda")
    out = torch.empty(4, dtype=torch.float64, device="cuda")
    args = (g.n, row.data_ptr(), col.data_ptr(), None, lab.data_ptr(), 1, out.data_ptr(), None)
    assert f(*args) == 0  # warm call: loads the module and looks up the scratch address
    torch.cuda.synchronize()
    free0, reserved0 = torch.cuda.mem_get_info()[0], torch.cuda.memory_reserved()
    for _ in range(2):
        assert f(*args) == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert torch.cuda.memory_reserved() == reserved0
    r = out.cpu().numpy()
    assert r[3] == g.m and np.isfinite(r[0])


def test_noalloc_flags_bad_input_as_nan(lv, golden):
    """Checks made on the device: a column outside [0, n) makes Q and m NaN (the call never
    synchronises, so it cannot return an error for it); a zero total weight gives m = 0 and
    Q NaN, which out[3] tells apart from bad input."""
    f = _entry(lv)
    g = golden.load_fixture()
    comm = np.arange(g.n, dtype=np.int32)
    bad = type(g)(n=g.n, row_ptr=g.row_ptr, col=g.col.copy())
    bad.col[5] = g.n + 3
    r = _noalloc_q(f, bad, comm, True)
    assert np.isnan(r[0]) and np.isnan(r[3])
    zero = type(g)(n=g.n, row_ptr=g.row_ptr, col=g.col, w=np.zeros(len(g.col), dtype=np.float32))
    r = _noalloc_q(f, zero, comm, False)
    assert np.isnan(r[0]) and r[3] == 0.0
    r = _noalloc_q(f, g, comm, True)  # the next call after bad input is clean again
    assert np.isfinite(r[0]) and r[3] == g.m


def test_noalloc_rejects_graph_beyond_scratch(lv):
    f = _entry(lv)
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    st = f(MAX_VERTICES + 1, dummy, dummy, None, dummy, 1, dummy, None)
    assert st == LV_ERR_RANGE
