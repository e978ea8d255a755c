"""The C ABI without a GPU: the library loads, exports every function include/louvain_b200.h
declares, its structs have the layout the header gives, host-only entry points behave, and
both the C++ drop-in header and a caller written against the reference's API compile and
link."""
import ctypes
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "louvain_b200.h")
HPP = os.path.join(ROOT, "include", "louvain_b200.hpp")
PKGDIR = os.path.join(ROOT, "louvain-fast-move-cuda_b200")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(lv_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_function(lv):
    L = lv.load_library()
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert missing == []
    assert L.missing_exports == ()
    assert set(lv.EXPORTS) <= set(names)


def _c_layout():
    prog = r'''
#include <stddef.h>
#include <stdio.h>
#include "louvain_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu\n", sizeof(lv_config), sizeof(lv_stats), sizeof(lv_community_info), sizeof(lv_trace_record));
  printf("%zu %zu %zu %zu\n", offsetof(lv_config, threshold), offsetof(lv_config, bin_max_degree),
         offsetof(lv_stats, bytes_optimization), offsetof(lv_stats, kernel_launches));
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "l.c")
        exe = os.path.join(d, "l")
        open(c, "w").write(prog)
        subprocess.run(["gcc", "-std=c99", "-I", os.path.dirname(HEADER), c, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    return [int(x) for x in out]


def test_struct_layouts_match_header(lv):
    s_cfg, s_stats, s_info, s_trace, o_thr, o_bins, o_bytes, o_launch = _c_layout()
    assert ctypes.sizeof(lv.Config) == s_cfg
    assert ctypes.sizeof(lv.Stats) == s_stats
    assert ctypes.sizeof(lv.CommunityInfo) == s_info
    assert lv.TRACE_DTYPE.itemsize == s_trace
    assert lv.Config.threshold.offset == o_thr
    assert lv.Config.bin_max_degree.offset == o_bins
    assert lv.Stats.bytes_optimization.offset == o_bytes
    assert lv.Stats.kernel_launches.offset == o_launch


def test_config_defaults_follow_reference_constants(lv):
    c = lv.config()
    assert c.mode == lv.MODE.SORT
    assert c.threshold == 0.001          # constants.h:15
    assert c.chunk_edges == 50_000_000   # constants.h:18
    assert c.max_iterations == 1_000_000_000  # constants.h:16
    assert c.fast_first == 1
    # the library's own default (lv_config_default), not only the Python wrapper's
    raw = lv.Config()
    lv.load_library().lv_config_default(raw)
    assert raw.use_graphs == 1 and raw.validate == 1 and raw.weight_mode == lv.WEIGHTS_AUTO
    assert raw.refine == 0 and raw.refine_passes == 0 and raw.refine_tolerance == 0.95


def test_refine_configuration_validated_before_device_work(lv):
    L = lv.load_library()
    for field, value in (("refine", 2), ("refine_passes", -1), ("refine_tolerance", 1.5),
                         ("refine_tolerance", float("nan"))):
        c = lv.config(refine=True)
        setattr(c, field, value)
        h = ctypes.c_void_p()
        assert L.lv_create(0, ctypes.byref(c), ctypes.byref(h)) == 1  # LV_ERR_ARGUMENT
        assert not h.value


def test_status_strings(lv):
    L = lv.load_library()
    texts = [L.lv_status_string(i).decode() for i in range(9)]
    assert texts[0] == "ok" and all(texts)
    assert L.lv_status_string(99).decode() == "unknown status"
    assert L.lv_abi_version() == 1


def test_create_without_gpu_fails_cleanly(lv):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(lv.LouvainError) as ei:
        lv.Engine(0)
    assert ei.value.status == 4  # LV_ERR_CUDA, no abort


def test_invalid_arguments_rejected_before_device_work(lv):
    L = lv.load_library()
    assert L.lv_run_csr(None, 1, None, None, None, 0, None, 0, None, None) == 1
    assert L.lv_community_destroy(None) == 1
    assert L.lv_server_create(None, 1, 1, None) == 1
    assert L.lv_autotune(None, 1, None, None, None, None, 0, 1, None, None) == 1
    f = L.lv_modularity_noalloc if hasattr(L, "lv_modularity_noalloc") else None
    if f is not None:
        f.restype = ctypes.c_int32
        f.argtypes = [ctypes.c_int64] + [ctypes.c_void_p] * 4 + [ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p]
        assert f(0, None, None, None, None, 1, None, None) == 1


def test_cpp_facade_compiles_and_links(lv):
    lib = lv.load_library()._name
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "facade")
        subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-I", os.path.dirname(HPP),
                        os.path.join(ROOT, "tests", "facade_main.cpp"), lib,
                        "-Wl,-rpath," + os.path.dirname(lib), "-o", exe], check=True)
        assert os.path.exists(exe)


def test_python_graphhost_parses_like_reference(lv, golden, tmp_path):
    g = golden.load_fixture()
    p = tmp_path / "fixture.edge"
    p.write_text(g.edge_list_text())
    h = lv.GraphHost(str(p), False, 0)
    assert h.n_nodes == 10000 and h.n_links == 19996 and h.total_weight == 19996.0
    np.testing.assert_array_equal(h.csr.row_ptr, g.row_ptr)
    np.testing.assert_array_equal(h.csr.col, g.col)
    with pytest.raises(lv.LouvainError):
        lv.GraphHost(str(p), True, 0)
