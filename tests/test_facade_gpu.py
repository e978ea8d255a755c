"""The C++ drop-in on the GPU: tests/facade_main.cpp is written like the reference's main.cu
(main.cu:16-33: GraphHost from an edge-list file, ModularityAlgorithms::Louvain, read the
Community). It is compiled against include/louvain_b200.hpp, linked with the engine library,
run on the reference's bundled fixture written as an edge list, and its community count,
modularity and best_communities must equal the reference's own outputs for that fixture in
SORT and HASH mode (tests/golden/fixture_power_law_10000__{SORT,HASH}.npz, produced by the
reference's CUDA build)."""
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

pytestmark = pytest.mark.gpu

SUMMARY = json.load(open(os.path.join(GOLDEN, "reference_summary.json")))
Q_TOL = 1e-12


@pytest.fixture(scope="module")
def facade_exe(lv, tmp_path_factory):
    lib = lv.load_library()._name
    d = tmp_path_factory.mktemp("facade")
    exe = str(d / "facade_main")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror",
                    "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "facade_main.cpp"), lib,
                    "-Wl,-rpath," + os.path.dirname(lib), "-o", exe], check=True)
    return exe


@pytest.mark.parametrize("mode", ["SORT", "HASH"])
def test_cpp_facade_runs_like_reference_main(mode, facade_exe, golden, tmp_path):
    g = golden.load_fixture()
    edges = tmp_path / "graph-power-law-10000-2-99-1.edge"
    edges.write_text(g.edge_list_text())
    out = tmp_path / "best.bin"
    p = subprocess.run([facade_exe, str(edges), mode, str(out)], capture_output=True, text=True,
                       timeout=300)
    assert p.returncode == 0, p.stderr
    k, q = p.stdout.split()
    rec = SUMMARY[f"fixture_power_law_10000__{mode}"]
    assert int(k) == rec["n_best"]
    assert abs(float(q) - rec["modularity"]) <= Q_TOL
    best = np.fromfile(out, dtype=np.uint32).astype(np.int32)
    ref = np.load(os.path.join(GOLDEN, f"fixture_power_law_10000__{mode}.npz"))["best"]
    np.testing.assert_array_equal(best, ref)


def test_cpp_facade_reports_bad_file(facade_exe, tmp_path):
    """An empty edge list: the reference exit(0)s (graph.cu:52-55); the facade throws
    louvain::Error, which the caller reports with a non-zero status."""
    empty = tmp_path / "empty.edge"
    empty.write_text("")
    p = subprocess.run([facade_exe, str(empty), "SORT", str(tmp_path / "o.bin")],
                       capture_output=True, text=True, timeout=120)
    assert p.returncode == 1 and "louvain error" in p.stderr
