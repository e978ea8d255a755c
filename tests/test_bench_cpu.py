"""bench.py's CPU reference arm keeps its output contract: one JSON line with the metric,
unit, direction and config of the GPU arm, `impl: reference`, a `cpu_baseline` that describes
this run (kind, cores, sample) with the line's own value, and an `e2e` object with no
host<->device bytes; with --refine the same, on the refined run."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT


@pytest.mark.parametrize("refine", [False, True])
def test_reference_arm_line(refine):
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--scale", "10",
           "--steps", "1", "--warmup", "0"] + (["--refine"] if refine else [])
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "louvain_edges_per_s" and d["unit"] == "edges/s"
    assert d["higher_is_better"] is True and d["steps"] == 1 and d["warmup"] == 0
    assert d["config"]["workload"] == "rmat_s10_ef16" and d["config"]["refine"] is refine
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["unit"] == d["unit"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
    assert 0.0 < d["modularity"] < 1.0 and d["n_communities"] >= 1
