"""Generate golden vectors by running the reference's own CUDA build.

This is the script that produced the committed fixtures in this directory. It needs a
CUDA GPU and the reference binary built by ``make -C oracle ref REF=<reference tree>``
(oracle/_ref/ref_louvain,
compiled from the reference's unmodified sources). For each case and mode it

  1. builds the input graph (the reference's bundled fixture, read from
     ``fixture_power_law_10000.npz``, or a seeded generator from the package),
  2. runs the CPU oracle first and skips the case if the oracle predicts that the
     reference's modularity scratch (community.h:69,85, sized 2*(E/2)) would be one entry
     short -- an out-of-bounds write on the device that this script must not trigger,
  3. writes the graph in the reference's input format and runs the reference binary,
  4. records the reference's final partition, community count, modularity, every
     ``VALUES : I S m`` line it prints from compute_modularity (community.h:102) and its
     own timed window (modularityAlgorithms.h:69-75).

usage:
  python tests/golden/make_golden.py --out <dir>            # parity cases
  python tests/golden/make_golden.py --out <dir> --rmat22   # + scale-22 run
  python tests/golden/make_golden.py --import-fixture <graph-power-law-10000-2-99-1.edge>
"""
from __future__ import annotations

import argparse
import hashlib
import importlib
import json
import os
import re
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
graphs = importlib.import_module("louvain-fast-move-cuda_b200.graphs")
import oracle as O  # noqa: E402

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "ref_louvain")
FIXTURE = os.path.join(HERE, "fixture_power_law_10000.npz")


def load_fixture() -> "graphs.CSRGraph":
    z = np.load(FIXTURE)
    return graphs.CSRGraph(n=int(z["n"]), row_ptr=z["row_ptr"], col=z["col"],
                           name="fixture_power_law_10000")


def import_fixture(path: str) -> None:
    g = graphs.read_edge_list(path)
    np.savez_compressed(FIXTURE, n=np.int64(g.n), row_ptr=g.row_ptr, col=g.col)
    print(f"wrote {FIXTURE}: n={g.n} E={g.E}")


def case_graph(spec: dict) -> "graphs.CSRGraph":
    kind = spec["kind"]
    if kind == "fixture":
        return load_fixture()
    if kind == "chung_lu_bounded":
        return graphs.chung_lu_bounded(spec["n"], spec["exponent"], spec["dmin"], spec["dmax"], spec["seed"])
    if kind == "chung_lu_mean":
        return graphs.chung_lu_mean(spec["n"], spec["exponent"], spec["mean_degree"], spec["seed"])
    if kind == "rmat":
        if spec["scale"] >= 20:
            try:
                import torch
                if torch.cuda.is_available():
                    u, v = graphs.rmat_pairs(spec["scale"], spec["edge_factor"], seed=spec["seed"])
                    return graphs.to_device_canonical(u, v, name=spec["name"])
            except ImportError:
                pass
        return graphs.rmat(spec["scale"], spec["edge_factor"], seed=spec["seed"])
    if kind == "pairs":
        e = np.array(spec["edges"], dtype=np.int64)
        return graphs.canonical_from_pairs(e[:, 0], e[:, 1], name=spec["name"])
    raise ValueError(kind)


CASES = [
    {"name": "fixture_power_law_10000", "kind": "fixture"},
    {"name": "chung_lu_10000_s1", "kind": "chung_lu_bounded", "n": 10000, "exponent": 2.0, "dmin": 1, "dmax": 99, "seed": 1},
    {"name": "chung_lu_10000_s2", "kind": "chung_lu_bounded", "n": 10000, "exponent": 2.0, "dmin": 1, "dmax": 99, "seed": 2},
    {"name": "chung_lu_10000_s3", "kind": "chung_lu_bounded", "n": 10000, "exponent": 2.0, "dmin": 1, "dmax": 99, "seed": 3},
    {"name": "rmat_s10_ef16", "kind": "rmat", "scale": 10, "edge_factor": 16, "seed": 1},
    {"name": "rmat_s12_ef16", "kind": "rmat", "scale": 12, "edge_factor": 16, "seed": 1},
    {"name": "rmat_s14_ef16", "kind": "rmat", "scale": 14, "edge_factor": 16, "seed": 1},
    {"name": "rmat_s16_ef8", "kind": "rmat", "scale": 16, "edge_factor": 8, "seed": 2},
    {"name": "chung_lu_mean_20000", "kind": "chung_lu_mean", "n": 20000, "exponent": 2.1, "mean_degree": 8.0, "seed": 1},
    {"name": "two_triangles_bridge", "kind": "pairs", "edges": [[0, 1], [1, 2], [0, 2], [3, 4], [4, 5], [3, 5], [2, 3]]},
    {"name": "star_6", "kind": "pairs", "edges": [[0, 1], [0, 2], [0, 3], [0, 4], [0, 5]]},
    {"name": "path_8", "kind": "pairs", "edges": [[i, i + 1] for i in range(7)]},
    {"name": "clique_pair_k5", "kind": "pairs", "edges": [[i, j] for i in range(5) for j in range(i + 1, 5)]
        + [[5 + i, 5 + j] for i in range(5) for j in range(i + 1, 5)] + [[4, 5]]},
]
RMAT22 = {"name": "rmat_s22_ef16", "kind": "rmat", "scale": 22, "edge_factor": 16, "seed": 1}

VALUES_RE = re.compile(r"^VALUES : (\d+) ([0-9.]+) ([0-9.]+)")
TOTAL_RE = re.compile(r"Total Execution Time: ([0-9.eE+-]+)ms")


def graph_digest(g) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(g.row_ptr, dtype=np.int64).tobytes())
    h.update(np.ascontiguousarray(g.col, dtype=np.int32).tobytes())
    return h.hexdigest()[:16]


def run_reference(g, mode: str, workdir: str, big: bool = False):
    out = os.path.join(workdir, f"res_{mode}.bin")
    if big:
        inp = os.path.join(workdir, "graph.csr")
        with open(inp, "wb") as f:
            np.array([g.n, g.E], dtype=np.int64).tofile(f)
            np.ascontiguousarray(g.row_ptr, dtype=np.int64).tofile(f)
            np.ascontiguousarray(g.col, dtype=np.int32).tofile(f)
        args = [REF_BIN, inp, mode, out, "csr"]
    else:
        inp = os.path.join(workdir, "graph.edge")
        with open(inp, "w") as f:
            f.write(g.edge_list_text())
        args = [REF_BIN, inp, mode, out, "edges"]
    t0 = time.time()
    p = subprocess.run(args, capture_output=True, text=True, timeout=3600)
    wall = time.time() - t0
    if p.returncode != 0:
        return {"error": f"exit {p.returncode}", "stderr": p.stderr[-2000:], "stdout_tail": p.stdout[-2000:]}
    with open(out, "rb") as f:
        n0, nb = np.frombuffer(f.read(8), dtype=np.uint32)
        q = float(np.frombuffer(f.read(8), dtype=np.float64)[0])
        ms = float(np.frombuffer(f.read(4), dtype=np.float32)[0])
        best = np.frombuffer(f.read(4 * int(n0)), dtype=np.uint32).astype(np.int32)
    values = [(int(m.group(1)), float(m.group(2)), float(m.group(3)))
              for m in (VALUES_RE.match(l) for l in p.stdout.splitlines()) if m]
    t = TOTAL_RE.search(p.stdout)
    return {"n_best": int(nb), "modularity": q, "best": best, "values": values,
            "ref_window_ms": float(t.group(1)) if t else None, "driver_ms": ms, "wall_s": wall}


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(tempfile.gettempdir(), "louvain_golden"),
                    help="directory for the new golden files (copy the ones you keep into tests/golden)")
    ap.add_argument("--rmat22", action="store_true")
    ap.add_argument("--only", default=None)
    ap.add_argument("--import-fixture", default=None)
    a = ap.parse_args()
    if a.import_fixture:
        import_fixture(a.import_fixture)
        return 0
    if not os.path.exists(REF_BIN):
        print(f"missing {REF_BIN}; run `make -C oracle ref REF=<reference tree>` first")
        return 2
    os.makedirs(a.out, exist_ok=True)
    cases = list(CASES) + ([RMAT22] if a.rmat22 else [])
    summary = {}
    for spec in cases:
        if a.only and spec["name"] != a.only:
            continue
        g = case_graph(spec)
        big = g.E > 5_000_000
        for mode in ("SORT", "HASH"):
            key = f"{spec['name']}__{mode}"
            o = O.Oracle(g, mode=O.SORT if mode == "SORT" else O.HASH, nthreads=0)
            o.louvain()
            rec = {"case": spec, "mode": mode, "n": g.n, "E": g.E, "digest": graph_digest(g),
                   "oracle_n_best": o.n_best, "oracle_modularity": o.modularity}
            if o.overrun_events:
                rec["skipped"] = "oracle predicts a short modularity scratch buffer in the reference"
                summary[key] = rec
                print(key, "SKIPPED", flush=True)
                continue
            with tempfile.TemporaryDirectory() as wd:
                r = run_reference(g, mode, wd, big=big)
            if "error" in r:
                rec.update(r)
                summary[key] = rec
                print(key, "ERROR", r["error"], flush=True)
                continue
            best = r.pop("best")
            rec.update(r)
            rec["best_sha"] = hashlib.sha256(best.astype(np.int32).tobytes()).hexdigest()[:16]
            rec["oracle_match"] = bool(np.array_equal(best, o.best()))
            if not big:
                np.savez_compressed(os.path.join(a.out, key + ".npz"), best=best,
                                    values=np.array(r["values"], dtype=np.float64).reshape(-1, 3))
            summary[key] = rec
            print(key, "n_best", rec["n_best"], "Q", rec["modularity"], "oracle_match",
                  rec["oracle_match"], "ref_ms", rec["ref_window_ms"], flush=True)
    with open(os.path.join(a.out, "summary.json"), "w") as f:
        json.dump(summary, f, indent=1, default=lambda x: x.tolist() if hasattr(x, "tolist") else str(x))
    return 0


if __name__ == "__main__":
    sys.exit(main())
