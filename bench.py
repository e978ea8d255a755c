#!/usr/bin/env python
"""Louvain benchmark on one B200 (or N replicas under torchrun).

Workload (the single large graph of the reference's headline configuration): R-MAT scale
22, edge factor 16, (a, b, c, d) = (.57, .19, .19, .05), seed 1, symmetrised, deduplicated,
self-loops and isolated vertices removed: n = 2,395,745, m = 64,157,087 undirected edges
(128,314,174 CSR entries), unit weights, SORT rule, threshold 1e-3 (the reference's
MODULARITY_CONVERGED_THRESHOLD). One step = one complete Louvain run (every level until the
stop rule) on that graph.

  value : m / device seconds per run, CSR already resident in HBM (device buffers in, device
          buffer out) -- edges/s, higher is better
  e2e   : the same through the C ABI with pinned host buffers: the CSR is copied in and the
          communities copied out inside every timed run
  roofline: algorithmic bytes of the optimisation kernels (12 B per active entry + 24 B per
          active vertex, per pass) over their device time, against MEASURED_PEAKS.json hbm_gbs

`--impl reference` times the reference's algorithm on the host cores instead: the CPU
restatement in oracle/ (the reference itself is CUDA-only), with every host thread, on the
same graph.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
PKG = "louvain-fast-move-cuda_b200"

SCALE, EDGE_FACTOR, SEED = 22, 16, 1
WORKLOAD = "rmat_s22_ef16"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=int, default=SCALE)
    ap.add_argument("--mode", default="SORT", choices=["SORT", "HASH"])
    ap.add_argument("--cpu-sample-scale", type=int, default=19)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def build_graph(scale, device=None):
    import importlib
    graphs = importlib.import_module(PKG + ".graphs")
    u, v = graphs.rmat_pairs(scale, EDGE_FACTOR, seed=SEED)
    if device is not None:
        return graphs.to_device_canonical(u, v, device=device, name=f"rmat_s{scale}_ef{EDGE_FACTOR}")
    return graphs.canonical_from_pairs(u, v, name=f"rmat_s{scale}_ef{EDGE_FACTOR}")


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx.append(float(p[2]))
            except ValueError:
                continue
            for name, val in zip(names, p[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        torch.cuda.set_device(local)
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_sample(args):
    """The oracle, single-threaded, on a bounded sample of the workload: an R-MAT graph of
    the same generator at a smaller scale (about 10-30 s of CPU work)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    g = build_graph(args.cpu_sample_scale)
    t = time.perf_counter()
    o = O.Oracle(g, mode=O.SORT if args.mode == "SORT" else O.HASH, nthreads=1)
    o.louvain()
    dt = time.perf_counter() - t
    return {"value": g.m / dt, "unit": "edges/s", "cores": 1, "kind": "port",
            "sample": f"R-MAT scale {args.cpu_sample_scale} ef16 (n={g.n}, m={g.m}), one full "
                      f"Louvain run, oracle/louvain_oracle.c, 1 thread, {dt:.2f} s"}


def run_reference(args, world, rank):
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    g = build_graph(args.scale)
    threads = os.cpu_count() or 1
    mode = O.SORT if args.mode == "SORT" else O.HASH
    for _ in range(args.warmup):
        O.Oracle(g, mode=mode, nthreads=threads).louvain()
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        o = O.Oracle(g, mode=mode, nthreads=threads)
        o.louvain()
        times.append(time.perf_counter() - t)
    sec = sum(times) / len(times)
    value = g.m / sec
    line = {
        "impl": "reference", "metric": "louvain_edges_per_s", "value": value, "unit": "edges/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32/f32+f64",
        "data": "synthetic",
        "config": {"workload": f"rmat_s{args.scale}_ef16", "n": g.n, "m": g.m, "mode": args.mode,
                   "threshold": 1e-3},
        "cpu_baseline": {"value": value, "unit": "edges/s", "cores": threads, "kind": "port",
                         "sample": f"the full workload graph per step, oracle/louvain_oracle.c "
                                   f"with {threads} OpenMP threads (the reference has no CPU path)"},
        "e2e": {"value": value, "unit": "edges/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "modularity": o.modularity, "n_communities": o.n_best,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    world, rank, local = dist_setup(args.gpus)
    if args.impl == "reference":
        rc = run_reference(args, world, rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return rc

    import importlib
    import torch
    lv = importlib.import_module(PKG)
    dev = f"cuda:{local}"
    torch.cuda.set_device(local)
    g = build_graph(args.scale, device=dev)
    mode = lv.MODE.SORT if args.mode == "SORT" else lv.MODE.HASH
    eng = lv.Engine(local, mode=mode)

    row_d = torch.from_numpy(g.row_ptr).to(dev)
    col_d = torch.from_numpy(g.col).to(dev)
    out_d = torch.empty(g.n, dtype=torch.int32, device=dev)
    row_h = torch.from_numpy(g.row_ptr).pin_memory()
    col_h = torch.from_numpy(g.col).pin_memory()
    out_h = torch.empty(g.n, dtype=torch.int32).pin_memory()
    row_h_np, col_h_np, out_h_np = row_h.numpy(), col_h.numpy(), out_h.numpy()

    for _ in range(args.warmup):
        eng.run_csr(g.n, row_d, col_d, None, out=out_d)
    torch.cuda.synchronize()

    # device-resident runs (value)
    stats = []
    with ClockSampler(local) as clk:
        barrier(world)
        torch.cuda.synchronize()
        s_ev = torch.cuda.Event(enable_timing=True)
        e_ev = torch.cuda.Event(enable_timing=True)
        s_ev.record()
        wall0 = time.perf_counter()
        for _ in range(args.steps):
            _, q, st = eng.run_csr(g.n, row_d, col_d, None, out=out_d)
            stats.append(st)
        # the engine runs on its own stream and synchronises it before returning; the torch
        # events bracket the same region on the current stream after that synchronisation
        e_ev.record()
        torch.cuda.synchronize()
        wall = time.perf_counter() - wall0
        barrier(world)
    engine_ms = sum(s.ms_total for s in stats) / len(stats)   # engine-stream CUDA events
    ms_step = max_over_ranks(engine_ms, world)
    value = world * g.m / (ms_step / 1e3)

    # end-to-end through the C ABI with pinned host buffers
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        out_np, q_e2e, st_e2e = eng.run_csr(g.n, row_h_np, col_h_np, None, out=out_h_np)
    torch.cuda.synchronize()
    e2e_sec = max_over_ranks((time.perf_counter() - t0) / args.steps, world)
    barrier(world)

    st = stats[-1]
    peak, peak_kind = measured_peak()
    achieved = st.bytes_optimization / (st.ms_optimization_kernels / 1e3) / 1e9 if st.ms_optimization_kernels > 0 else 0.0
    line = {
        "metric": "louvain_edges_per_s", "value": value, "unit": "edges/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32 weights, f32 gains, f64 totals", "data": "synthetic",
        "config": {"workload": f"rmat_s{args.scale}_ef16", "n": g.n, "m": g.m, "mode": args.mode,
                   "threshold": 1e-3, "parallelism": "replicas" if world > 1 else "single",
                   "l2": "inputs larger than L2 (CSR 1.03 GB)"},
        "modularity": q, "n_communities": st.n_communities, "levels": st.levels,
        "passes": st.iterations,
        "window_ms": st.ms_window, "optimization_ms": st.ms_optimization,
        "aggregation_ms": st.ms_aggregation, "wall_ms_per_step": wall / args.steps * 1e3,
        "e2e": {"value": world * g.m / e2e_sec, "unit": "edges/s",
                "h2d_bytes_per_step": int(g.row_ptr.nbytes + g.col.nbytes),
                "d2h_bytes_per_step": int(g.n * 4), "ms_per_step": e2e_sec * 1e3,
                "modularity": q_e2e},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None,
                     "kernel": "optimisation kernels (binning + gain evaluation), all passes",
                     "bytes": st.bytes_optimization, "ms": st.ms_optimization_kernels,
                     "peak_source": peak_kind},
        "clocks": clk.summary(),
        "gpu_launches": int(sum(s.kernel_launches for s in stats)),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_sample(args)
    if rank == 0:
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
