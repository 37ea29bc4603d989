#!/usr/bin/env python
"""Benchmark of the multicut solve (one JSON line on stdout, rank 0).

Workload (default, --config c2): one PD-mode solve of the 3-D voxel grid
256x256x64 with 6-neighbour + long-range (+-4 x/y, +-2 z) edges, 24,805,376
edges, synthetic Beta(0.5,0.5) boundary probabilities (seed 1002).  A step is
one complete solve of that instance; `value` is edges/s over all ranks with
the input resident in HBM (300 MB, larger than the 126 MB L2), timed with CUDA
events on the launch stream; `e2e` runs the same solve through the C ABI's
host entry point (rama_solve_host: host arrays in, labels out).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config c1|c2|c2p|c3|c4]

--impl reference times the reference solver built from source for sm_100a
(oracle/_ref/librama_ref.so, its rama_cuda entry points) on the same
workload; the reference has no CPU code path.  The cpu_baseline of the default
arm is the project's CPU restatement (oracle/, single thread) on a bounded
sample of the same instance family, with a sequential GAEC timed beside it.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    "c1": dict(desc="2-D grid 64x64, PD", mode="PD"),
    "c2": dict(desc="3-D grid 256x256x64 + long range (+-4 x/y, +-2 z), PD", mode="PD"),
    "c2p": dict(desc="3-D grid 256x256x64 + long range (+-4 x/y, +-2 z), P", mode="P"),
    "c3": dict(desc="random geometric k-NN graph, 1M points, k=20, D (dual only)", mode="D"),
    "c4": dict(desc="512 Delaunay region-adjacency graphs, n log-uniform [500,20000], batched PD", mode="PD"),
    "c2s": dict(desc="3-D grid 64x64x32 + long range (profiling-size C2), PD", mode="PD"),
}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def make_instance(cfg):
    from rama_b200 import instances as I

    if cfg == "c1":
        return I.grid2d()
    if cfg in ("c2", "c2p"):
        return I.grid3d_longrange()
    if cfg == "c3":
        return I.knn_rgg()
    if cfg == "c2s":
        return I.grid3d_longrange(64, 64, 32, seed=1002)
    raise ValueError(cfg)


def cpu_sample(cfg):
    """A bounded sample of the same instance family for the CPU baseline."""
    from rama_b200 import instances as I

    if cfg in ("c2", "c2p"):
        return I.grid3d_longrange(128, 128, 64, seed=1002), "3-D grid 128x128x64 + long range, same generator"
    if cfg in ("c1", "c2s"):
        return make_instance(cfg), "full instance"
    if cfg == "c3":
        return I.knn_rgg(50_000, 20, seed=1003), "k-NN graph, 50k points, k=20, same generator"
    if cfg == "c4":
        b = I.delaunay_batch(count=64, seed=1004)
        return (b.i, b.j, b.c, b), "first 64 graphs of the same Delaunay batch generator"
    return I.grid2d(), "2-D grid 64x64"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during timing."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(5)
            except Exception:
                self.p.kill()

    def summary(self):
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for k, nm in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        busy = [x for x in sm if x > 0.5 * (mx or 1)] or sm
        return {"sm_mhz": statistics.median(busy) if busy else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(n_gpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("gloo", timeout=timedelta(seconds=600))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_ours(args, rank, world, local):
    import torch

    from rama_b200 import _lib
    from rama_b200.solver import Solver

    torch.cuda.set_device(local)
    cfg = args.config
    mode = CONFIGS[cfg]["mode"]
    if cfg == "c4":
        return run_ours_batch(args, rank, world, local)
    i, j, c = make_instance(cfg)
    E = len(c)
    dev = torch.device("cuda", local)
    d_i = torch.from_numpy(i).to(dev)
    d_j = torch.from_numpy(j).to(dev)
    d_c = torch.from_numpy(c).to(dev)
    N = int(max(i.max(), j.max())) + 1
    labels = torch.empty(N, dtype=torch.int32, device=dev)
    s = Solver(local)
    stream = torch.cuda.current_stream(dev)
    st = C.c_void_p(stream.cuda_stream)

    def one():
        return s.solve_device(d_i, d_j, d_c, mode=mode, labels=labels, stream=st, team=args.team)

    for _ in range(args.warmup):
        one()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    kernel_ms = []
    lbs = []
    with Clocks(local) as clk:
        barrier(world)
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            _, lb = one()
            lbs.append(lb)
            kernel_ms.append(s.stats().device_ms)
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
    ms = ev0.elapsed_time(ev1)
    ms_max = max_over_ranks(ms, world)
    stats = s.stats()
    obj = s.objective(d_i, d_j, d_c, labels[:N])
    # end to end through the host entry point (pinned host arrays in, labels out)
    h_i = torch.from_numpy(i).pin_memory()
    h_j = torch.from_numpy(j).pin_memory()
    h_c = torch.from_numpy(c).pin_memory()
    h_lab = torch.empty(N, dtype=torch.int32).pin_memory()
    o = _lib.options(mode)
    nl, lbv, sms = C.c_int64(0), C.c_double(0), C.c_double(0)
    e2e_t = []
    for k in range(max(1, min(args.steps, 3)) + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _lib.check(_lib.load().rama_solve_host(s.handle.h, C.c_void_p(h_i.data_ptr()), C.c_void_p(h_j.data_ptr()),
                                               C.c_void_p(h_c.data_ptr()), E, C.byref(o),
                                               C.c_void_p(h_lab.data_ptr()), N, C.byref(nl), C.byref(lbv),
                                               C.byref(sms)))
        if k > 0:
            e2e_t.append(time.perf_counter() - t0)
    e2e_s = max_over_ranks(statistics.median(e2e_t), world)
    if rank != 0:
        return None
    value = world * E * args.steps / (ms_max / 1e3)
    # roofline of the dominant kernel (the solve kernel): algorithmic bytes per
    # launch over the kernel's average device time
    hbm, src = peaks()
    alg = algorithmic_bytes(stats, E)
    kms = statistics.median(kernel_ms)
    achieved = alg / (kms / 1e3) / 1e9
    line = {
        "metric": "edges/s", "value": value, "unit": "edges/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (costs, messages) / f64 (bound, objective)",
        "data": "synthetic (seeded generator with the configuration's shapes and distributions)",
        "config": {"workload": CONFIGS[cfg]["desc"], "edges": E, "nodes": N, "mode": mode,
                   "parallelism": "replicas" if world > 1 else "single GPU",
                   "l2": "input 12 B/edge x %d edges > 126 MB L2" % E},
        "solves_per_s": world * args.steps / (ms_max / 1e3),
        "objective": obj, "lower_bound": lbs[-1], "rounds": stats.rounds, "team": stats.team,
        "phase_ms": {n: round(stats.phase_ms[k], 3) for k, n in enumerate(_lib.PHASES) if n != "-"},
        "e2e": {"value": world * E / e2e_s, "unit": "edges/s", "h2d_bytes_per_step": 12 * E,
                "d2h_bytes_per_step": 4 * N + 8, "api": "rama_solve_host"},
        "gpu_launches": args.steps,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": None, "peak_source": src, "kernel": "k_solve_grid" if stats.team == 2 else "k_solve_cta",
                     "kernel_ms": kms, "algorithmic_bytes": alg},
        "clocks": clk.summary(),
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(cfg, mode)
    return line


def algorithmic_bytes(stats, E):
    """Lower-bound bytes a solve must move: read the edges once per contraction
    round and write the coarsened list (12 B/edge read + 8 B/edge map gathers
    + 12 B/edge written), matching reads the doubled edge list (12 B per arc),
    and the dual reads/writes triangle and edge state per message-passing
    iteration.  Sorting passes and temporaries are overhead, not work."""
    # the device reports the counts it processed (see rama_stats)
    b = getattr(stats, "alg_bytes", 0)
    if b:
        return float(b)
    return float(E) * (12 + 8 + 12 + 24)


def run_ours_batch(args, rank, world, local):
    """512 Delaunay graphs per rank (seed 1004 + rank), one batched launch per
    step; instances are independent, so ranks share nothing (weak scaling)."""
    import torch

    from rama_b200 import instances as I
    from rama_b200.solver import Solver

    batch = I.delaunay_batch(seed=1004 + rank)
    dev = torch.device("cuda", local)
    d_i = torch.from_numpy(batch.i).to(dev)
    d_j = torch.from_numpy(batch.j).to(dev)
    d_c = torch.from_numpy(batch.c).to(dev)
    lo = np.zeros(batch.count + 1, np.int64)
    lo[1:] = np.cumsum(batch.node_counts)
    d_lab = torch.empty(int(lo[-1]), dtype=torch.int32, device=dev)
    s = Solver(local)
    stream = torch.cuda.current_stream(dev)
    st = C.c_void_p(stream.cuda_stream)
    E = int(batch.edge_offsets[-1])

    def one():
        _, _, lbs, codes, rc = s.solve_batch_device(d_i, d_j, d_c, batch.edge_offsets, lo, mode="PD", d_labels=d_lab,
                                                    stream=st)
        assert rc == 0, rc
        return lbs

    for _ in range(args.warmup):
        one()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        barrier(world)
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            one()
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
    ms = max_over_ranks(ev0.elapsed_time(ev1), world)
    stats = s.stats()
    # the plain form: one instance per launch (each on its own team choice)
    t0 = time.perf_counter()
    plain_ms = 0.0
    for k in range(batch.count):
        a, b = batch.edge_offsets[k], batch.edge_offsets[k + 1]
        s.solve_device(d_i[a:b], d_j[a:b], d_c[a:b], mode="PD", labels=d_lab[lo[k]:lo[k + 1]], stream=st)
        plain_ms += s.stats().device_ms
    torch.cuda.synchronize()
    plain_wall = time.perf_counter() - t0
    if rank != 0:
        return None
    hbm, src = peaks()
    achieved = float(stats.alg_bytes) / (stats.device_ms / 1e3) / 1e9 if stats.device_ms else 0.0
    value = world * E * args.steps / (ms / 1e3)
    return {
        "metric": "edges/s", "value": value, "unit": "edges/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (costs, messages) / f64 (bound, objective)", "data": "synthetic",
        "config": {"workload": CONFIGS["c4"]["desc"], "instances": batch.count, "edges": E,
                   "parallelism": "instances dealt to CTAs, largest first; ranks hold separate batches"},
        "solves_per_s": world * batch.count * args.steps / (ms / 1e3),
        "plain": {"value": E / (plain_ms / 1e3), "unit": "edges/s", "device_ms": plain_ms, "wall_s": plain_wall,
                  "form": "one instance per launch"},
        "gpu_launches": args.steps,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": None, "peak_source": src, "kernel": "k_solve_cta", "kernel_ms": stats.device_ms,
                     "algorithmic_bytes": float(stats.alg_bytes)},
        "clocks": clk.summary(),
    }


def cpu_baseline(cfg, mode):
    from oracle import oracle_py as O

    sample, desc = cpu_sample(cfg)
    if len(sample) == 4:  # a batch: solve the instances one after the other
        b = sample[3]
        insts = [b.instance(k) for k in range(b.count)]
    else:
        insts = [sample]
    i, j, c = sample[0], sample[1], sample[2]
    t0 = time.perf_counter()
    for (ii, jj, cc) in insts:
        lab, lb, _ = O.solve(ii, jj, cc, mode)
    t1 = time.perf_counter()
    t2 = time.perf_counter()
    for (ii, jj, cc) in insts:
        glab = O.gaec(ii, jj, cc)
    t3 = time.perf_counter()
    i, j, c = insts[-1]
    return {"value": len(c) / (t1 - t0), "unit": "edges/s", "cores": 1, "kind": "port",
            "sample": f"{desc}: {len(c)} edges, mode {mode}, oracle restatement of the RAMA solve, "
                      f"{t1 - t0:.2f} s",
            "gaec": {"value": len(c) / (t3 - t2), "unit": "edges/s", "cores": 1,
                     "objective": O.objective(i, j, c, glab), "rama_oracle_objective": O.objective(i, j, c, lab)},
            "host_cores": os.cpu_count()}


def run_reference(args, rank, world, local):
    if rank != 0:
        return None
    from oracle import ref_py as R

    if not R.available():
        return {"impl": "reference", "unavailable": "oracle/_ref/librama_ref.so not built"}
    import torch

    torch.cuda.set_device(local)
    cfg = args.config
    mode = CONFIGS[cfg]["mode"]
    i, j, c = make_instance(cfg)
    E = len(c)
    N = int(max(i.max(), j.max())) + 1
    dev = torch.device("cuda", local)
    d_i = torch.from_numpy(i).to(dev)
    d_j = torch.from_numpy(j).to(dev)
    d_c = torch.from_numpy(c).to(dev)
    lab = torch.empty(N, dtype=torch.int32, device=dev)

    def one():
        return R.rama_device(C.c_void_p(d_i.data_ptr()), C.c_void_p(d_j.data_ptr()), C.c_void_p(d_c.data_ptr()), E,
                             C.c_void_p(lab.data_ptr()), N, mode)

    for _ in range(args.warmup):
        one()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    lbv = None
    with Clocks(local) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            _, lbv = one()
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    e2e = []
    for k in range(2):
        t0 = time.perf_counter()
        R.rama(i, j, c, mode)
        if k > 0:
            e2e.append(time.perf_counter() - t0)
    from oracle import oracle_py as O

    obj = O.objective(i, j, c, lab.cpu().numpy()) if not CONFIGS[cfg]["mode"] == "D" else None
    value = E * args.steps / (ms / 1e3)
    return {
        "impl": "reference", "metric": "edges/s", "value": value, "unit": "edges/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": CONFIGS[cfg]["desc"], "edges": E, "nodes": N, "mode": mode},
        "objective": obj, "lower_bound": lbv,
        "e2e": {"value": E / statistics.median(e2e), "unit": "edges/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "cpu_baseline": {"value": value, "unit": "edges/s", "cores": 0, "kind": "reference",
                         "sample": "the reference solver itself (built from source for sm_100a into oracle/_ref) "
                                   "on the full workload; it runs on the GPU -- the reference has no CPU path"},
        "clocks": clk.summary(),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2", choices=sorted(CONFIGS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--team", type=int, default=0, help="0 auto, 1 one CTA, 2 cooperative grid")
    args = ap.parse_args()
    rank, world, local = dist_setup(args.gpus)
    if args.impl == "reference":
        line = run_reference(args, rank, world, local)
    else:
        line = run_ours(args, rank, world, local)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    sys.stdout.flush()
    os._exit(0)


if __name__ == "__main__":
    main()
