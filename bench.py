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
                    [--config c1|c2|c2p|c3|c4|c5] [--requests R] [--rates 100,1000,5000]

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
    "c4s": dict(desc="64 Delaunay region-adjacency graphs of the C4 generator (profiling size), batched PD",
                mode="PD"),
    "c5": dict(desc="served: Poisson arrivals of grids 16^3..128^3, Delaunay 1e3..2e6 edges, k-NN (k=10) "
                    "1e4..5e5 nodes; modes P/PD/D 50/40/10%", mode="mixed"),
}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) of one solve
# launch per input edge, from one ncu capture of a profiling-size case of the
# same generator; the full instances are too large to capture under replay,
# so the traffic is scaled by edge count (the algorithmic bytes per edge of
# the two sizes are close: see roofline.algorithmic_bytes).
#   C2 (k_solve_grid), 3-D grid 64x64x32 + long range, 753,664 edges, PD:
#     335,417,600 B read + 1,157,507,584 B written;
#   C4 (k_solve_mixed), 64 Delaunay graphs of the C4 generator, 1,048,829
#     edges, PD: 407,300,096 B read + 1,957,661,440 B written.
# Commands: ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum,gpu__time_duration.sum
#   --clock-control none -k regex:k_solve_grid -s 1 -c 1
#   python bench.py --config c2s --steps 2 --warmup 1 --no-cpu-baseline --no-tune
# (and -k regex:k_solve_ -s 1 -c 2 ... --config c4s --steps 3 --warmup 3 for C4)
TRAFFIC_B_PER_EDGE = {("c2", "PD"): (335417600 + 1157507584) / 753664,
                      ("c2s", "PD"): (335417600 + 1157507584) / 753664,
                      ("c4", "PD"): (407300096 + 1957661440) / 1048829,
                      ("c4s", "PD"): (407300096 + 1957661440) / 1048829}


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


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


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
    if cfg in ("c4", "c4s"):
        return run_ours_batch(args, rank, world, local)
    if cfg == "c5":
        return run_ours_served(args, rank, world, local)
    i, j, c = make_instance(cfg)
    E = len(c)
    dev = torch.device("cuda", local)
    d_i = torch.from_numpy(i).to(dev)
    d_j = torch.from_numpy(j).to(dev)
    d_c = torch.from_numpy(c).to(dev)
    N = int(max(i.max(), j.max())) + 1
    labels = torch.empty(N, dtype=torch.int32, device=dev)
    s = Solver(local)
    tuning = tune_solver(s, local, args)
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
    # launch (tallied on the device, see algorithmic_bytes) over the kernel's
    # average device time
    hbm, src = peaks()
    alg = algorithmic_bytes(stats, E)
    kms = statistics.median(kernel_ms)
    achieved = alg / (kms / 1e3) / 1e9
    tpe = TRAFFIC_B_PER_EDGE.get((cfg, mode)) if stats.team == 2 else None
    traffic = tpe * E if tpe else None
    phases = phase_roofline(stats, hbm)
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
                     "traffic": traffic, "peak_source": src, "kernel": KERNEL_OF_TEAM.get(stats.team, "?"),
                     "kernel_ms": kms, "algorithmic_bytes": alg, "phases": phases},
        "clocks": clk.summary(),
        "tuning": tuning,
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(cfg, mode)
        if "fp64_error" in line["cpu_baseline"]:
            line["lb_error_vs_fp64"] = line["cpu_baseline"]["fp64_error"]
    return line


KERNEL_OF_TEAM = {1: "k_solve_cta", 2: "k_solve_grid", 3: "k_solve_mixed"}


def phase_roofline(stats, hbm):
    """Per phase of the last solve: device time, algorithmic bytes (tallied
    on the device), achieved GB/s and the fraction of the HBM peak."""
    from rama_b200 import _lib

    out = {}
    for k, name in enumerate(_lib.PHASES):
        ms, b = float(stats.phase_ms[k]), float(stats.phase_bytes[k])
        if name == "-" or (ms == 0.0 and b == 0.0):
            continue
        gbs = b / (ms / 1e3) / 1e9 if ms > 0 else 0.0
        out[name] = {"ms": round(ms, 3), "bytes": b, "gbs": round(gbs, 1), "frac": round(gbs / hbm, 4)}
    # a step's bytes are tallied where the step ends, its time in the
    # sub-phases it marks: the steps as a whole carry the meaningful rates
    groups = {}
    for step, parts in PHASE_GROUPS.items():
        ms = sum(out[p]["ms"] for p in parts if p in out)
        b = sum(out[p]["bytes"] for p in parts if p in out)
        if ms > 0:
            gbs = b / (ms / 1e3) / 1e9
            groups[step] = {"ms": round(ms, 3), "bytes": b, "gbs": round(gbs, 1), "frac": round(gbs / hbm, 4)}
    out["steps"] = groups
    return out


PHASE_GROUPS = {
    "init": ("init",),
    "cycle search": ("cycles", "csr", "cyc_search"),
    "message passing": ("mp_norm", "mp_chords", "mp_incid", "mp_build", "mp_iter", "dual_commit"),
    "matching": ("matching", "match_first", "match_iter", "match_labels"),
    "forest": ("woc_msf", "woc_csr", "woc_checks", "woc_root", "woc_paths", "woc"),
    "contraction": ("contract", "csort_big", "csort_slot", "csort_scatter", "csort_rank", "contract_runs"),
}


def tune_solver(s, device, args):
    """Launch parameters from the project's autotuner (rama_b200.autotune):
    the cached choices for this device, tuned first when there are none.
    None of them changes a result."""
    if args.no_tune:
        return {"source": "built-in defaults", "tuning": s.handle.tuning().as_dict()}
    from rama_b200 import autotune

    entry = autotune.ensure(device, budget_s=args.tune_budget)
    autotune.apply(s.handle, device)
    return {"source": entry["source"], "tuning": entry["tuning"], "default": entry["default"],
            "tuning_s": entry.get("seconds")}


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

    batch = I.delaunay_batch(count=64 if args.config == "c4s" else 512, seed=1004 + rank)
    dev = torch.device("cuda", local)
    d_i = torch.from_numpy(batch.i).to(dev)
    d_j = torch.from_numpy(batch.j).to(dev)
    d_c = torch.from_numpy(batch.c).to(dev)
    lo = np.zeros(batch.count + 1, np.int64)
    lo[1:] = np.cumsum(batch.node_counts)
    d_lab = torch.empty(int(lo[-1]), dtype=torch.int32, device=dev)
    s = Solver(local)
    tuning = tune_solver(s, local, args)
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
    tpe = TRAFFIC_B_PER_EDGE.get((args.config, "PD"))
    return {
        "metric": "edges/s", "value": value, "unit": "edges/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (costs, messages) / f64 (bound, objective)", "data": "synthetic",
        "config": {"workload": CONFIGS[args.config]["desc"], "instances": batch.count, "edges": E,
                   "parallelism": "instances dealt to CTAs, largest first; ranks hold separate batches"},
        "solves_per_s": world * batch.count * args.steps / (ms / 1e3),
        "plain": {"value": E / (plain_ms / 1e3), "unit": "edges/s", "device_ms": plain_ms, "wall_s": plain_wall,
                  "form": "one instance per launch"},
        "gpu_launches": args.steps,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": tpe * E if tpe else None, "peak_source": src,
                     "kernel": "k_solve_mixed / k_solve_cta", "kernel_ms": stats.device_ms,
                     "algorithmic_bytes": float(stats.alg_bytes)},
        "clocks": clk.summary(),
        "tuning": tuning,
    }


def run_ours_served(args, rank, world, local):
    """Continuous batching of a Poisson request stream (rama_b200.server).

    A pool of distinct request graphs (seeded, the served mix's kinds and size
    ranges, pinned in host memory) stands in for the clients; each request of
    the stream is a pool graph with its own mode.  Per arrival rate the server
    serves `--requests` requests in real time: every request's graph is copied
    host -> device when its lane admits it and its labels come back to the
    host, so the numbers are end to end.  `value` = edges/s at the highest
    rate; `plain` = the same requests solved one at a time (each alone on its
    automatic team) on a bounded sample.  Ranks serve separate streams."""
    import torch

    from rama_b200 import instances as I
    from rama_b200 import server as S
    from rama_b200.solver import Solver

    rates = [float(x) for x in args.rates.split(",")]
    t_gen = time.perf_counter()
    pool = I.served_pool(size=args.pool, seed=1005 + rank)
    pinned = [tuple(torch.from_numpy(np.ascontiguousarray(x)).pin_memory() for x in g) for g in pool]
    nodes = [int(max(g[0].max(), g[1].max())) + 1 for g in pool]
    gen_s = time.perf_counter() - t_gen
    tsolver = Solver(local)
    tuning = tune_solver(tsolver, local, args)
    srv = S.Server(device=local, lanes=args.lanes, lane_bytes=args.lane_gb << 30, max_batch=256,
                   tuning=tsolver.handle.tuning())
    # warm-up: every pool graph once, all queued at once
    warm = [S.Request(k, *pinned[k], mode="PD", num_nodes=nodes[k]) for k in range(len(pool))]
    for _ in range(max(1, args.warmup // 3)):
        srv.serve(warm, realtime=False)
    per_rate = []
    lanes_alg0 = sum(ln.alg_bytes for ln in srv.lanes)
    with Clocks(local) as clk:
        for rate in rates:
            stream = I.served_stream(num_requests=args.requests, rate=rate, pool_size=len(pool), seed=1006 + rank)
            reqs = [S.Request(k, *pinned[p], mode=m, arrival=t, num_nodes=nodes[p]) for k, (t, m, p) in
                    enumerate(stream)]
            barrier(world)
            st = srv.serve(reqs, realtime=True)
            bad = sum(r.status != 0 for r in reqs)
            summ = st.summary()
            summ.update(rate_per_s=rate, failed=bad, h2d_bytes=int(sum(12 * r.num_edges for r in reqs)),
                        d2h_bytes=int(sum(4 * r.num_nodes for r in reqs)))
            per_rate.append(summ)
    alg = sum(ln.alg_bytes for ln in srv.lanes) - lanes_alg0
    busy_s = sum(x["wall_s"] for x in per_rate)
    srv.close()
    # plain form: the first requests of the last stream, one solve at a time
    s = Solver(local)
    sample = reqs[: min(len(reqs), args.plain_sample)]
    plain_ms, plain_edges = 0.0, 0
    for r in sample:
        d = [x.to(torch.device("cuda", local), non_blocking=True) for x in (r.i, r.j, r.c)]
        s.solve_device(*d, mode=r.mode)
        torch.cuda.synchronize()
        plain_ms += s.stats().device_ms
        plain_edges += r.num_edges
    if rank != 0:
        return None
    top = per_rate[-1]
    hbm, src = peaks()
    achieved = alg / busy_s / 1e9 if busy_s else 0.0
    value = world * top["edges_per_s"]
    return {
        "metric": "edges/s", "value": value, "unit": "edges/s", "n_gpus": world, "steps": len(rates),
        "warmup": args.warmup, "ms_per_step": top["wall_s"] * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (costs, messages) / f64 (bound, objective)",
        "data": "synthetic (seeded pool of request graphs with the served mix's kinds and size ranges)",
        "config": {"workload": CONFIGS["c5"]["desc"], "requests_per_rate": args.requests, "rates_per_s": rates,
                   "pool_graphs": len(pool), "pool_edges": int(sum(len(g[2]) for g in pool)),
                   "lanes": args.lanes, "lane_bytes": args.lane_gb << 30, "solo_min_edges": srv.solo_min_edges,
                   "parallelism": "continuous batching: lanes = handle + stream + fixed HBM budget; requests of "
                                  "solo_min_edges or more alone on the whole GPU, the rest batched on clusters "
                                  "or one CTA each"},
        "solves_per_s": world * top["solves_per_s"],
        "served": per_rate,
        "plain": {"value": plain_edges / (plain_ms / 1e3) if plain_ms else 0.0, "unit": "edges/s",
                  "solves_per_s": len(sample) / (plain_ms / 1e3) if plain_ms else 0.0, "requests": len(sample),
                  "device_ms": plain_ms, "form": "one request per launch, device time only"},
        "e2e": {"value": value, "unit": "edges/s", "h2d_bytes_per_step": top["h2d_bytes"],
                "d2h_bytes_per_step": top["d2h_bytes"], "api": "rama_b200.server.Server.serve"},
        "gpu_launches": int(sum(x["batches"] for x in per_rate)),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": None, "peak_source": src, "kernel": "k_solve_mixed / k_solve_cta",
                     "algorithmic_bytes": alg, "note": "algorithmic bytes of all served batches / served wall time"},
        "pool_generation_s": gen_s,
        "clocks": clk.summary(),
        "tuning": tuning,
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
    edges = sum(len(x[2]) for x in insts)
    i, j, c = insts[-1]
    gaec_obj = O.objective(i, j, c, glab)
    rama_obj = O.objective(i, j, c, lab)
    return {"value": edges / (t1 - t0), "unit": "edges/s", "cores": 1, "kind": "port",
            "sample": f"{desc}: {edges} edges, mode {mode}, oracle restatement of the RAMA solve, "
                      f"{t1 - t0:.2f} s",
            "gaec_value": edges / (t3 - t2), "gaec_objective": gaec_obj, "rama_oracle_objective": rama_obj,
            "gaec": {"value": edges / (t3 - t2), "unit": "edges/s", "cores": 1,
                     "what": "project-written sequential greedy additive edge contraction + union-find",
                     "objective": gaec_obj, "rama_oracle_objective": rama_obj},
            "cpu_model": cpu_model(), "host_cores": os.cpu_count(),
            **({"fp64_error": fp64_error(O, i, j, c)} if mode == "D" else {})}


def fp64_error(O, i, j, c):
    """Error of the bound against the FP64 oracle on the sample: the same
    triangle selection with every cost, message and bound in double.  The GPU
    solve of the sample runs through the C ABI like the timed solves."""
    from rama_b200.solver import Solver

    t0 = time.perf_counter()
    lb64 = O.dual_lb_f64(i, j, c, "D")
    t1 = time.perf_counter()
    _, lb_gpu, _ = Solver(0).solve(i, j, c, mode="D")
    return {"edges": len(c), "lb_gpu": lb_gpu, "lb_fp64": lb64, "abs": abs(lb_gpu - lb64),
            "rel": abs(lb_gpu - lb64) / max(1.0, abs(lb64)), "fp64_oracle_s": round(t1 - t0, 2),
            "what": "GPU: FP32 messages, compensated FP64 bound; oracle: all FP64, same triangle selection"}


def run_reference_many(args, local, R):
    """Reference arm of the batched (c4) and served (c5) configs: the reference
    has no batch or serving API, so its form is one rama_cuda call per
    instance; a bounded sample of the same instances is timed with CUDA
    events around each call."""
    import torch

    from rama_b200 import instances as I

    cfg = args.config
    if cfg == "c4":
        batch = I.delaunay_batch(seed=1004)
        insts = [(batch.instance(k), "PD") for k in range(batch.count)]
        sample = insts[: args.ref_sample]
        what = "the first %d of the 512 Delaunay graphs, PD, one rama_cuda call each" % len(sample)
    else:
        pool = I.served_pool(size=args.pool, seed=1005)
        stream = I.served_stream(num_requests=args.requests, rate=1000.0, pool_size=len(pool), seed=1006)
        sample = [(pool[p], m) for (_, m, p) in stream[: args.ref_sample]]
        what = "the first %d requests of the served stream, one rama_cuda call each" % len(sample)
    dev = torch.device("cuda", local)
    stream_ = torch.cuda.current_stream(dev)
    times, edges = [], 0
    with Clocks(local) as clk:
        for w, ((i, j, c), mode) in enumerate(sample[: args.warmup] + sample):
            E = len(c)
            N = int(max(i.max(), j.max())) + 1
            d_i, d_j, d_c = (torch.from_numpy(np.ascontiguousarray(x)).to(dev) for x in (i, j, c))
            lab = torch.empty(N, dtype=torch.int32, device=dev)
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            ev0.record(stream_)
            R.rama_device(C.c_void_p(d_i.data_ptr()), C.c_void_p(d_j.data_ptr()), C.c_void_p(d_c.data_ptr()), E,
                          C.c_void_p(lab.data_ptr()), N, mode)
            ev1.record(stream_)
            torch.cuda.synchronize()
            if w >= args.warmup:
                times.append(ev0.elapsed_time(ev1))
                edges += E
    tot_s = sum(times) / 1e3
    value = edges / tot_s
    lat = np.asarray(times)
    # end to end through the reference's host overload (host arrays in, labels
    # out: 12 B per edge in, 4 B per node out)
    e2e_s, h2d, d2h = 0.0, 0, 0
    for (i, j, c), mode in sample:
        t0 = time.perf_counter()
        lab_h, _, _ = R.rama(i, j, c, mode)
        e2e_s += time.perf_counter() - t0
        h2d += 12 * len(c)
        d2h += 4 * len(lab_h)
    return {
        "impl": "reference", "metric": "edges/s", "value": value, "unit": "edges/s", "n_gpus": 1,
        "steps": len(times), "warmup": args.warmup, "ms_per_step": float(lat.mean()), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": CONFIGS[cfg]["desc"], "sample": what, "edges": edges},
        "solves_per_s": len(times) / tot_s, "p50_ms": float(np.percentile(lat, 50)),
        "p99_ms": float(np.percentile(lat, 99)),
        "e2e": {"value": edges / e2e_s, "unit": "edges/s", "h2d_bytes_per_step": h2d // max(1, len(times)),
                "d2h_bytes_per_step": d2h // max(1, len(times)),
                "api": "rama_cuda(const std::vector<int>&, ...) host overload, one call per instance"},
        "cpu_baseline": {"value": value, "unit": "edges/s", "cores": 0, "kind": "reference",
                         "sample": what + " (the reference solver built from source for sm_100a; it has no CPU "
                                          "path)"},
        "clocks": clk.summary(),
    }


def run_reference(args, rank, world, local):
    if rank != 0:
        return None
    from oracle import ref_py as R

    if not R.available():
        return {"impl": "reference", "unavailable": "oracle/_ref/librama_ref.so not built"}
    import torch

    torch.cuda.set_device(local)
    if args.config in ("c4", "c5"):
        return run_reference_many(args, local, R)
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
        "e2e": {"value": E / statistics.median(e2e), "unit": "edges/s", "h2d_bytes_per_step": 12 * E,
                "d2h_bytes_per_step": 4 * N, "api": "rama_cuda(const std::vector<int>&, ...) host overload"},
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
    ap.add_argument("--team", type=int, default=0, help="0 auto, 1 one CTA, 2 cooperative grid, 3 cluster")
    ap.add_argument("--requests", type=int, default=2000, help="c5: requests per arrival rate")
    ap.add_argument("--rates", default="100,1000,5000", help="c5: arrival rates per second")
    ap.add_argument("--pool", type=int, default=32, help="c5: distinct request graphs")
    ap.add_argument("--lanes", type=int, default=12, help="c5: server lanes")
    ap.add_argument("--lane-gb", type=int, default=8, help="c5: HBM budget per lane (GiB)")
    ap.add_argument("--plain-sample", type=int, default=200, help="c5: requests solved one at a time")
    ap.add_argument("--ref-sample", type=int, default=64, help="c4/c5 reference arm: instances timed")
    ap.add_argument("--no-tune", action="store_true", help="keep the built-in launch parameters")
    ap.add_argument("--tune-budget", type=float, default=45.0, help="seconds of autotuning trials when uncached")
    args = ap.parse_args()
    if args.config == "c5":
        # lanes overlap only when each stream has its own hardware queue
        os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", str(max(8, args.lanes)))
    rank, world, local = dist_setup(args.gpus)
    if args.impl == "reference":
        line = run_reference(args, rank, world, local)
    else:
        line = run_ours(args, rank, world, local)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    # the JSON line stays the last line on stdout: what prints at exit (the
    # reference's timers report from its static destructors) goes to stderr
    sys.stdout.flush()
    os.dup2(sys.stderr.fileno(), sys.stdout.fileno())
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    sys.stdout.flush()


if __name__ == "__main__":
    main()
