"""Autotuner of the solver's launch parameters (rama_tuning).

    python -m rama_b200.autotune [--device D] [--budget SECONDS] [--force]

The solver computes the same result on every execution team -- one CTA, a
thread-block cluster of 2 to 16 CTAs, or the whole GPU -- so the choice of
team and of its size only decides how fast a solve runs.  The handle's
built-in choices are guesses; this module measures them on the device:

* grid_ctas_per_sm, grid_small_ctas_per_sm, grid_small_max: CTAs per SM of
  the whole-GPU solve, for large graphs and for graphs below a size (fewer
  CTAs take cheaper grid barriers, more CTAs hide more memory latency), timed
  on 3-D grids of growing size;
* cluster_ctas: the cluster size, timed on mid-size Delaunay graphs, and
  again (against the built-in size) inside the batch trial below, which has
  the last word: a batch runs many clusters side by side;
* single_cluster_min / single_grid_min: where a single solve moves from one
  CTA to a cluster and from a cluster to the whole GPU -- each team is timed
  on graphs of increasing size and the switch goes to the first size at which
  the larger team wins;
* batch_cluster_min / batch_cluster_share / cta_threads: which instances of
  a batch get a cluster, and whether the instances solved alone take CTAs of
  512 threads (two per SM) or 256 (three per SM), timed together on a batch
  of 256 Delaunay graphs of uneven size.

Every trial solve's labels and bound are checked to equal the first trial's:
a tuning never changes a result, and the tuner fails loudly if one would.

The choices are cached per device (GPU name, SM count, library build) in a
JSON file: $RAMA_TUNE_CACHE, else ~/.cache/rama_b200/tuning.json.
`apply(handle)` sets the cached choices on a handle; `ensure(device)` tunes
first when the cache has none for this device.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import time
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from . import instances as I

KNOBS = ("grid_ctas_per_sm", "grid_small_ctas_per_sm", "grid_small_max", "cluster_ctas", "single_cluster_min",
         "single_grid_min", "batch_cluster_min", "batch_cluster_share", "cta_threads")


def cache_path() -> str:
    p = os.environ.get("RAMA_TUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "rama_b200", "tuning.json")


def device_key(device: int = 0) -> str:
    """GPU name, SM count and a digest of the built library: a rebuilt solver
    is tuned again."""
    import torch

    p = torch.cuda.get_device_properties(device)
    h = hashlib.sha1()
    with open(_lib.LIB_PATH, "rb") as f:
        for chunk in iter(lambda: f.read(1 << 20), b""):
            h.update(chunk)
    return f"{p.name}|{p.multi_processor_count}|{h.hexdigest()[:16]}"


def load_cache(path: Optional[str] = None) -> Dict[str, dict]:
    path = path or cache_path()
    try:
        with open(path) as f:
            d = json.load(f)
        return d if isinstance(d, dict) else {}
    except (OSError, ValueError):
        return {}


def save_cache(entry_key: str, entry: dict, path: Optional[str] = None) -> None:
    path = path or cache_path()
    d = load_cache(path)
    d[entry_key] = entry
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    # one temporary per process: ranks tuning at the same time replace the
    # file whole, never a half-written one
    tmp = "%s.%d.tmp" % (path, os.getpid())
    with open(tmp, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


# ---------------------------------------------------------------------------
# decisions from timing tables (pure functions; tested on the CPU)
# ---------------------------------------------------------------------------
def pick_fastest(times: Dict[object, float]):
    """The option with the smallest time; ties go to the first listed."""
    best = None
    for k, v in times.items():
        if best is None or v < times[best]:
            best = k
    return best


def crossover(sizes: Sequence[int], small_team: Sequence[float], large_team: Sequence[float],
              default: int) -> int:
    """Edge count from which the larger team should run a single solve: the
    first measured size at which it is faster and stays faster at every larger
    size (a size between the last loss and that win), or `default` when the
    measurements never cross, or one past the largest size when the larger
    team never wins."""
    n = len(sizes)
    assert n == len(small_team) == len(large_team) and n > 0
    wins = [l < s for s, l in zip(small_team, large_team)]
    if all(wins):
        return int(sizes[0])
    if not any(wins):
        return int(sizes[-1]) + 1
    k = n
    while k > 0 and wins[k - 1]:
        k -= 1
    if k == n:
        return default
    # switch halfway (geometrically) between the last size the small team won
    # and the first size of the larger team's unbroken run of wins
    return int(round(float(np.sqrt(float(sizes[k - 1]) * float(sizes[k])))))


# ---------------------------------------------------------------------------
# measurement
# ---------------------------------------------------------------------------
class _Trial:
    """Times solves on one handle with a given tuning and checks each result
    against the first one seen for the same instance."""

    def __init__(self, device: int):
        import torch

        from .solver import Solver

        self.torch = torch
        self.solver = Solver(device)
        self.base = self.solver.handle.tuning()
        self.ref: Dict[object, Tuple[np.ndarray, float]] = {}

    def set(self, **kw):
        t = _lib.RamaTuning()
        for k in KNOBS:
            setattr(t, k, kw.get(k, getattr(self.base, k)))
        self.solver.handle.set_tuning(t)

    def solve(self, key: str, inst, mode: str, team: int, reps: int = 3) -> float:
        """Median device time (ms) of `reps` solves after one warm-up."""
        d = [self.torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in inst]
        ms = []
        for r in range(reps + 1):
            lab, lb = self.solver.solve_device(*d, mode=mode, team=team)
            if r > 0:
                ms.append(self.solver.stats().device_ms)
        self._check(key, lab.cpu().numpy(), lb)
        return float(np.median(ms))

    def batch(self, key: str, batch, mode: str, reps: int = 2) -> float:
        ms = []
        for r in range(reps + 1):
            res, status, rc = self.solver.solve_batch(batch, mode=mode)
            _lib.check(rc)
            if r > 0:
                ms.append(self.solver.stats().device_ms)
        for k, (lab, lb) in enumerate(res):
            self._check((key, k), np.asarray(lab), lb)
        return float(np.median(ms))

    def _check(self, key, lab, lb):
        if key not in self.ref:
            self.ref[key] = (lab, lb)
            return
        rlab, rlb = self.ref[key]
        if not (np.array_equal(rlab, lab) and rlb == lb):
            raise AssertionError(f"a launch parameter changed the result of {key}: the solver is not team-independent")


def tune(device: int = 0, budget_s: float = 60.0, quick: bool = False) -> dict:
    """Measures every knob on this device; returns the chosen tuning plus the
    timing tables it came from."""
    t0 = time.perf_counter()
    tr = _Trial(device)
    base = tr.base.as_dict()
    rng = np.random.default_rng(2024)
    tables: dict = {}
    chosen = dict(base)

    # whole-GPU solves: CTAs per SM, on 3-D grids of growing size (fewer
    # CTAs take cheaper grid barriers, which pays on smaller graphs; more
    # CTAs keep more memory traffic in flight, which pays on larger ones)
    dims = [(48, 48, 24), (96, 96, 48), (160, 160, 64)] if not quick else [(32, 32, 16), (64, 64, 32)]
    opts = list(range(1, int(base["grid_ctas_per_sm"]) + 1))
    gsizes, gt = [], {g: [] for g in opts}
    for k, (nx, ny, nz) in enumerate(dims):
        inst = I.grid3d_longrange(nx, ny, nz, seed=7)
        gsizes.append(len(inst[2]))
        for g in opts:
            tr.set(grid_ctas_per_sm=g, grid_small_ctas_per_sm=g, grid_small_max=0)
            gt[g].append(tr.solve("grid%d" % k, inst, "PD", team=2))
    large = pick_fastest({g: gt[g][-1] for g in opts})
    small = pick_fastest({g: gt[g][0] for g in opts})
    chosen["grid_ctas_per_sm"] = large
    chosen["grid_small_ctas_per_sm"] = small
    chosen["grid_small_max"] = 0 if small == large else crossover(gsizes, gt[small], gt[large], 0)
    tables["grid"] = {"edges": gsizes, **{"ctas_per_sm_%d_ms" % g: gt[g] for g in opts}}
    tr.set(**chosen)

    # cluster size on mid-size graphs
    mids = [I.delaunay(n, rng) for n in ((6000, 20000) if not quick else (3000,))]
    tc = {}
    for csz in (4, 8, 16):
        try:
            tr.set(**{**chosen, "cluster_ctas": csz})
        except _lib.RamaError:
            continue  # this cluster size does not fit on the device
        tc[csz] = sum(tr.solve("mid%d" % k, g, "PD", team=3) for k, g in enumerate(mids))
    chosen["cluster_ctas"] = pick_fastest(tc)
    tables["cluster_ctas"] = tc
    tr.set(**chosen)

    # single-solve crossovers: CTA vs cluster, cluster vs grid
    npts = [300, 800, 1500, 3000, 8000, 20000, 50000] if not quick else [300, 1500, 8000]
    graphs = [I.delaunay(n, rng) for n in npts]
    sizes = [len(g[2]) for g in graphs]
    cta, clu, grd = [], [], []
    for k, g in enumerate(graphs):
        if time.perf_counter() - t0 > budget_s:
            sizes = sizes[: len(cta)]
            break
        cta.append(tr.solve("single%d" % k, g, "PD", team=1))
        clu.append(tr.solve("single%d" % k, g, "PD", team=3))
        grd.append(tr.solve("single%d" % k, g, "PD", team=2))
    if sizes:
        chosen["single_cluster_min"] = crossover(sizes, cta, clu, int(base["single_cluster_min"]))
        chosen["single_grid_min"] = max(chosen["single_cluster_min"],
                                        crossover(sizes, clu, grd, int(base["single_grid_min"])))
    tables["single"] = {"edges": sizes, "cta_ms": cta, "cluster_ms": clu, "grid_ms": grd}
    tr.set(**chosen)

    # batches: which instances get a cluster, on a batch large enough that
    # many clusters and CTAs run side by side (the cluster size that is best
    # for one solve alone need not be best there: both are tried, and the
    # batch decides); and the CTA size of the instances that run alone (a
    # batch without cluster instances runs on the per-instance CTA kernel of
    # that size)
    batch = I.delaunay_batch(count=256 if not quick else 24, nmin=500, nmax=20000, seed=11)
    csizes = [chosen["cluster_ctas"]] + [c for c in tc if c != chosen["cluster_ctas"] and c == base["cluster_ctas"]]
    tb = {}
    for csz in csizes:
        for threads in (512, 256):
            for bmin, share in ((10000, 1.0), (20000, 1.5), (20000, 3.0), (40000, 1.5), (1 << 40, 1.5)):
                if time.perf_counter() - t0 > budget_s and tb:
                    break
                tr.set(**{**chosen, "cluster_ctas": csz, "batch_cluster_min": bmin, "batch_cluster_share": share,
                          "cta_threads": threads})
                tb[(bmin, share, threads, csz)] = tr.batch("batch", batch, "PD")
    bmin, share, threads, csz = pick_fastest(tb)
    chosen["batch_cluster_min"], chosen["batch_cluster_share"], chosen["cta_threads"] = bmin, share, threads
    chosen["cluster_ctas"] = csz
    tables["batch"] = {f"{k[0]}/{k[1]}/{k[2]}/{k[3]}": v for k, v in tb.items()}
    tr.set(**chosen)
    return {"tuning": chosen, "default": base, "tables": tables, "seconds": round(time.perf_counter() - t0, 1)}


def apply(handle, device: int = 0, path: Optional[str] = None) -> Optional[dict]:
    """Sets the cached tuning of this device on `handle`; returns it, or None
    when the cache has none."""
    entry = load_cache(path).get(device_key(device))
    if not entry:
        return None
    t = _lib.RamaTuning()
    for k in KNOBS:
        setattr(t, k, entry["tuning"][k])
    handle.set_tuning(t)
    return entry


def ensure(device: int = 0, budget_s: float = 60.0, path: Optional[str] = None) -> dict:
    """The cached tuning of this device, tuning it first when there is none.
    Returns the cache entry plus "source": "cache" or "tuned now"."""
    key = device_key(device)
    entry = load_cache(path).get(key)
    if entry:
        return {**entry, "source": "cache"}
    entry = tune(device, budget_s)
    save_cache(key, entry, path)
    return {**entry, "source": "tuned now"}


def main(argv: Optional[List[str]] = None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--budget", type=float, default=60.0, help="seconds of trial solves (approximate)")
    ap.add_argument("--force", action="store_true", help="tune again even when cached")
    a = ap.parse_args(argv)
    if a.force:
        entry = tune(a.device, a.budget)
        save_cache(device_key(a.device), entry)
    else:
        entry = ensure(a.device, a.budget)
    print(json.dumps(entry, indent=1, default=str))


if __name__ == "__main__":
    main()
