"""Continuous-batching multicut server.

Requests arrive over time: the host arrays (i, j, c) of one instance and a
mode.  The server owns `lanes` solver handles, each with its own CUDA
stream, a fixed device workspace of `lane_bytes` and device buffers for its
inputs and labels.

Admission is by HBM footprint.  An idle lane takes the waiting requests in
arrival order while the sum of their footprints fits its budget (a request's
footprint is its workspace slice, 1024 bytes per edge plus 1 MiB, as the
solver allocates it, plus 16 bytes per edge and 4 per node of inputs and
labels).  It copies their graphs to the device and launches them as one
asynchronous batch (``rama_batch_launch``: instances that hold much more
than the batch's load per CTA run on cluster teams, the rest one per CTA).
A request of at least `solo_min_edges` edges (default: the size from which a
single solve runs on the whole GPU, from the handle's tuning) is launched
alone, on the whole GPU: on one CTA or one cluster it would take many times
longer than a plain solve, and every request queued behind it would wait.

Lanes run concurrently on their own streams, so the kernels of requests
admitted at different times overlap on the GPU.  A lane that finishes hands
back its results and takes the next requests at once (continuous batching).
Each graph stays resident on the device through all its rounds: a solve is
one kernel launch with no host round-trip.

A request's result does not depend on the batch it ran in.  Every
order-sensitive step of the solver is defined by element index, not by the
team or the other instances, so a request solved in the mix returns the same
labels and lower bound, bit for bit, as when solved alone.

Kernels of more than 8 streams only overlap when the process starts with
``CUDA_DEVICE_MAX_CONNECTIONS`` at least the number of lanes (set it before
CUDA is first used).
"""
from __future__ import annotations

import ctypes as C
import time
from collections import deque
from dataclasses import dataclass, field
from typing import Callable, List, Optional, Sequence

import numpy as np

from . import _lib

MiB = 1 << 20


def workspace_slice(num_edges: int) -> int:
    """Device workspace the solver gives one instance of a batch (bytes)."""
    return (num_edges * 1024 + MiB + 4095) & ~4095


def footprint(num_edges: int, num_nodes: int) -> int:
    """HBM one request holds while it is on the GPU: its workspace slice plus
    its inputs (i, j, c: 12 bytes per edge, rounded up to 16) and labels."""
    return workspace_slice(num_edges) + 16 * num_edges + 4 * num_nodes + 4096


@dataclass
class Request:
    rid: int
    i: object  # int32 host array (numpy, or a pinned torch tensor)
    j: object
    c: object  # float32
    mode: str = "PD"
    arrival: float = 0.0  # seconds after the start of the stream
    num_nodes: int = -1
    # filled in by the server
    labels: Optional[np.ndarray] = None
    lb: float = float("nan")
    status: int = -1
    admitted: float = float("nan")
    finished: float = float("nan")
    lane: int = -1

    def __post_init__(self):
        if self.num_nodes < 0:
            n = len(self.c)
            self.num_nodes = int(max(_amax(self.i), _amax(self.j)) + 1) if n else 0

    @property
    def num_edges(self) -> int:
        return len(self.c)

    @property
    def bytes(self) -> int:
        return footprint(self.num_edges, self.num_nodes)

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def _amax(x):
    return int(x.max()) if len(x) else -1


def admit(pending: deque, budget: int, max_count: int) -> List[Request]:
    """Takes requests from the front of `pending` (arrival order) while their
    footprints fit `budget` and there are at most `max_count` of them.  The
    front request is always taken when it fits the budget on its own."""
    group: List[Request] = []
    used = 0
    while pending and len(group) < max_count:
        r = pending[0]
        if used + r.bytes > budget:
            break
        group.append(pending.popleft())
        used += r.bytes
    return group


class Lane:
    """One solver handle + stream + device buffers; runs one batch at a time."""

    def __init__(self, index: int, device: int, lane_bytes: int, io_edges: int, io_nodes: int):
        import torch

        self.index = index
        self.device = device
        self.budget = lane_bytes
        ws = max(lane_bytes - 16 * io_edges - 4 * io_nodes, 64 * MiB)
        self.handle = _lib.Handle(device, workspace_bytes=ws)
        self.stream = torch.cuda.Stream(device=device)
        dev = torch.device("cuda", device)
        self.d_i = torch.empty(max(io_edges, 1), dtype=torch.int32, device=dev)
        self.d_j = torch.empty(max(io_edges, 1), dtype=torch.int32, device=dev)
        self.d_c = torch.empty(max(io_edges, 1), dtype=torch.float32, device=dev)
        self.d_lab = torch.empty(max(io_nodes, 1), dtype=torch.int32, device=dev)
        self.h_lab = torch.empty(max(io_nodes, 1), dtype=torch.int32, pin_memory=True)
        self.io_edges, self.io_nodes = io_edges, io_nodes
        self.group: List[Request] = []
        self.label_off = None
        self.busy = False
        self.alg_bytes = 0.0  # algorithmic bytes of the batches this lane ran

    def fits(self, group: Sequence[Request]) -> bool:
        return (sum(r.num_edges for r in group) <= self.io_edges and sum(r.num_nodes for r in group) <= self.io_nodes
                and sum(workspace_slice(r.num_edges) for r in group) <= self.handle_ws)

    @property
    def handle_ws(self) -> int:
        return max(self.budget - 16 * self.io_edges - 4 * self.io_nodes, 64 * MiB)

    def launch(self, group: List[Request], now: float, solo: bool = False):
        import torch

        n = len(group)
        eo = np.zeros(n + 1, np.int64)
        lo = np.zeros(n + 1, np.int64)
        eo[1:] = np.cumsum([r.num_edges for r in group])
        lo[1:] = np.cumsum([r.num_nodes for r in group])
        with torch.cuda.stream(self.stream):
            for k, r in enumerate(group):
                a, b = int(eo[k]), int(eo[k + 1])
                if b > a:
                    self.d_i[a:b].copy_(_as_tensor(r.i), non_blocking=True)
                    self.d_j[a:b].copy_(_as_tensor(r.j), non_blocking=True)
                    self.d_c[a:b].copy_(_as_tensor(r.c), non_blocking=True)
        opts = (_lib.RamaOptions * n)(*[_lib.options(r.mode, team=2 if solo else 0) for r in group])
        st = C.c_void_p(self.stream.cuda_stream)
        _lib.check(_lib.load().rama_batch_launch(self.handle.h, self.d_i.data_ptr(), self.d_j.data_ptr(),
                                                 self.d_c.data_ptr(), eo.ctypes.data, n, opts, n,
                                                 self.d_lab.data_ptr(), lo.ctypes.data, st))
        for r in group:
            r.admitted = now
            r.lane = self.index
        self.group = group
        self.label_off = lo
        self.busy = True

    def poll(self) -> bool:
        r = _lib.load().rama_batch_poll(self.handle.h)
        if r < 0:
            raise _lib.RamaError(_lib.RAMA_ERR_CUDA, _lib.load().rama_last_error().decode(errors="replace"))
        return r == 1

    def finish(self, now: float) -> List[Request]:
        import torch

        n = len(self.group)
        nl = np.zeros(n, np.int64)
        lbs = np.zeros(n, np.float64)
        status = np.zeros(n, np.int32)
        rc = _lib.load().rama_batch_wait(self.handle.h, nl.ctypes.data, lbs.ctypes.data, status.ctypes.data)
        self.alg_bytes += float(self.handle.stats().alg_bytes)
        total = int(self.label_off[-1])
        with torch.cuda.stream(self.stream):
            if total:
                self.h_lab[:total].copy_(self.d_lab[:total], non_blocking=True)
        self.stream.synchronize()
        lab = self.h_lab.numpy()
        for k, r in enumerate(self.group):
            a = int(self.label_off[k])
            r.labels = lab[a:a + int(nl[k])].copy()
            r.lb = float(lbs[k])
            r.status = int(status[k]) if rc == 0 or status[k] else int(rc)
            r.finished = now
        done, self.group, self.busy = self.group, [], False
        return done


def _as_tensor(x):
    import torch

    if isinstance(x, torch.Tensor):
        return x
    return torch.from_numpy(np.ascontiguousarray(x))


@dataclass
class ServeStats:
    requests: int = 0
    edges: int = 0
    wall_s: float = 0.0
    latencies: List[float] = field(default_factory=list)
    max_busy_lanes: int = 0
    batches: int = 0

    def summary(self) -> dict:
        lat = np.asarray(self.latencies) if self.latencies else np.zeros(1)
        return {
            "requests": self.requests,
            "solves_per_s": self.requests / self.wall_s if self.wall_s > 0 else 0.0,
            "edges_per_s": self.edges / self.wall_s if self.wall_s > 0 else 0.0,
            "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "mean_ms": float(lat.mean() * 1e3),
            "wall_s": self.wall_s,
            "batches": self.batches,
            "max_concurrent_lanes": self.max_busy_lanes,
        }


class Server:
    """Continuous batching over `lanes` lanes of `lane_bytes` of HBM each."""

    def __init__(self, device: int = 0, lanes: int = 8, lane_bytes: int = 8 << 30, max_batch: int = 256,
                 io_edges: Optional[int] = None, io_nodes: Optional[int] = None,
                 solo_min_edges: Optional[int] = None, tuning=None):
        if io_edges is None:
            io_edges = lane_bytes // 1100
        if io_nodes is None:
            io_nodes = io_edges
        self.max_batch = max_batch
        self.lanes = [Lane(k, device, lane_bytes, io_edges, io_nodes) for k in range(lanes)]
        if tuning is not None:
            for ln in self.lanes:
                ln.handle.set_tuning(tuning)
        self.lane_bytes = lane_bytes
        if solo_min_edges is None:
            solo_min_edges = int(self.lanes[0].handle.tuning().single_grid_min)
        self.solo_min_edges = solo_min_edges

    def close(self):
        for ln in self.lanes:
            ln.handle.close()

    def admissible(self, r: Request) -> bool:
        return self.lanes[0].fits([r])

    def _take(self, pending: deque, lane: Lane):
        """The next group for `lane` and whether it runs alone on the whole
        GPU: a large request at the front of the queue goes alone; otherwise
        the small requests up to the next large one, by footprint."""
        if pending and pending[0].num_edges >= self.solo_min_edges:
            return [pending.popleft()], True
        group = admit(pending, lane.budget, self.max_batch)
        # a large request ends the group (it runs alone later)
        for k, r in enumerate(group):
            if r.num_edges >= self.solo_min_edges:
                for x in reversed(group[k:]):
                    pending.appendleft(x)
                group = group[:k]
                break
        # the I/O buffers and the workspace bound the group too
        while group and not lane.fits(group):
            pending.appendleft(group.pop())
        return group, False

    def serve(self, requests: Sequence[Request], clock: Callable[[], float] = time.perf_counter,
              realtime: bool = True) -> ServeStats:
        """Serves `requests` (sorted by arrival).  With `realtime`, a request
        becomes visible at its arrival time; otherwise all are queued at once.
        Requests that fit no lane get status RAMA_ERR_OOM without running."""
        reqs = list(requests)
        stats = ServeStats(requests=len(reqs), edges=sum(r.num_edges for r in reqs))
        pending: deque = deque()
        nxt = 0
        done = 0
        t0 = clock()
        while done < len(reqs):
            now = clock() - t0
            while nxt < len(reqs) and (not realtime or reqs[nxt].arrival <= now):
                r = reqs[nxt]
                nxt += 1
                if not realtime:
                    r.arrival = 0.0
                if self.admissible(r):
                    pending.append(r)
                else:
                    r.status = _lib.RAMA_ERR_OOM
                    r.finished = now
                    done += 1
            progressed = False
            for ln in self.lanes:
                if ln.busy and ln.poll():
                    now = clock() - t0
                    for r in ln.finish(now):
                        stats.latencies.append(r.latency)
                        done += 1
                    progressed = True
            for ln in self.lanes:
                if not ln.busy and pending:
                    group, solo = self._take(pending, ln)
                    if group:
                        ln.launch(group, clock() - t0, solo=solo)
                        stats.batches += 1
                        progressed = True
            stats.max_busy_lanes = max(stats.max_busy_lanes, sum(ln.busy for ln in self.lanes))
            if not progressed:
                if not pending and not any(ln.busy for ln in self.lanes) and nxt < len(reqs):
                    time.sleep(max(0.0, min(reqs[nxt].arrival - (clock() - t0), 1e-3)))
                else:
                    time.sleep(20e-6)
        stats.wall_s = clock() - t0
        return stats
