"""Batches of independent instances spread over several GPUs.

One instance does not shard (every round needs a global sort and matching),
but the instances of a batch are independent.  `lpt_shards` deals them to
ranks by greedy longest-processing-time: largest first (by edge count, ties
by index), each to the rank with the smallest load so far (ties to the lower
rank).  `solve_batch_sharded` solves this rank's shard as one batch on its
own GPU and gathers every rank's results with torch.distributed (any
backend; the data path has no collective, only the final gather of labels
and bounds).  Each instance's result equals its single solve, so the
combined result does not depend on the number of ranks.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np

from . import instances as I


def lpt_shards(sizes: Sequence[int], world: int) -> List[List[int]]:
    """Instance indices per rank, each list in increasing index order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k))
    load = [0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(k)
        load[r] += int(sizes[k])
    return [sorted(x) for x in out]


def solve_batch_sharded(batch: "I.Batch", mode: str = "PD", rank: int = 0, world: int = 1,
                        solve: Optional[Callable[["I.Batch", str], List[Tuple[np.ndarray, float]]]] = None,
                        group=None) -> List[Tuple[np.ndarray, float]]:
    """Solves `batch` over `world` ranks: this rank takes its LPT shard, and
    the (labels, lower bound) of every instance come back on every rank, in
    batch order.  `solve` solves a sub-batch (default: one rama_solve_batch
    on this process's current GPU)."""
    sizes = np.diff(np.asarray(batch.edge_offsets, np.int64))
    shards = lpt_shards(sizes, world)
    mine = shards[rank]
    if solve is None:
        from .solver import Solver

        def solve(b, m):
            res, status, rc = Solver().solve_batch(b, mode=m)
            if rc != 0:
                raise RuntimeError(f"batch solve failed on rank {rank}: status {status.tolist()}")
            return res

    # A rank whose solve fails still takes part in the gather (otherwise the
    # other ranks would wait in it for ever): it sends its error instead of
    # results, and every rank raises after the gather.
    error = None
    local: list = []
    try:
        part = solve(I.pack([batch.instance(k) for k in mine]), mode) if mine else []
        local = [(k, np.asarray(lab), float(lb)) for k, (lab, lb) in zip(mine, part)]
    except Exception as e:  # noqa: BLE001 -- re-raised on every rank below
        if world == 1:
            raise
        error = f"rank {rank}: {type(e).__name__}: {e}"
    if world == 1:
        gathered = [(None, local)]
    else:
        import torch.distributed as dist

        gathered = [None] * world
        dist.all_gather_object(gathered, (error, local), group=group)
    failed = [err for err, _ in gathered if err is not None]
    if failed:
        raise RuntimeError("sharded batch solve failed: " + "; ".join(failed))
    out: List[Optional[Tuple[np.ndarray, float]]] = [None] * batch.count
    for _, lst in gathered:
        for k, lab, lb in lst:
            out[k] = (lab, lb)
    if any(x is None for x in out):
        raise RuntimeError("an instance was not solved by any rank")
    return out  # type: ignore[return-value]
