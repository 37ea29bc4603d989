"""Batches spread over ranks (rama_b200.shard): the LPT deal, and two gloo
ranks on the CPU that each solve their shard (with the oracle standing in for
the GPU) and gather results equal to a one-process solve."""
import os
import socket

import numpy as np
import pytest

from rama_b200 import instances, shard


def test_lpt_deals_largest_first_to_the_lightest_rank():
    sizes = [5, 9, 1, 9, 3, 7]
    s = shard.lpt_shards(sizes, 2)
    # 9 (k=1) -> r0, 9 (k=3) -> r1, 7 -> r0, 5 -> r1, 3 -> r1, 1 -> r0
    assert s == [[1, 2, 5], [0, 3, 4]]
    assert sorted(sum(s, [])) == list(range(len(sizes)))
    loads = [sum(sizes[k] for k in x) for x in s]
    assert max(loads) - min(loads) <= max(sizes)
    assert shard.lpt_shards(sizes, 1) == [list(range(6))]
    assert shard.lpt_shards([], 3) == [[], [], []]


def _oracle_batch_solve(b, mode):
    from oracle import oracle_py as O

    out = []
    for k in range(b.count):
        lab, lb, _ = O.solve(*b.instance(k), mode)
        out.append((lab, lb))
    return out


def _batch():
    rng = np.random.default_rng(41)
    return instances.pack([instances.delaunay(int(n), rng) for n in (40, 300, 90, 20, 150, 60, 500)])


def _rank_main(rank, world, port, outdir):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res = shard.solve_batch_sharded(_batch(), "PD", rank, world, solve=_oracle_batch_solve)
        np.savez(os.path.join(outdir, f"r{rank}.npz"), lb=np.array([x[1] for x in res]),
                 **{f"lab{k}": x[0] for k, x in enumerate(res)})
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_gather_the_one_process_result(tmp_path):
    import torch.multiprocessing as mp

    want = shard.solve_batch_sharded(_batch(), "PD", 0, 1, solve=_oracle_batch_solve)
    mp.spawn(_rank_main, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    for r in range(2):
        got = np.load(tmp_path / f"r{r}.npz")
        assert np.array_equal(got["lb"], np.array([x[1] for x in want]))
        for k, (lab, _) in enumerate(want):
            assert np.array_equal(got[f"lab{k}"], lab)


def _failing_solve(b, mode):
    raise RuntimeError("planted failure")


def _rank_main_one_fails(rank, world, port, outdir):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        solve = _failing_solve if rank == 1 else _oracle_batch_solve
        try:
            shard.solve_batch_sharded(_batch(), "PD", rank, world, solve=solve)
            msg = "no error"
        except RuntimeError as e:
            msg = str(e)
        with open(os.path.join(outdir, f"r{rank}.txt"), "w") as f:
            f.write(msg)
    finally:
        dist.destroy_process_group()


def test_a_failing_rank_raises_on_every_rank(tmp_path):
    """Rank 1's solve raises; both ranks leave the gather and raise an error
    that names rank 1, instead of rank 0 waiting in the gather."""
    import torch.multiprocessing as mp

    mp.spawn(_rank_main_one_fails, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    for r in range(2):
        msg = (tmp_path / f"r{r}.txt").read_text()
        assert "rank 1" in msg and "planted failure" in msg, msg


@pytest.mark.gpu
def test_one_rank_solves_the_batch_on_the_gpu(oracle):
    b = _batch()
    res = shard.solve_batch_sharded(b, "PD")
    for k in range(b.count):
        olab, olb, _ = oracle.solve(*b.instance(k), "PD")
        assert np.array_equal(res[k][0], olab) and res[k][1] == olb
