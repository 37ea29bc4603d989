"""Continuous-batching server: admission by HBM footprint (CPU) and results
that are the same in the mix as alone (GPU)."""
from collections import deque
from types import SimpleNamespace

import numpy as np
import pytest

from rama_b200 import instances, server


def _req(nbytes, rid):
    return SimpleNamespace(bytes=nbytes, rid=rid)


def test_admit_takes_arrival_order_within_budget():
    q = deque(_req(b, k) for k, b in enumerate((30, 50, 10, 40, 5)))
    g = server.admit(q, budget=100, max_count=10)
    assert [r.rid for r in g] == [0, 1, 2]  # 30 + 50 + 10; 40 would exceed 100
    assert [r.rid for r in q] == [3, 4]     # the rest waits, in order
    g = server.admit(q, budget=100, max_count=1)
    assert [r.rid for r in g] == [3]


def test_admit_never_skips_the_front_request():
    q = deque([_req(120, 0), _req(1, 1)])
    assert server.admit(q, budget=100, max_count=10) == []  # too big: the lane stays idle
    assert [r.rid for r in q] == [0, 1]


def _sreq(edges, rid):
    return SimpleNamespace(bytes=edges * 1100, num_edges=edges, num_nodes=edges, rid=rid)


def test_large_requests_go_alone_and_end_a_group():
    """A request of at least solo_min_edges runs alone (on the whole GPU); a
    group of small ones stops in front of it, and it is taken next."""
    me = SimpleNamespace(solo_min_edges=1000, max_batch=10)
    lane = SimpleNamespace(budget=10 ** 9, fits=lambda g: True)
    q = deque([_sreq(10, 0), _sreq(20, 1), _sreq(5000, 2), _sreq(30, 3)])
    g, solo = server.Server._take(me, q, lane)
    assert [r.rid for r in g] == [0, 1] and not solo
    g, solo = server.Server._take(me, q, lane)
    assert [r.rid for r in g] == [2] and solo
    g, solo = server.Server._take(me, q, lane)
    assert [r.rid for r in g] == [3] and not solo and not q


def test_footprint_counts_the_solver_slice():
    # the solver's slice: 1024 B per edge + 1 MiB, rounded up to 4 KiB
    assert server.workspace_slice(0) == 1 << 20
    assert server.workspace_slice(1000) == (1000 * 1024 + (1 << 20) + 4095) // 4096 * 4096
    assert server.footprint(1000, 500) == server.workspace_slice(1000) + 16 * 1000 + 4 * 500 + 4096


def test_served_stream_is_poisson_over_the_pool():
    s = instances.served_stream(num_requests=2000, rate=500.0, pool_size=7, seed=3)
    t = np.array([x[0] for x in s])
    assert np.all(np.diff(t) >= 0)
    assert abs(t[-1] - 2000 / 500.0) < 0.5  # mean inter-arrival 1/rate
    modes = [x[1] for x in s]
    assert abs(modes.count("P") / 2000 - 0.5) < 0.05 and abs(modes.count("D") / 2000 - 0.1) < 0.03
    assert {x[2] for x in s} <= set(range(7))


@pytest.mark.gpu
def test_results_in_the_mix_equal_solo_solves():
    """Requests of different sizes and modes arrive while others run; every
    result equals the same request solved alone (labels and bound, exactly)."""
    from rama_b200.solver import Solver

    pool = instances.served_pool(size=10, seed=21, max_edges=60000)
    stream = instances.served_stream(num_requests=30, rate=3000.0, pool_size=10, seed=22)
    # requests of 20,000 edges and more run alone on the whole GPU
    srv = server.Server(device=0, lanes=3, lane_bytes=512 << 20, max_batch=8, solo_min_edges=20000)
    try:
        reqs = [server.Request(k, *pool[p], mode=m, arrival=t) for k, (t, m, p) in enumerate(stream)]
        st = srv.serve(reqs, realtime=True)
        assert all(r.status == 0 for r in reqs)
        # everything queued at once: the lanes run side by side
        reqs2 = [server.Request(k, *pool[p], mode=m) for k, (t, m, p) in enumerate(stream)]
        st2 = srv.serve(reqs2, realtime=False)
        assert st2.max_busy_lanes >= 2
    finally:
        srv.close()
    solo = Solver(0)
    for r, r2 in zip(reqs, reqs2):
        lab, lb, _ = solo.solve(r.i, r.j, r.c, mode=r.mode)
        assert np.array_equal(r.labels, lab) and r.lb == lb
        assert np.array_equal(r2.labels, lab) and r2.lb == lb
    s = st.summary()
    assert s["requests"] == 30 and s["p99_ms"] >= s["p50_ms"] > 0
