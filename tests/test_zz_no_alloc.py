"""rama_solve_small_static: the solve entry point that allocates no device memory.

It serves callers that cannot call cudaMalloc -- an application whose device
memory is fully reserved by its own pool allocator, a latency-critical loop
that cannot afford cudaMalloc's device synchronisation, or a process with a
fixed device-memory budget.  Its scratch memory is a fixed 32 MiB array inside
the library.  The test calls it twice in a row through the C ABI and checks
each result against the regular entry point, rama_solve: the labels and the
lower bound must be identical, the same tolerance the other parity tests use.

This file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from rama_b200 import _lib, instances

pytestmark = pytest.mark.gpu


def _static(d_i, d_j, d_c, n, opts, d_lab):
    nl = C.c_int64(0)
    lb = C.c_double(0)
    rc = _lib.load().rama_solve_small_static(C.c_void_p(d_i.data_ptr()), C.c_void_p(d_j.data_ptr()),
                                             C.c_void_p(d_c.data_ptr()), n, C.byref(opts),
                                             C.c_void_p(d_lab.data_ptr()), d_lab.numel(), C.byref(nl), C.byref(lb),
                                             None)
    return rc, nl.value, lb.value


@pytest.mark.parametrize("mode", ("PD", "P"))
def test_static_matches_rama_solve_twice(mode):
    import torch

    from rama_b200.solver import Solver

    i, j, c = instances.grid2d(24, 24, seed=31)
    d_i, d_j, d_c = (torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (i, j, c))
    n = len(c)
    N = int(max(i.max(), j.max())) + 1
    ref_lab, ref_lb = Solver(0).solve_device(d_i, d_j, d_c, mode=mode)
    ref_lab = ref_lab.cpu().numpy()
    opts = _lib.options(mode)
    for _ in range(2):
        d_lab = torch.full((N,), -7, dtype=torch.int32, device="cuda")
        rc, nl, lb = _static(d_i, d_j, d_c, n, opts, d_lab)
        assert rc == 0, _lib.load().rama_last_error()
        torch.cuda.synchronize()
        assert nl == N
        assert lb == ref_lb
        assert np.array_equal(d_lab.cpu().numpy(), ref_lab)


def test_static_rejects_oversized_instance():
    import torch

    d = torch.zeros(8, dtype=torch.int32, device="cuda")
    opts = _lib.options("PD")
    nl = C.c_int64(0)
    lb = C.c_double(0)
    rc = _lib.load().rama_solve_small_static(C.c_void_p(d.data_ptr()), C.c_void_p(d.data_ptr()),
                                             C.c_void_p(d.data_ptr()), 30001, C.byref(opts), C.c_void_p(d.data_ptr()),
                                             8, C.byref(nl), C.byref(lb), None)
    assert rc == _lib.RAMA_ERR_INVALID_ARG
    assert b"exceed the limit of 30000" in _lib.load().rama_last_error()


def test_static_rejects_node_id_beyond_limit():
    """A node id of RAMA_STATIC_MAX_NODES (65,536) is refused on the device
    before the solve starts."""
    import torch

    i = np.array([0, 1, 2], np.int32)
    j = np.array([1, 2, 65536], np.int32)
    c = np.array([1.0, -1.0, 0.5], np.float32)
    d_i, d_j, d_c = (torch.from_numpy(x).cuda() for x in (i, j, c))
    d_lab = torch.zeros(65537, dtype=torch.int32, device="cuda")
    rc, nl, _ = _static(d_i, d_j, d_c, 3, _lib.options("PD"), d_lab)
    assert rc == _lib.RAMA_ERR_INVALID_ARG
    assert nl == 0
    assert b"65536" in _lib.load().rama_last_error()


@pytest.mark.parametrize("mode", ("PD", "PD+"))
def test_static_near_the_edge_limit(mode):
    """An instance just under the 30,000-edge limit fits the fixed array and
    gives rama_solve's result, twice in a row."""
    import torch

    from rama_b200.solver import Solver

    i, j, c = instances.grid2d(122, 123, seed=37)  # 29,767 edges
    assert 29000 < len(c) <= 30000
    d_i, d_j, d_c = (torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (i, j, c))
    N = int(max(i.max(), j.max())) + 1
    s = Solver(0)
    ref_lab, ref_lb = s.solve_device(d_i, d_j, d_c, mode=mode, team=1)
    ref_lab = ref_lab.cpu().numpy()
    assert s.stats().workspace_peak < (32 << 20) - 4096
    for _ in range(2):
        d_lab = torch.full((N,), -7, dtype=torch.int32, device="cuda")
        rc, nl, lb = _static(d_i, d_j, d_c, len(c), _lib.options(mode), d_lab)
        assert rc == 0, _lib.load().rama_last_error()
        assert nl == N
        assert lb == ref_lb
        assert np.array_equal(d_lab.cpu().numpy(), ref_lab)
