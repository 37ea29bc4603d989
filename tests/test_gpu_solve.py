"""Full solves on the GPU: parity with the CPU oracle (bit-exact labels and
bound, both execution teams), the reference-compatible entry points, and
batching (an instance's result does not depend on its batch)."""
import numpy as np
import pytest

from rama_b200 import instances

pytestmark = pytest.mark.gpu


def cases():
    out = []
    for s, (n, deg) in enumerate([(20, 3), (40, 4), (80, 5), (150, 6), (300, 4), (60, 8), (3000, 5)]):
        out.append(("rnd%d" % s, instances.random_graph(n, deg, seed=100 + s)))
    out.append(("grid12", instances.grid2d(12, 12, seed=77)))
    out.append(("grid64", instances.grid2d(64, 64, seed=1001)))
    out.append(("hub", hub_graph()))
    return out


def hub_graph(spokes=6000, seed=5):
    """Node 0 joined to `spokes` nodes, which form a ring: its row (and, after
    a contraction, its cluster's row) holds more than 4096 edges, which sends
    the bucket sorts of the initial sort and of the contraction to their radix
    fallbacks."""
    rng = np.random.default_rng(seed)
    k = np.arange(1, spokes + 1, dtype=np.int32)
    i = np.concatenate([np.zeros(spokes, np.int32), k[:-1]])
    j = np.concatenate([k, k[1:]])
    c = rng.normal(0.3, 1.0, size=len(i)).astype(np.float32)
    return i, j, c


CASES = cases()
IDS = [c[0] for c in CASES]


@pytest.mark.parametrize("team", (1, 2, 3))
@pytest.mark.parametrize("mode", ("P", "PD", "PD+", "D"))
@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_solve_matches_oracle(solver, oracle, case, mode, team):
    _, (i, j, c) = case
    olab, olb, _ = oracle.solve(i, j, c, mode)
    glab, glb, st = solver.solve(i, j, c, mode=mode, team=team)
    assert glb == olb
    assert np.array_equal(glab, olab)


@pytest.mark.parametrize("team", (1, 2, 3))
@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_solve_with_pentagon_check_matches_oracle(solver, oracle, case, team):
    """woc_pentagons = 1: forest contractions also cut conflicted 5-cycles."""
    _, (i, j, c) = case
    olab, olb, _ = oracle.solve(i, j, c, "P", woc_pentagons=1)
    glab, glb, _ = solver.solve(i, j, c, mode="P", team=team, woc_pentagons=1)
    assert glb == olb
    assert np.array_equal(glab, olab)


@pytest.mark.parametrize("case", CASES[-3:], ids=IDS[-3:])
def test_bound_below_objective(solver, oracle, case):
    _, (i, j, c) = case
    lab, lb, _ = solver.solve(i, j, c, mode="PD")
    assert lb <= oracle.objective(i, j, c, lab) + 1e-9


def test_device_objective_matches_oracle(solver, oracle):
    import torch

    i, j, c = instances.grid2d(64, 64, seed=1001)
    lab, _, _ = solver.solve(i, j, c, mode="PD")
    d = [torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (i, j, c, lab)]
    assert solver.objective(*d) == oracle.objective(i, j, c, lab)


def test_invalid_input_is_rejected(solver):
    from rama_b200._lib import RamaError

    with pytest.raises(RamaError):
        solver.solve(np.array([0, 1]), np.array([0, 2]), np.array([1.0, 2.0]))  # self loop
    with pytest.raises(RamaError):
        solver.solve(np.array([-1, 1]), np.array([2, 2]), np.array([1.0, 2.0]))


def test_empty_instance(solver):
    lab, lb, _ = solver.solve(np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32))
    assert len(lab) == 0 and lb == 0.0


def test_batch_with_clusters_equals_single_solves(solver, oracle):
    """Instances of 20,000 edges and more go to cluster teams, the rest to
    CTAs; every result equals the oracle's."""
    rng = np.random.default_rng(8)
    insts = [instances.delaunay(int(n), rng) for n in (9000, 300, 12000, 7000, 50, 2500)]
    insts += [instances.random_graph(5000, 6, seed=12), instances.grid2d(150, 150, seed=6)]
    batch = instances.pack(insts)
    for mode in ("PD", "D"):
        res, status, rc = solver.solve_batch(batch, mode=mode)
        assert rc == 0 and not status.any()
        for k, (i, j, c) in enumerate(insts):
            olab, olb, _ = oracle.solve(i, j, c, mode)
            assert np.array_equal(res[k][0], olab)
            assert res[k][1] == olb


def test_batch_equals_single_solves(solver, oracle):
    rng = np.random.default_rng(3)
    insts = [instances.delaunay(int(n), rng) for n in (50, 700, 120, 2000, 33, 900)]
    insts += [instances.random_graph(200, 5, seed=9), instances.grid2d(20, 30, seed=4)]
    batch = instances.pack(insts)
    for mode in ("P", "PD"):
        res, status, rc = solver.solve_batch(batch, mode=mode)
        assert rc == 0 and not status.any()
        for k, (i, j, c) in enumerate(insts):
            lab, lb, _ = solver.solve(i, j, c, mode=mode, team=1)
            assert np.array_equal(res[k][0], lab)
            assert res[k][1] == lb
            olab, olb, _ = oracle.solve(i, j, c, mode)
            assert np.array_equal(lab, olab) and lb == olb


# ---------------------------------------------------------------- rama_py API
def test_rama_py_pytorch():
    """test/test_pytorch.py of the reference."""
    import torch
    import rama_py

    opts = rama_py.multicut_solver_options("P")
    opts.verbose = False
    res = rama_py.rama_cuda([0, 1, 2], [1, 2, 0], [1.1, -2, 3], opts)
    expected = res[0]
    i = torch.Tensor([0, 1, 2]).to("cuda").to(torch.int32)
    j = torch.Tensor([1, 2, 0]).to("cuda").to(torch.int32)
    costs = torch.Tensor([1.1, -2, 3]).to("cuda").to(torch.float32)
    node_mapping, lb = rama_py.rama_torch(i, j, costs, opts)
    assert torch.all(node_mapping.cpu() == torch.Tensor(expected))


def test_rama_py_pointers():
    """test/test_pytorch_pointers.py of the reference."""
    import torch
    import rama_py

    opts = rama_py.multicut_solver_options("P")
    opts.verbose = False
    res = rama_py.rama_cuda([0, 1, 2], [1, 2, 0], [1.1, -2, 3], opts)
    expected = res[0]
    i = torch.Tensor([0, 1, 2]).to("cuda").contiguous().to(torch.int32)
    j = torch.Tensor([1, 2, 0]).to("cuda").contiguous().to(torch.int32)
    costs = torch.Tensor([1.1, -2, 3]).to("cuda").contiguous().to(torch.float32)
    num_nodes = max(i.max(), j.max()) + 1
    node_labels = torch.ones(num_nodes, device=i.device).to(torch.int32)
    num_edges = i.numel()
    opts.dump_timeline = True
    timeline = rama_py.rama_cuda_gpu_pointers(i.data_ptr(), j.data_ptr(), costs.data_ptr(), node_labels.data_ptr(),
                                              num_nodes, num_edges, i.device.index, opts)
    assert torch.all(node_labels.cpu() == torch.Tensor(expected))
    assert isinstance(timeline, list) and len(timeline) >= 1


def test_rama_py_full_and_timeline(oracle):
    import rama_py

    i, j, c = instances.grid2d(16, 16, seed=5)
    opts = rama_py.multicut_solver_options("PD")
    opts.dump_timeline = True
    labels, lb, ms, timeline = rama_py.rama_cuda(i.tolist(), j.tolist(), c.tolist(), opts)
    olab, olb, st = oracle.solve(i, j, c, "PD")
    assert labels == olab.tolist() and lb == olb
    assert len(timeline) == st.rounds and timeline[-1] == labels


def test_cli(tmp_path, oracle):
    import os
    import subprocess

    from rama_b200 import build

    i, j, c = instances.grid2d(10, 10, seed=11)
    f = tmp_path / "g.txt"
    with open(f, "w") as fh:
        fh.write("MULTICUT\n")
        for a, b, w in zip(i, j, c):
            fh.write(f"{a} {b} {float(w)!r}\n")
    out = tmp_path / "sol.txt"
    r = subprocess.run([build.CLI, "-f", str(f), "-o", str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "cost w.r.t original objective" in r.stdout and "final lower bound" in r.stdout
    lines = [ln for ln in open(out).read().split("\n") if ln.strip()]
    seen = sorted(int(x) for ln in lines for x in ln.split())
    assert seen == list(range(100))


def test_sanitize_graph_matches_oracle(solver, oracle):
    """sanitize_graph: duplicate edges dropped (first survives), nodes without
    edges get label -1 (include/rama_utils.h:429-493 of the reference)."""
    rng = np.random.default_rng(17)
    i, j, c = instances.random_graph(400, 4, seed=17)
    i = (i * 3 + 2).astype(np.int32)  # gaps in the ids
    j = (j * 3 + 2).astype(np.int32)
    dup = rng.integers(0, len(c), size=40)
    i = np.concatenate([i, j[dup]])  # duplicates, reversed orientation
    j = np.concatenate([j, i[dup]])
    c = np.concatenate([c, rng.normal(size=40).astype(np.float32)])
    for mode in ("P", "PD"):
        olab, olb, _ = oracle.solve(i, j, c, mode, sanitize_graph=1)
        glab, glb, _ = solver.solve(i, j, c, mode=mode, sanitize_graph=1)
        assert np.array_equal(glab, olab) and glb == olb
        assert (glab[0] == -1) and (glab[1] == -1)


def test_async_batch_mixed_modes(solver, oracle):
    """rama_batch_launch with per-instance options; poll until done, then wait.
    Every instance equals its single solve in its own mode."""
    import ctypes as C

    import torch

    from rama_b200 import _lib

    rng = np.random.default_rng(23)
    insts = [instances.delaunay(int(n), rng) for n in (300, 80, 1500, 40, 600)]
    modes = ["P", "PD", "D", "PD+", "PD"]
    batch = instances.pack(insts)
    d = [torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (batch.i, batch.j, batch.c)]
    lo = np.zeros(batch.count + 1, np.int64)
    lo[1:] = np.cumsum(batch.node_counts)
    lab = torch.empty(int(lo[-1]), dtype=torch.int32, device="cuda")
    opts = (_lib.RamaOptions * batch.count)(*[_lib.options(m) for m in modes])
    eo = np.ascontiguousarray(batch.edge_offsets, np.int64)
    L = _lib.load()
    h = solver.handle.h
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check(L.rama_batch_launch(h, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), eo.ctypes.data, batch.count,
                                   opts, batch.count, lab.data_ptr(), lo.ctypes.data, st))
    for _ in range(100000):
        r = L.rama_batch_poll(h)
        if r != 0:
            break
    assert r >= 0
    nl = np.zeros(batch.count, np.int64)
    lbs = np.zeros(batch.count)
    status = np.zeros(batch.count, np.int32)
    _lib.check(L.rama_batch_wait(h, nl.ctypes.data, lbs.ctypes.data, status.ctypes.data))
    out = lab.cpu().numpy()
    for k, (i, j, c) in enumerate(insts):
        olab, olb, _ = oracle.solve(i, j, c, modes[k])
        assert lbs[k] == olb
        assert np.array_equal(out[lo[k]:lo[k] + nl[k]], olab)
