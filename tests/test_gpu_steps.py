"""Parity of every CUDA solver step with the CPU oracle (through the C ABI).

Each step runs on both execution teams (one CTA, the cooperative grid) and
must reproduce the oracle bit for bit: integer outputs, and -- because both
follow the same canonical summation trees -- the float outputs too.
"""
import numpy as np
import pytest

from rama_b200 import instances

pytestmark = pytest.mark.gpu
TEAMS = (1, 2)


def graphs():
    out = []
    for s, (n, deg) in enumerate([(20, 3), (40, 4), (80, 5), (150, 6), (300, 4), (60, 8), (2000, 6)]):
        out.append(("rnd%d" % s, *instances.random_graph(n, deg, seed=100 + s)))
    out.append(("grid12", *instances.grid2d(12, 12, seed=77)))
    out.append(("grid64", *instances.grid2d(64, 64, seed=1001)))
    return out


GRAPHS = graphs()
IDS = [g[0] for g in GRAPHS]


def _G(oracle, i, j, c):
    G = oracle.Graph.from_edges(i, j, c)
    r, co, w = G.arrays()
    return G, r, co, w, G.dims[0], G.dims[1]


@pytest.mark.parametrize("team", TEAMS)
@pytest.mark.parametrize("g", GRAPHS, ids=IDS)
def test_init(solver, oracle, g, team):
    _, i, j, c = g
    G, r, co, w, rows, cols = _G(oracle, i, j, c)
    gr, gc, gw, grows, gcols = solver.step_init(i, j, c, team=team)
    assert np.array_equal(gr, r) and np.array_equal(gc, co) and np.array_equal(gw, w)
    assert (grows, gcols) == (rows, cols)


@pytest.mark.parametrize("team", TEAMS)
@pytest.mark.parametrize("g", GRAPHS, ids=IDS)
def test_contract(solver, oracle, g, team):
    _, i, j, c = g
    G, r, co, w, rows, cols = _G(oracle, i, j, c)
    rng = np.random.default_rng(7)
    N = max(rows, cols)
    m = rng.integers(0, max(N // 3, 1), size=N)
    _, m = np.unique(m, return_inverse=True)
    m = m.astype(np.int32)
    H = G.contract(m)
    hr, hc, hw = H.arrays()
    gr, gc, gw, grows, gcols = solver.step_contract(r, co, w, rows, cols, m, team=team)
    assert np.array_equal(gr, hr) and np.array_equal(gc, hc)
    assert np.array_equal(gw, hw)
    assert (grows, gcols) == H.dims


@pytest.mark.parametrize("team", TEAMS)
@pytest.mark.parametrize("g", GRAPHS, ids=IDS)
def test_coarsen(solver, oracle, g, team):
    """The solver's own contraction (self-loops removed, bad contractions
    flagged) against contract + has_bad_contractions + remove_diagonal."""
    _, i, j, c = g
    G, r, co, w, rows, cols = _G(oracle, i, j, c)
    rng = np.random.default_rng(8)
    N = max(rows, cols)
    m = rng.integers(0, max(N // 3, 1), size=N)
    _, m = np.unique(m, return_inverse=True)
    m = m.astype(np.int32)
    H = G.contract(m)
    bad = H.has_bad_contractions()
    H.remove_diagonal()
    hr, hc, hw = H.arrays()
    gr, gc, gw, grows, gcols, gbad = solver.step_coarsen(r, co, w, rows, cols, m, team=team)
    assert np.array_equal(gr, hr) and np.array_equal(gc, hc)
    assert np.array_equal(gw, hw)
    assert (grows, gcols) == H.dims
    assert gbad == bad


@pytest.mark.parametrize("nodes,edges,groups", [(3000, 30000, 2), (5000, 60000, 3), (20000, 200000, 5)])
def test_contract_runs_longer_than_a_chunk(solver, oracle, nodes, edges, groups):
    """A map onto a few nodes makes self-loop and parallel-edge runs of more
    than 4096 edges.  The plain contraction sums each by one warp, the
    solver's coarsening shares their chunks out over many warps; both must
    equal the oracle's chunked RSUM bit for bit (and the self-loop sums decide
    the bad-contraction flag)."""
    rng = np.random.default_rng(nodes)
    i = rng.integers(0, nodes, size=edges).astype(np.int32)
    j = rng.integers(0, nodes, size=edges).astype(np.int32)
    keep = i != j
    i, j = i[keep], j[keep]
    c = (rng.normal(size=len(i)) * 10.0 ** rng.integers(-3, 3, size=len(i))).astype(np.float32)
    G, r, co, w, rows, cols = _G(oracle, i, j, c)
    N = max(rows, cols)
    m = (np.arange(N) % groups).astype(np.int32)
    H = G.contract(m)
    hr, hc, hw = H.arrays()
    for team in TEAMS:
        gr, gc, gw, grows, gcols = solver.step_contract(r, co, w, rows, cols, m, team=team)
        assert np.array_equal(gr, hr) and np.array_equal(gc, hc)
        assert np.array_equal(gw, hw)
        assert (grows, gcols) == H.dims
    bad = H.has_bad_contractions()
    H.remove_diagonal()
    hr, hc, hw = H.arrays()
    for team in TEAMS:
        gr, gc, gw, grows, gcols, gbad = solver.step_coarsen(r, co, w, rows, cols, m, team=team)
        assert np.array_equal(gr, hr) and np.array_equal(gc, hc)
        assert np.array_equal(gw, hw)
        assert (grows, gcols) == H.dims and gbad == bad


@pytest.mark.parametrize("team", TEAMS)
@pytest.mark.parametrize("g", GRAPHS, ids=IDS)
def test_matching(solver, oracle, g, team):
    _, i, j, c = g
    G, r, co, w, rows, cols = _G(oracle, i, j, c)
    om, onr = oracle.matching(G, 0.05)
    gm, gnr = solver.step_matching(r, co, w, rows, cols, 0.05, team=team)
    assert gnr == onr
    assert np.array_equal(gm, om)


@pytest.mark.parametrize("team", TEAMS)
@pytest.mark.parametrize("g", GRAPHS, ids=IDS)
def test_msf(solver, oracle, g, team):
    _, i, j, c = g
    G, r, co, w, rows, cols = _G(oracle, i, j, c)
    pos = w > 0
    ids = oracle.msf(r[pos], co[pos], w[pos])
    flags = solver.step_msf(r[pos], co[pos], w[pos], team=team)
    assert np.array_equal(np.nonzero(flags)[0], ids)


@pytest.mark.parametrize("team", TEAMS)
@pytest.mark.parametrize("g", GRAPHS, ids=IDS)
def test_woc(solver, oracle, g, team):
    _, i, j, c = g
    G, r, co, w, rows, cols = _G(oracle, i, j, c)
    om, onr = oracle.woc(G)
    gm, gnr = solver.step_woc(r, co, w, rows, cols, team=team)
    assert gnr == onr
    assert np.array_equal(gm, om)


@pytest.mark.parametrize("team", TEAMS)
@pytest.mark.parametrize("g", GRAPHS, ids=IDS)
def test_woc_pentagons(solver, oracle, g, team):
    """The optional 5-cycle forest check gives the oracle's map too."""
    _, i, j, c = g
    G, r, co, w, rows, cols = _G(oracle, i, j, c)
    om, onr = oracle.woc(G, pentagons=True)
    gm, gnr = solver.step_woc(r, co, w, rows, cols, team=team, pentagons=True)
    assert gnr == onr
    assert np.array_equal(gm, om)


@pytest.mark.parametrize("team", TEAMS)
@pytest.mark.parametrize("seed", range(4))
def test_cc(solver, oracle, seed, team):
    rng = np.random.default_rng(1200 + seed)
    n = 50 + 500 * seed
    m = n // 2 + 7 * seed
    a = rng.integers(0, n, size=m)
    b = rng.integers(0, n, size=m)
    keep = a != b
    a, b = a[keep], b[keep]
    src = np.concatenate([a, b])
    dst = np.concatenate([b, a])
    order = np.lexsort((dst, src))
    src, dst = src[order], dst[order]
    off = np.zeros(n + 1, np.int64)
    np.add.at(off, src + 1, 1)
    off = np.cumsum(off).astype(np.int32)
    assert np.array_equal(solver.step_cc(off, dst.astype(np.int32), team=team), oracle.connected_components(off, dst))


@pytest.mark.parametrize("team", TEAMS)
@pytest.mark.parametrize("tf", (0.5, 2.0, 50.0))
@pytest.mark.parametrize("L", (3, 4, 5))
@pytest.mark.parametrize("g", GRAPHS, ids=IDS)
def test_cycles(solver, oracle, g, L, tf, team):
    """Triangle buffers agree slot for slot, truncated budgets included."""
    _, i, j, c = g
    G, r, co, w, rows, cols = _G(oracle, i, j, c)
    ot, oraw = oracle.conflicted_cycles(G, L, tf)
    gt, graw = solver.step_cycles(r, co, w, rows, cols, L, tf, team=team)
    assert graw == oraw
    assert np.array_equal(gt, ot)


@pytest.mark.parametrize("team", TEAMS)
@pytest.mark.parametrize("g", GRAPHS, ids=IDS)
def test_message_passing(solver, oracle, g, team):
    _, i, j, c = g
    G, r, co, w, rows, cols = _G(oracle, i, j, c)
    tri, _ = oracle.conflicted_cycles(G, 5, 3.0)
    if len(tri) == 0:
        pytest.skip("no conflicted cycles")
    mp = oracle.MessagePassing(G, tri[:, 0], tri[:, 1], tri[:, 2])
    lb0 = mp.lower_bound()
    for _ in range(4):
        mp.iteration()
    lb1 = mp.lower_bound()
    er, ec, ew, _ = mp.edges()
    glb0, glb1, gr, gc, gw = solver.step_mp(r, co, w, rows, cols, tri, 4, team=team)
    assert np.array_equal(gr, er) and np.array_equal(gc, ec)
    assert np.array_equal(gw, ew)
    assert glb0 == lb0 and glb1 == lb1


@pytest.mark.parametrize("team", TEAMS)
@pytest.mark.parametrize("g", GRAPHS, ids=IDS)
def test_dual(solver, oracle, g, team):
    _, i, j, c = g
    G, r, co, w, rows, cols = _G(oracle, i, j, c)
    D, lb, _ = oracle.dual_solver(G, 5, 10, 2.0, 2)
    dr, dc, dw = D.arrays()
    glb, gr, gc, gw, grows, gcols = solver.step_dual(r, co, w, rows, cols, 5, 10, 2.0, 2, team=team)
    assert np.array_equal(gr, dr) and np.array_equal(gc, dc) and np.array_equal(gw, dw)
    assert (grows, gcols) == D.dims
    assert glb == lb


@pytest.mark.parametrize("team", TEAMS)
@pytest.mark.parametrize("n", (0, 1, 31, 4096, 4097, 1_000_003))
def test_csum(solver, oracle, n, team):
    x = np.random.default_rng(n).normal(size=n).astype(np.float32) * 100
    assert solver.step_csum(x, team=team) == oracle.csum(x)


@pytest.mark.parametrize("team", TEAMS)
@pytest.mark.parametrize("n,bits", [(1, 8), (1000, 5), (100_000, 20), (300_001, 44), (1_000_000, 3),
                                    (3_000_017, 44)])
def test_radix_sort_is_stable(solver, n, bits, team):
    rng = np.random.default_rng(bits)
    keys = rng.integers(0, 1 << bits, size=n, dtype=np.uint64)
    vals = np.arange(n, dtype=np.int32)
    gk, gv = solver.step_sort(keys, vals, bits, team=team)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(gk, keys[order])
    assert np.array_equal(gv, vals[order])


@pytest.mark.parametrize("team", TEAMS)
def test_radix_sort_skips_constant_digits(solver, team):
    """Digits that are equal in every key leave the order as it is."""
    rng = np.random.default_rng(5)
    keys = (rng.integers(0, 256, size=200_000, dtype=np.uint64) << np.uint64(16)) | np.uint64(7)
    vals = np.arange(len(keys), dtype=np.int32)
    gk, gv = solver.step_sort(keys, vals, 32, team=team)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(gk, keys[order])
    assert np.array_equal(gv, vals[order])
