"""Pins the CPU oracle (oracle/rama_oracle.c) without a GPU.

1. Every known-answer test of the reference's own test suite (test/*.cu and
   test/*.py in pawelswoboda/RAMA), restated on the oracle.
2. Fixtures produced by the reference itself on seeded inputs
   (tests/golden/ref_fixtures.npz, made by tests/golden/make_ref_fixtures.py
   with the reference built from source): integer steps bit-exact, float steps
   within the reference's own float tolerance, triangle sets compared where the
   reference's triangle budget was not exhausted (beyond it the reference keeps
   a scheduling-dependent subset).
"""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden", "ref_fixtures.npz")


# ---------------------------------------------------------------- known answers
def test_compute_offsets(oracle):
    # test/compute_offsets_test.cu:8-33
    assert oracle.compute_offsets([0, 1, 2, 2, 3, 4, 4], 4).tolist() == [0, 1, 2, 4, 5, 7]
    assert oracle.compute_offsets([2, 2, 4, 4, 4, 5, 7, 7], 7).tolist() == [0, 0, 0, 2, 2, 5, 6, 6, 8]


def test_compress_label_sequence(oracle):
    # unique/invert semantics of test/compute_unique_test.cu:8-23 through the
    # label compression used by every contraction map
    out = oracle.compress_label_sequence([4, 0, 4, 2, 2], 4)
    assert out.tolist() == [2, 0, 2, 1, 1]


def test_connected_components(oracle):
    # test/cc_gpu_test.cu:56-68
    for off, cols, ncc in (([0, 1, 2, 4, 5, 6], [1, 0, 3, 4, 2, 2], 2), ([0, 0, 1, 2], [2, 1], 2)):
        lab = oracle.connected_components(off, cols)
        assert len(set(lab.tolist())) == ncc
        for v in range(len(off) - 1):
            for k in range(off[v], off[v + 1]):
                assert lab[cols[k]] == lab[v]
        # canonical: label = smallest vertex of the component
        assert all(lab[v] <= v for v in range(len(lab)))


def test_matching_count(oracle):
    # test/maximum_matching_vertex_based_test.cu:10-31
    g = oracle.Graph.from_edges([0, 1, 0, 3, 3], [1, 2, 2, 0, 1], [2.0, 3.0, -1.0, 1, 2])
    _, nr = oracle.matching(g, 0.0)
    assert nr == 4


@pytest.mark.parametrize("case,expected", [
    (([0, 1, 2], [1, 2, 0], [-1, 2, 1]), (1, 1, 1)),
    (([0, 1, 2, 3], [1, 2, 3, 0], [-1, 2, 1, 3]), (0, 2, 2)),
    (([0, 1, 2, 3], [1, 2, 3, 0], [-1, -2, 1, 3]), (0, 0, 0)),
    (([0, 1, 2, 3, 4], [1, 2, 3, 4, 0], [-1, 2, 1, 3, 2]), (0, 0, 3)),
])
def test_conflicted_cycle_counts(oracle, case, expected):
    # test/conflicted_cycles_test.cu:28-110 (budget factor 10)
    g = oracle.Graph.from_edges(*case)
    got = tuple(oracle.conflicted_cycles(g, L, 10.0)[1] for L in (3, 4, 5))
    assert got == expected


def test_message_passing_lb(oracle):
    # test/multicut_message_passing_test.cu:6-29
    g = oracle.Graph.from_edges([0, 0, 0, 1, 2], [1, 2, 3, 3, 3], [1.0, 1.0, -2.0, 1.0, 1.0])
    mp = oracle.MessagePassing(g, [0, 0], [1, 2], [3, 3])
    assert abs(mp.lower_bound() - (-2.0)) <= 1e-6
    mp.send_messages_to_triplets()
    for _ in range(3):
        mp.iteration()
    assert abs(mp.lower_bound()) <= 1e-6


@pytest.mark.parametrize("i,j,c,apart", [
    ([0, 1, 1, 0, 0], [1, 2, 3, 3, 2], [2.0, 3.0, 1.0, -3, -2], [(0, 3), (0, 2)]),
    ([0, 1, 1, 0, 0, 0, 3, 3, 3], [1, 2, 3, 3, 2, 4, 4, 5, 2], [2.0, 3.0, 1.0, -3, -2, 0.5, 0.75, 0.9, 0.8],
     [(0, 3), (0, 2)]),
    ([0, 1, 1, 0, 3, 3, 3, 1, 0, 0], [1, 2, 3, 4, 4, 5, 2, 5, 2, 3], [2.0, 3.0, 1.0, 0.5, 0.75, 0.9, 0.8, -2, -3, -1],
     [(1, 5), (0, 2), (0, 3)]),
])
def test_woc_separates_repulsive_pairs(oracle, i, j, c, apart):
    # test/edge_contractions_woc_test.cu:9-80
    m, _ = oracle.woc(oracle.Graph.from_edges(i, j, c))
    for a, b in apart:
        assert m[a] != m[b]


def test_full_solve_runs(oracle):
    # test/rama_cuda_test.cu:6-12 and test/test_pytorch.py (mode P)
    lab, lb, _ = oracle.solve([0, 0, 1], [1, 2, 2], [1.5, -3.0, 1.0], "PD")
    assert len(lab) == 3
    lab, lb, _ = oracle.solve([0, 1, 2], [1, 2, 0], [1.1, -2, 3], "P")
    assert lab.tolist() == [0, 1, 0]


# ---------------------------------------------------------------- reference fixtures
@pytest.fixture(scope="module")
def F():
    return np.load(GOLD)


def _g(F, name, key):
    return F[f"{name}/{key}"]


def _norm_tris(t):
    t = np.sort(np.asarray(t).reshape(-1, 3), axis=1)
    if len(t) == 0:
        return set()
    t = t[(t[:, 0] != t[:, 1]) & (t[:, 1] != t[:, 2])]
    return set(map(tuple, t.tolist()))


CASES = range(7)


@pytest.mark.parametrize("k", CASES)
def test_fixture_init_contract(oracle, F, k):
    i, j, c = (_g(F, f"init{k}", x) for x in "ijc")
    G = oracle.Graph.from_edges(i, j, c)
    r, co, w = G.arrays()
    assert np.array_equal(r, _g(F, f"init{k}", "row"))
    assert np.array_equal(co, _g(F, f"init{k}", "col"))
    assert np.array_equal(w, _g(F, f"init{k}", "cost"))
    assert list(G.dims) == _g(F, f"init{k}", "dims").tolist()
    H = G.contract(_g(F, f"contract{k}", "map"))
    r2, c2, w2 = H.arrays()
    assert np.array_equal(r2, _g(F, f"contract{k}", "row"))
    assert np.array_equal(c2, _g(F, f"contract{k}", "col"))
    assert list(H.dims) == _g(F, f"contract{k}", "dims").tolist()
    # parallel edges summed: float order differs, tolerance of fp32 summation
    np.testing.assert_allclose(w2, _g(F, f"contract{k}", "cost"), rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("k", CASES)
def test_fixture_matching_woc_msf(oracle, F, k):
    i, j, c = (_g(F, f"init{k}", x) for x in "ijc")
    G = oracle.Graph.from_edges(i, j, c)
    m, nr = oracle.matching(G, 0.05)
    assert np.array_equal(m, _g(F, f"matching{k}", "map"))
    assert nr == _g(F, f"matching{k}", "nr")[0]
    m, nr = oracle.woc(G)
    assert np.array_equal(m, _g(F, f"woc{k}", "map"))
    assert nr == _g(F, f"woc{k}", "nr")[0]
    mi, mj, mw = (_g(F, f"msf{k}", x) for x in ("i", "j", "w"))
    ids = oracle.msf(mi, mj, mw)
    mine = set(zip(mi[ids].tolist(), mj[ids].tolist()))
    ref = set(zip(_g(F, f"msf{k}", "mi").tolist(), _g(F, f"msf{k}", "mj").tolist()))
    assert mine == ref


WOC5 = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_woc5.npz")


def test_fixture_woc_pentagons(oracle):
    """The optional 5-cycle forest check (the reference's check_pentagons_cuda,
    disabled there) against the reference run with it enabled; the same
    graphs without the check match the reference's default path."""
    if not os.path.exists(WOC5):
        pytest.skip("tests/golden/ref_woc5.npz not generated")
    W = np.load(WOC5)
    cases = sorted({k.split("/")[0] for k in W.files})
    differ = 0
    for g in cases:
        G = oracle.Graph.from_sorted(W[f"{g}/row"], W[f"{g}/col"], W[f"{g}/cost"])
        assert list(G.dims) == W[f"{g}/dims"].tolist()
        m5, n5 = oracle.woc(G, pentagons=True)
        m4, n4 = oracle.woc(G)
        assert np.array_equal(m5, W[f"{g}/map5"]) and n5 == W[f"{g}/nr5"][0], g
        assert np.array_equal(m4, W[f"{g}/map4"]) and n4 == W[f"{g}/nr4"][0], g
        differ += not np.array_equal(W[f"{g}/map5"], W[f"{g}/map4"])
    assert differ > 0  # the check changes the result on some of these graphs


@pytest.mark.parametrize("k", CASES)
@pytest.mark.parametrize("L", (3, 4, 5))
def test_fixture_cycles(oracle, F, k, L):
    i, j, c = (_g(F, f"init{k}", x) for x in "ijc")
    G = oracle.Graph.from_edges(i, j, c)
    tri, raw = oracle.conflicted_cycles(G, L, 50.0)
    R = int(np.sum(G.arrays()[2] < np.float32(np.min(G.arrays()[2]) * np.float32(1e-4))))
    budget = int(np.float32(50.0) * np.float32(R))
    rt = _g(F, f"cycles{k}_{L}", "tri")
    if raw > budget:
        pytest.skip("triangle budget exhausted: the reference keeps a scheduling-dependent subset")
    assert raw == len(rt)
    assert _norm_tris(tri) == _norm_tris(rt)


@pytest.mark.parametrize("k", CASES)
def test_fixture_message_passing(oracle, F, k):
    if f"mp{k}/tri" not in F.files:
        pytest.skip("no triangles")
    i, j, c = (_g(F, f"init{k}", x) for x in "ijc")
    G = oracle.Graph.from_edges(i, j, c)
    tn = _g(F, f"mp{k}", "tri")
    mp = oracle.MessagePassing(G, tn[:, 0], tn[:, 1], tn[:, 2])
    lb0 = mp.lower_bound()
    mp.send_messages_to_triplets()
    for _ in range(3):
        mp.iteration()
    lb1 = mp.lower_bound()
    r, co, w, _ = mp.edges()
    assert np.array_equal(r, _g(F, f"mp{k}", "row"))
    assert np.array_equal(co, _g(F, f"mp{k}", "col"))
    assert abs(lb0 - _g(F, f"mp{k}", "lb0")[0]) <= 1e-5 * max(1.0, abs(lb0))
    assert abs(lb1 - _g(F, f"mp{k}", "lb1")[0]) <= 1e-4 * max(1.0, abs(lb1))
    np.testing.assert_allclose(w, _g(F, f"mp{k}", "cost"), rtol=1e-4, atol=1e-4)


@pytest.mark.parametrize("k", CASES)
def test_fixture_dual(oracle, F, k):
    i, j, c = (_g(F, f"init{k}", x) for x in "ijc")
    G = oracle.Graph.from_edges(i, j, c)
    _, raw5 = oracle.conflicted_cycles(G, 5, 50.0)
    w = G.arrays()[2]
    R = int(np.sum(w < np.float32(w.min() * np.float32(1e-4))))
    if raw5 > int(np.float32(50.0) * np.float32(R)):
        pytest.skip("triangle budget exhausted: the reference keeps a scheduling-dependent subset")
    D, lb, _ = oracle.dual_solver(G, 5, 10, 50.0, 1)
    dr, dc, _ = D.arrays()
    assert np.array_equal(dr, _g(F, f"dual{k}", "row"))
    assert np.array_equal(dc, _g(F, f"dual{k}", "col"))
    ref_lb = _g(F, f"dual{k}", "lb")[0]
    assert abs(lb - ref_lb) <= 1e-4 * max(1.0, abs(ref_lb))


def _valid_multicut(i, j, labels):
    """labels cover every node and every cluster is connected in the graph."""
    n = len(labels)
    parent = list(range(n))

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    for a, b in zip(i.tolist(), j.tolist()):
        if labels[a] == labels[b]:
            ra, rb = find(a), find(b)
            if ra != rb:
                parent[ra] = rb
    comps = {}
    for v in range(n):
        comps.setdefault(labels[v], set()).add(find(v))
    return all(len(s) == 1 for s in comps.values())


@pytest.mark.parametrize("k", CASES)
def test_fixture_full_solve_primal(oracle, F, k):
    """Mode P has no dual: the oracle reproduces the reference's labels."""
    i, j, c = (_g(F, f"init{k}", x) for x in "ijc")
    lab, lb, _ = oracle.solve(i, j, c, "P")
    ref_lab = _g(F, f"rama{k}_P", "labels")
    assert np.array_equal(lab, ref_lab)
    assert abs(lb - _g(F, f"rama{k}_P", "lb")[0]) <= 1e-6 * max(1.0, abs(lb))
    assert _valid_multicut(i, j, lab)


def _recorded_spread(F):
    """The reference's run-to-run spread of the PD objective on the spread
    graphs (5 runs each, default budget): (max - min) / |mean|, largest."""
    keys = sorted({k.split("/")[0] for k in F.files if k.startswith("spread")})
    worst = 0.0
    for name in keys:
        o = _g(F, name, "obj")
        worst = max(worst, float((o.max() - o.min()) / max(1.0, abs(o.mean()))))
    return worst


def test_fixture_full_solves_dual_modes(oracle, F):
    """PD and PD+ with the default triangle budget, every fixture graph.  Where
    no cycle search truncated, the oracle's objective equals the reference's.
    Where the budget truncates, the reference keeps whichever triangles its
    atomics admit and its own objective varies from run to run (up to the
    recorded spread, 15.6 % on these graphs); the oracle's objective must lie
    within that spread of the reference's, and must not be worse on average
    (mean signed gap at most 0.5 %).  Every solution is a partition of all
    nodes with LB <= objective.  Clusters need not be connected in the input
    graph: the dual adds triangle chords that later rounds contract, in the
    reference as well."""
    spread = _recorded_spread(F)
    assert spread > 0.0
    gaps = []
    for k in CASES:
        i, j, c = (_g(F, f"init{k}", x) for x in "ijc")
        for mode in ("PD", "PD+"):
            lab, lb, st = oracle.solve(i, j, c, mode)
            assert len(lab) == int(max(i.max(), j.max())) + 1 and lab.min() >= 0
            obj = oracle.objective(i, j, c, lab)
            assert lb <= obj + 1e-6
            ref_obj = oracle.objective(i, j, c, _g(F, f"rama{k}_{mode}", "labels"))
            gap = (obj - ref_obj) / max(1.0, abs(ref_obj))  # > 0: worse than the reference
            if st.truncations == 0:
                assert abs(gap) <= 1e-6, (k, mode, obj, ref_obj)
            assert abs(gap) <= spread, (k, mode, gap, spread)
            gaps.append(gap)
    assert float(np.mean(gaps)) <= 5e-3, gaps


def test_untruncated_full_solves(oracle, F):
    """Full solves with tri_memory_factor=1000: the initial dual never
    exhausts its triangle budget, so the bound is within 1e-4 (relative) of
    the reference's.  The objective is compared within 0.1% where no cycle
    search of the solve overflowed: the primal rounds' dual uses a fixed
    budget factor of 1.0 (src/rama_cuda.cu:92 of the reference), and past it
    the reference's triangle subset, hence its clustering, depends on thread
    scheduling."""
    keys = sorted({k.split("/")[0] for k in F.files if k.startswith("untrunc")})
    if not keys:
        pytest.skip("fixture file predates the untruncated cases")
    compared = 0
    for name in keys:
        i, j, c = (_g(F, name, x) for x in "ijc")
        mode = str(_g(F, name, "mode"))
        lab, lb, st = oracle.solve(i, j, c, mode, tri_memory_factor=1000.0)
        ref_lb = _g(F, name, "lb")[0]
        assert abs(lb - ref_lb) <= 1e-4 * max(1.0, abs(ref_lb)), name
        if mode != "D" and st.truncations == 0:
            obj = oracle.objective(i, j, c, lab)
            ref_obj = oracle.objective(i, j, c, _g(F, name, "labels"))
            assert abs(obj - ref_obj) <= 1e-3 * max(1.0, abs(ref_obj)), name
            compared += 1
    assert compared > 0


def test_reference_spread(oracle, F):
    """The reference disagrees with itself once its triangle budget truncates
    (5 runs, default budget): its objective and bound move from run to run on
    these graphs.  The oracle's bound on each of them lies inside the
    reference's range of bounds, widened by the largest spread of the bound
    seen on any of them."""
    keys = sorted({k.split("/")[0] for k in F.files if k.startswith("spread")})
    if not keys:
        pytest.skip("fixture file predates the spread cases")
    assert _recorded_spread(F) > 1e-3
    lb_spread = 0.0
    for name in keys:
        lb = _g(F, name, "lb")
        lb_spread = max(lb_spread, float((lb.max() - lb.min()) / max(1.0, abs(lb.mean()))))
    assert lb_spread > 1e-4
    for name in keys:
        k = int(name[len("spread"):])
        i, j, c = (_g(F, f"init{k}", x) for x in "ijc")
        _, lb, _ = oracle.solve(i, j, c, "PD")
        ref = _g(F, name, "lb")
        scale = max(1.0, abs(ref.mean()))
        assert ref.min() - lb_spread * scale <= lb <= ref.max() + lb_spread * scale, (name, lb, ref)


@pytest.mark.parametrize("k", range(4))
def test_fixture_cc(oracle, F, k):
    lab = oracle.connected_components(_g(F, f"cc{k}", "offsets"), _g(F, f"cc{k}", "cols"))
    assert np.array_equal(lab, _g(F, f"cc{k}", "labels"))


# ---------------------------------------------------------------- canonical sums
def test_csum_exact_on_integers(oracle):
    x = np.arange(100000, dtype=np.float32) - 50000.5
    assert oracle.csum(x) == float(np.sum(x.astype(np.float64)))


def _lane_tree(vals):
    """32 lanes (value k to lane k mod 32, in order, from +0.0), then the
    pairwise tree over the lanes; in double."""
    lanes = np.zeros(32)
    for k, v in enumerate(vals):
        lanes[k % 32] += float(v)
    off = 1
    while off < 32:
        for l in range(0, 32, 2 * off):
            lanes[l] = lanes[l] + lanes[l + off]
        off *= 2
    return lanes[0]


def test_rsum_matches_definition(oracle):
    rng = np.random.default_rng(5)
    for n in (0, 1, 2, 3, 7, 31, 32, 33, 100, 1000, 4095, 4096):
        x = rng.normal(size=n).astype(np.float32)
        assert oracle.rsum(x) == np.float32(_lane_tree(x))


def test_rsum_of_more_than_4096_values_is_by_chunks(oracle):
    """Beyond 4096 values: each chunk of 4096 is summed as above (in double),
    then the chunk sums are (chunk c to lane c mod 32)."""
    rng = np.random.default_rng(6)
    for n in (4097, 8192, 12289, 40000, 4096 * 33 + 5):
        x = (rng.normal(size=n) * 10.0 ** rng.integers(-3, 4, size=n)).astype(np.float32)
        chunks = [_lane_tree(x[c:c + 4096]) for c in range(0, n, 4096)]
        want = np.float32(_lane_tree(chunks))
        assert oracle.rsum(x) == want
    # and it differs from the unchunked lane sum somewhere (the definition matters)
    x = (rng.normal(size=40000) * 10.0 ** rng.integers(-6, 7, size=40000)).astype(np.float32)
    assert oracle.rsum(x) == np.float32(_lane_tree([_lane_tree(x[c:c + 4096]) for c in range(0, 40000, 4096)]))
