"""Parity with the reference solver itself, at the benchmark configurations.

The reference (pawelswoboda/RAMA) is built from its own sources for sm_100a
(oracle/build_ref.sh -> oracle/_ref/librama_ref.so) and run on the same GPU
and the same inputs.  The inputs are bounded samples of the benchmark
configurations, from the same generators and seeds:

  c1   2-D grid 64x64 (the whole configuration, 8,064 edges)
  c2s  3-D grid 64x64x32 + long range (753,664 edges; C2 is 256x256x64)
  c3s  k-NN graph, 20,000 points, k = 20 (220,524 edges; C3 has 1M points)
  c4s  the first 16 graphs of the 512-graph Delaunay batch

Checked against the reference (src/rama_cuda.cu:64-164 and the steps it
calls):
  * bit for bit: the sorted graph (dCOO init), the matching contraction map,
    the contracted edge keys, connected-component labels, the forest
    contraction map, and the triangle sets of the conflicted-cycle search
    when the budget does not truncate;
  * contracted costs within float rounding (the reference sums parallel
    edges in float, this solver in double rounded once);
  * message passing on the same triangles: bounds within 1e-4 relative;
  * full solves: every labelling is a valid multicut whose clusters are
    connected in the input graph; the bound never exceeds the objective; in
    mode P the objective is within 0.1 % of the reference's; in mode D with a
    budget that never truncates, the bound is within 1e-4 of the reference's.
"""
import numpy as np
import pytest

from rama_b200 import instances

pytestmark = pytest.mark.gpu


def _cases():
    b = instances.delaunay_batch(seed=1004)
    return {
        "c1": instances.grid2d(64, 64, seed=1001),
        "c2s": instances.grid3d_longrange(64, 64, 32, seed=1002),
        "c3s": instances.knn_rgg(20_000, 20, seed=1003),
        "c4s": [b.instance(k) for k in range(16)],
    }


_CACHE = {}


def case(name):
    if not _CACHE:
        _CACHE.update(_cases())
    return _CACHE[name]


def single_graphs():
    """(id, i, j, c): the single-instance samples and 4 of the Delaunay graphs."""
    out = [(n, *case(n)) for n in ("c1", "c2s", "c3s")]
    out += [("c4s_%d" % k, *case("c4s")[k]) for k in (0, 5, 10, 15)]
    return out


IDS = ["c1", "c2s", "c3s", "c4s_0", "c4s_5", "c4s_10", "c4s_15"]


@pytest.fixture(scope="module")
def graphs():
    return {g[0]: g[1:] for g in single_graphs()}


@pytest.fixture(scope="module")
def inits(ref, graphs):
    """The reference's sorted graph of every sample."""
    return {k: ref.init(*v) for k, v in graphs.items()}


def _norm_tris(t):
    t = np.sort(np.asarray(t, np.int64).reshape(-1, 3), axis=1)
    t = t[(t[:, 0] != t[:, 1]) & (t[:, 1] != t[:, 2])]
    return np.unique(t, axis=0)


def _connected_clusters(i, j, labels):
    """Every cluster of `labels` is connected by input edges inside it."""
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components

    n = len(labels)
    keep = labels[i] == labels[j]
    A = coo_matrix((np.ones(int(keep.sum())), (i[keep], j[keep])), shape=(n, n))
    ncc, _ = connected_components(A, directed=False)
    return ncc == len(np.unique(labels))


def _objective(i, j, c, labels):
    cut = labels[i] != labels[j]
    return float(np.sum(c[cut].astype(np.float64)))


@pytest.mark.parametrize("name", IDS)
def test_init_bit_exact(solver, inits, graphs, name):
    r, co, w, rows, cols = inits[name]
    gr, gc, gw, grows, gcols = solver.step_init(*graphs[name], team=2)
    assert np.array_equal(gr, r) and np.array_equal(gc, co)
    assert np.array_equal(gw, w)
    assert (grows, gcols) == (rows, cols)


@pytest.mark.parametrize("name", IDS)
def test_matching_map_bit_exact(solver, ref, inits, name):
    r, co, w, rows, cols = inits[name]
    rm, rnr = ref.matching(r, co, w, rows, cols, 0.05)
    gm, gnr = solver.step_matching(r, co, w, rows, cols, 0.05, team=2)
    assert gnr == rnr
    assert np.array_equal(gm, rm)


@pytest.mark.parametrize("name", IDS)
def test_contraction_keys_bit_exact(solver, ref, inits, name):
    r, co, w, rows, cols = inits[name]
    m, _ = solver.step_matching(r, co, w, rows, cols, 0.05, team=2)
    rr, rc, rw, rrows, rcols = ref.contract(r, co, w, rows, cols, m)
    gr, gc, gw, grows, gcols = solver.step_contract(r, co, w, rows, cols, m, team=2)
    assert np.array_equal(gr, rr) and np.array_equal(gc, rc)
    assert (grows, gcols) == (rrows, rcols)
    # parallel edges: float sum (reference) vs double sum rounded once (here)
    assert np.allclose(gw, rw, rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("name", IDS)
def test_cc_labels_bit_exact(solver, ref, inits, name):
    r, co, w, rows, cols = inits[name]
    n = max(rows, cols)
    pos = w > 0
    a = np.concatenate([r[pos], co[pos]])
    b = np.concatenate([co[pos], r[pos]])
    order = np.lexsort((b, a))
    a, b = a[order], b[order]
    off = np.searchsorted(a, np.arange(n + 1)).astype(np.int32)
    adj = b.astype(np.int32)
    assert np.array_equal(solver.step_cc(off, adj, team=2), ref.cc(off, adj))


@pytest.mark.parametrize("name", IDS)
def test_forest_contraction_map_bit_exact(solver, ref, inits, name):
    r, co, w, rows, cols = inits[name]
    rm, rnr = ref.woc(r, co, w, rows, cols)
    gm, gnr = solver.step_woc(r, co, w, rows, cols, team=2)
    assert gnr == rnr
    assert np.array_equal(gm, rm)


def _rep_count(w):
    """Repulsive edges of the cycle search (src/conflicted_cycles_cuda.cu:170-174)."""
    return int(np.sum(w < np.min(w) * np.float32(1e-4)))


def _untruncated_search(solver, r, co, w, rows, cols, L):
    """This solver's L-cycle search with a budget factor large enough that
    nothing is truncated; returns (triangles, factor)."""
    R = max(_rep_count(w), 1)
    f = 2.0
    for _ in range(4):
        t, raw = solver.step_cycles(r, co, w, rows, cols, L, tri_factor=f, team=2)
        if raw <= int(np.float32(f) * np.float32(R)):
            return t, f
        f *= 8.0  # a truncated search reports budget + 1, not the full count
    raise AssertionError("the cycle search still truncates at factor %g" % f)


@pytest.mark.parametrize("L", (3, 4))
@pytest.mark.parametrize("name", IDS)
def test_triangle_sets_bit_exact_untruncated(solver, ref, inits, name, L):
    r, co, w, rows, cols = inits[name]
    gt, f = _untruncated_search(solver, r, co, w, rows, cols, L)
    rt = ref.conflicted_cycles(r, co, w, rows, cols, L, tri_factor=f)
    assert np.array_equal(_norm_tris(gt), _norm_tris(rt))


@pytest.mark.parametrize("name", IDS)
def test_message_passing_bound_within_1e4(solver, ref, inits, name):
    r, co, w, rows, cols = inits[name]
    gt, _ = _untruncated_search(solver, r, co, w, rows, cols, 3)
    tris = _norm_tris(gt).astype(np.int32)
    if len(tris) == 0:
        pytest.skip("no conflicted 3-cycle in this sample")
    glb0, glb1, _, _, _ = solver.step_mp(r, co, w, rows, cols, tris, 10, team=2)
    rlb0, rlb1, _, _, _ = ref.mp(r, co, w, rows, cols, tris, False, 10)
    assert abs(glb0 - rlb0) <= 1e-4 * abs(rlb0)
    assert abs(glb1 - rlb1) <= 1e-4 * abs(rlb1)
    assert glb1 >= glb0 - 1e-9 * abs(glb0)


def _solve_pairs(solver, ref, mode, names, **kw):
    out = []
    for name in names:
        graphs = case(name) if name == "c4s" else [case(name)]
        for (i, j, c) in graphs:
            lab, lb, _ = solver.solve(i, j, c, mode=mode, **kw)
            rlab, rlb, _ = ref.rama(i, j, c, mode, **kw)
            out.append((name, i, j, c, lab, lb, rlab, rlb))
    return out


@pytest.mark.parametrize("name", ("c1", "c2s", "c3s", "c4s"))
def test_mode_p_objective_within_0p1_percent(solver, ref, name):
    for _, i, j, c, lab, lb, rlab, rlb in _solve_pairs(solver, ref, "P", [name]):
        N = int(max(i.max(), j.max())) + 1
        assert len(lab) == N and lab.min() >= 0
        assert _connected_clusters(i, j, lab)
        obj, robj = _objective(i, j, c, lab), _objective(i, j, c, rlab)
        assert abs(obj - robj) <= 1e-3 * max(1.0, abs(robj)), (obj, robj)
        assert lb <= obj + 1e-6 * abs(obj)
        assert abs(lb - rlb) <= 1e-4 * abs(rlb)


@pytest.mark.parametrize("name", ("c1", "c2s", "c3s", "c4s"))
def test_mode_pd_valid_multicut_and_bound_below_objective(solver, ref, name):
    """Every labelling induces a valid multicut (the edges between different
    labels; no cycle crosses it exactly once).  Clusters need not be connected
    in the input graph in this mode, for the reference either: message passing
    adds the triangles' chords to the graph, and a contraction along a chord
    joins nodes that no input edge joins."""
    for _, i, j, c, lab, lb, rlab, rlb in _solve_pairs(solver, ref, "PD", [name]):
        N = int(max(i.max(), j.max())) + 1
        assert len(lab) == N and lab.min() >= 0
        obj, robj = _objective(i, j, c, lab), _objective(i, j, c, rlab)
        assert lb <= obj + 1e-6 * abs(obj)
        assert rlb <= robj + 1e-4 * abs(robj)


@pytest.mark.parametrize("name", ("c1", "c2s", "c3s", "c4s"))
def test_mode_d_untruncated_bound_within_1e4(solver, ref, name):
    """D mode on 3-cycles with a budget that holds every emission: neither
    side truncates, so both bound the same triangle sets."""
    kw = dict(max_cycle_length_lb=3, tri_memory_factor=200.0)
    for _, i, j, c, lab, lb, rlab, rlb in _solve_pairs(solver, ref, "D", [name], **kw):
        assert abs(lb - rlb) <= 1e-4 * max(1.0, abs(rlb)), (lb, rlb)


@pytest.mark.parametrize("name", ("c3s", "c4s"))
def test_mode_d_truncated_bound_not_below_reference(solver, ref, name):
    """D mode as configured (3- to 5-cycles, budget 2 x repulsive edges): the
    budget truncates, and the reference keeps whichever triangles its atomics
    admit (its bound varies from run to run).  The canonical round-robin
    truncation here must give a bound no worse than the reference's worst of
    two runs, less 0.1 %."""
    for _, i, j, c, lab, lb, rlab, rlb in _solve_pairs(solver, ref, "D", [name]):
        _, rlb2, _ = ref.rama(i, j, c, "D")
        worst = min(rlb, rlb2)
        assert lb >= worst - 1e-3 * abs(worst), (lb, rlb, rlb2)
