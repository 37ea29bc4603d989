"""The autotuner of the launch parameters (rama_b200.autotune): its
decisions from timing tables and its cache on the CPU; on the GPU, that the
tuning it chooses leaves every result unchanged."""
import json

import numpy as np
import pytest

from rama_b200 import autotune


def test_pick_fastest_prefers_the_first_of_equal_times():
    assert autotune.pick_fastest({4: 2.0, 8: 1.0, 16: 1.0}) == 8
    assert autotune.pick_fastest({1: 3.0}) == 1


def test_crossover_between_last_loss_and_the_run_of_wins():
    sizes = [1000, 4000, 16000, 64000]
    # the larger team loses at 1k and 4k, wins from 16k on: switch at sqrt(4k * 16k)
    assert autotune.crossover(sizes, [1, 2, 9, 30], [3, 4, 6, 10], default=7) == 8000
    # a win that does not last: the unbroken run starts at 64k
    assert autotune.crossover(sizes, [1, 5, 9, 30], [3, 4, 12, 10], default=7) == int(round((16000 * 64000) ** 0.5))
    assert autotune.crossover(sizes, [5, 5, 5, 5], [1, 1, 1, 1], default=7) == 1000
    assert autotune.crossover(sizes, [1, 1, 1, 1], [5, 5, 5, 5], default=7) == 64001


def test_cache_round_trip(tmp_path):
    p = str(tmp_path / "t.json")
    assert autotune.load_cache(p) == {}
    autotune.save_cache("B200|148|abc", {"tuning": {"cluster_ctas": 8}}, p)
    autotune.save_cache("other|1|x", {"tuning": {"cluster_ctas": 4}}, p)
    d = autotune.load_cache(p)
    assert d["B200|148|abc"]["tuning"]["cluster_ctas"] == 8 and len(d) == 2
    with open(p, "w") as f:
        f.write("not json")
    assert autotune.load_cache(p) == {}


@pytest.mark.gpu
def test_tuned_parameters_give_identical_results(tmp_path):
    """A quick tuning run (which itself checks every trial against the first
    result of its instance), then solves with the default and the tuned
    parameters on every team: identical labels and bounds."""
    from rama_b200 import instances
    from rama_b200.solver import Solver

    entry = autotune.tune(0, budget_s=20.0, quick=True)
    json.dumps(entry, default=str)
    s = Solver(0)
    t = s.handle.tuning()
    for k in autotune.KNOBS:
        setattr(t, k, entry["tuning"][k])
    rng = np.random.default_rng(3)
    graphs = [instances.delaunay(n, rng) for n in (400, 3000, 12000)]
    for g in graphs:
        want = [Solver(0).solve(*g, mode="PD", team=tm)[:2] for tm in (1, 3, 2)]
        s.handle.set_tuning(t)
        got = [s.solve(*g, mode="PD", team=tm)[:2] for tm in (0, 1, 3, 2)]
        for lab, lb in want[1:] + got:
            assert np.array_equal(lab, want[0][0]) and lb == want[0][1]


@pytest.mark.gpu
def test_set_tuning_rejects_values_out_of_range():
    from rama_b200 import _lib
    from rama_b200.solver import Solver

    s = Solver(0)
    t = s.handle.tuning()
    t.cluster_ctas = 3
    with pytest.raises(_lib.RamaError):
        s.handle.set_tuning(t)
    t = s.handle.tuning()
    t.grid_ctas_per_sm = 0
    with pytest.raises(_lib.RamaError):
        s.handle.set_tuning(t)
    t = s.handle.tuning()
    t.cta_threads = 300
    with pytest.raises(_lib.RamaError):
        s.handle.set_tuning(t)


@pytest.mark.gpu
def test_small_cta_kernel_gives_the_same_batch_results():
    """A batch without cluster instances on CTAs of 256 threads (three per SM)
    and on CTAs of 512: the same labels and bounds."""
    from rama_b200 import instances
    from rama_b200.solver import Solver

    b = instances.delaunay_batch(count=40, nmin=300, nmax=6000, seed=17)
    s = Solver(0)
    want, _, rc = s.solve_batch(b, mode="PD")
    assert rc == 0
    t = s.handle.tuning()
    t.cta_threads, t.batch_cluster_min = 256, 1 << 40
    s.handle.set_tuning(t)
    got, _, rc = s.solve_batch(b, mode="PD")
    assert rc == 0
    for (lab, lb), (glab, glb) in zip(want, got):
        assert np.array_equal(lab, glab) and lb == glb
