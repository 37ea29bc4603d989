"""Host-side checks that need no GPU: the C ABI library loads and exports
every entry point declared in include/*.h, the options mirror the reference's
presets, and the text front ends parse like the reference."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    from rama_b200 import _lib, build

    build.build()
    return _lib.load()


def declared_functions():
    names = set()
    with open(os.path.join(ROOT, "include", "rama_b200.h")) as f:
        txt = f.read()
    for m in re.finditer(r"^\s*(?:const\s+)?(?:int|void|char)\s*\*?\s*(rama_\w+)\s*\(", txt, re.M):
        names.add(m.group(1))
    return names


def test_exports_every_declared_symbol(lib):
    from rama_b200 import _lib

    names = declared_functions()
    assert names == set(_lib.EXPORTS)
    for n in names:
        assert hasattr(lib, n), n


@pytest.mark.parametrize("mode,vals", [
    (None, (5, 10, 3, 5, 1, 0)),
    ("PD", (5, 10, 3, 5, 1, 0)),
    ("P", (0, 0, 0, 0, 1, 0)),
    ("PD+", (5, 10, 5, 10, 1, 0)),
    ("D", (5, 10, 3, 5, 5, 1)),
    ("bogus", (5, 10, 3, 5, 1, 0)),
])
def test_option_presets(lib, mode, vals):
    # include/multicut_solver_options.h:22-53 of the reference
    from rama_b200 import _lib

    o = _lib.options(mode)
    got = (o.max_cycle_length_lb, o.num_dual_itr_lb, o.max_cycle_length_primal, o.num_dual_itr_primal,
           o.num_outer_itr_dual, o.only_compute_lb)
    assert got == vals
    assert abs(o.mean_multiplier_mm - 0.05) < 1e-7 and abs(o.matching_thresh_crossover_ratio - 0.05) < 1e-7
    assert o.tri_memory_factor == 2.0 and o.max_time_sec == -1


def test_rama_py_options(lib, capsys):
    import rama_py

    o = rama_py.multicut_solver_options("PD+")
    assert "PD+ solver" in capsys.readouterr().out
    assert (o.max_cycle_length_primal, o.num_dual_itr_primal) == (5, 10)
    o2 = rama_py.multicut_solver_options(5, 10, 3, 5, 1, 0.05, 0.05, 2.0, False, -1, False)
    assert o2.num_outer_itr_dual == 1 and o2.max_time_sec == -1
    assert repr(o2).startswith("<multicut_solver_options>:max_cycle_length_lb: 5, num_dual_itr_lb: 10")
    assert "mean_multiplier_mm: 0.050000" in repr(o2)


def test_read_multicut_file(tmp_path):
    import rama_py

    p = tmp_path / "a.txt"
    p.write_text("MULTICUT\n0 1 1.5\n1 2 -2\n0 2 0.25\n")
    assert rama_py.read_multicut_file(str(p)) == ([0, 1, 0], [1, 2, 2], [1.5, -2.0, 0.25])
    q = tmp_path / "b.txt"
    q.write_text("GRAPH\n0 1 1\n")
    with pytest.raises(RuntimeError, match="first line must be 'MULTICUT'"):
        rama_py.read_multicut_file(str(q))
    with pytest.raises(RuntimeError, match="Could not open"):
        rama_py.read_multicut_file(str(tmp_path / "missing.txt"))


def test_cli_arguments(lib, tmp_path):
    from rama_b200 import build

    build.build_cli()
    r = subprocess.run([build.CLI, "--help"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "max_cycle_dual" in r.stdout
    r = subprocess.run([build.CLI, "-f", str(tmp_path / "nope.txt")], capture_output=True, text=True, timeout=60)
    assert r.returncode != 0 and "Path does not exist" in r.stderr
    f = tmp_path / "g.txt"
    f.write_text("MULTICUT\n0 1 1\n")
    r = subprocess.run([build.CLI, str(f), "7"], capture_output=True, text=True, timeout=60)
    assert r.returncode != 0 and "not in range" in r.stderr
