"""Error paths of the solve and the reference-shaped C++ entry points.

* A contraction that leaves a cluster with a negative internal cost is the
  reference's "Found bad contractions" (src/rama_cuda.cu:136-137): the oracle
  and the CUDA path report RAMA_ERR_BAD_CONTRACTION, the C++ host overload of
  include/rama_cuda.h throws std::runtime_error with the reference's message,
  and the reference itself (built here) throws the same.
* tests/cpp/rama_cuda_api.cu uses include/rama_cuda.h like a caller of the
  reference (nvcc, so the thrust::device_vector overload is compiled): built
  on the CPU, run on the GPU.
"""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# two parallel edges 0-1 (+5 and -10) and an edge 1-2: matching (mode P) joins
# 0 and 1 along the +5 edge, and their cluster's internal cost is then -5
BAD = (np.array([0, 0, 1], np.int32), np.array([1, 1, 2], np.int32), np.array([5.0, -10.0, 1.0], np.float32))


def test_oracle_reports_bad_contraction(oracle):
    with pytest.raises(RuntimeError, match="status 5"):
        oracle.solve(*BAD, "P")


@pytest.fixture(scope="module")
def api_binary(tmp_path_factory):
    from rama_b200 import build

    build.build_lib()
    out = str(tmp_path_factory.mktemp("cpp") / "rama_cuda_api")
    lib_dir = os.path.join(ROOT, "rama_b200")
    cmd = ["nvcc", "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
           "-I", os.path.join(ROOT, "include"), "-o", out, os.path.join(ROOT, "tests", "cpp", "rama_cuda_api.cu"),
           "-L", lib_dir, "-l:librama_b200.so", "-Xlinker", "-rpath=" + lib_dir]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-4000:]
    return out


def test_cpp_entry_points_compile(api_binary):
    """Both overloads of include/rama_cuda.h, the thrust one included, build
    against librama_b200.so."""
    assert os.path.exists(api_binary)


@pytest.mark.gpu
def test_cpp_thrust_overload_matches_host_overload(api_binary):
    r = subprocess.run([api_binary, "thrust"], capture_output=True, text=True, timeout=300)
    # the preset constructor prints the reference's banner line first
    assert r.returncode == 0 and r.stdout.splitlines()[-1].startswith("ok"), r.stdout + r.stderr


@pytest.mark.gpu
def test_cpp_host_overload_throws_bad_contraction(api_binary):
    r = subprocess.run([api_binary, "bad"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.splitlines()[-1] == "ok", r.stdout + r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("team", (1, 3, 2))
def test_bad_contraction_through_the_c_abi(solver, team):
    from rama_b200 import _lib

    with pytest.raises(_lib.RamaError) as ei:
        solver.solve(*BAD, mode="P", team=team)
    assert ei.value.code == _lib.RAMA_ERR_BAD_CONTRACTION
    assert "Found bad contractions" in str(ei.value)


@pytest.mark.gpu
def test_reference_throws_the_same(ref):
    with pytest.raises(RuntimeError, match="Found bad contractions"):
        ref.rama(*BAD, "P")
