"""Generates tests/golden/ref_woc5.npz: the reference's forest contraction with
its 5-cycle forest check enabled (oracle/ref_harness.cu ref_woc_pentagons,
the reference's own check_pentagons_cuda).  Needs a CUDA device:

    python tests/golden/make_woc5_fixtures.py [out.npz]

Every case stores the sorted input graph, the contraction map with the check
and without it, so the CPU tests can pin the oracle's pentagon option.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import ref_py as R  # noqa: E402
from rama_b200 import instances  # noqa: E402


def main(out):
    F = {}
    k = 0
    for s in range(14):
        n = [20, 40, 80, 150, 300, 60, 500, 1000, 200, 120, 700, 64, 90, 400][s]
        deg = [3, 4, 5, 6, 4, 8, 3, 3, 5, 4, 6, 3, 7, 4][s]
        i, j, c = instances.random_graph(n, deg, seed=300 + s)
        rng = np.random.default_rng(700 + s)
        c = (c + rng.uniform(-1e-3, 1e-3, size=len(c))).astype(np.float32)
        r, co, w, rows, cols = R.init(i, j, c)
        m5, n5 = R.woc(r, co, w, rows, cols, pentagons=True)
        m4, n4 = R.woc(r, co, w, rows, cols, pentagons=False)
        F[f"g{k}/row"], F[f"g{k}/col"], F[f"g{k}/cost"] = r, co, w
        F[f"g{k}/dims"] = np.array([rows, cols])
        F[f"g{k}/map5"], F[f"g{k}/nr5"] = m5, np.array([n5])
        F[f"g{k}/map4"], F[f"g{k}/nr4"] = m4, np.array([n4])
        k += 1
    np.savez_compressed(out, **F)
    print("wrote", out, k, "cases")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden", "ref_woc5.npz"))
