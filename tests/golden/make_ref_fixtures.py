"""Generates tests/golden/ref_fixtures.npz by running the reference solver.

The reference (pawelswoboda/RAMA) is built from source into
oracle/_ref/librama_ref.so by oracle/build_ref.sh; it needs a CUDA device, so
this script runs on a GPU machine:

    python tests/golden/make_ref_fixtures.py [out.npz]

Every case stores its inputs and the reference's outputs, so the CPU tests in
tests/test_oracle_golden.py can pin the oracle without a GPU.  Inputs are small
seeded random graphs (rama_b200.instances.random_graph / grid2d).
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import ref_py as R  # noqa: E402
from rama_b200 import instances  # noqa: E402


def distinct_costs(c, seed):
    rng = np.random.default_rng(seed)
    return (c + rng.uniform(-1e-3, 1e-3, size=len(c))).astype(np.float32)


def main(out):
    F = {}

    def put(name, **arrs):
        for k, v in arrs.items():
            F[f"{name}/{k}"] = np.asarray(v)

    graphs = []
    for s in range(6):
        n = [20, 40, 80, 150, 300, 60][s]
        deg = [3, 4, 5, 6, 4, 8][s]
        i, j, c = instances.random_graph(n, deg, seed=100 + s)
        graphs.append((i, j, distinct_costs(c, 500 + s)))
    gi, gj, gc = instances.grid2d(12, 12, seed=77)
    graphs.append((gi, gj, gc))

    for k, (i, j, c) in enumerate(graphs):
        r, co, w, rows, cols = R.init(i, j, c)
        put(f"init{k}", i=i, j=j, c=c, row=r, col=co, cost=w, dims=[rows, cols])
        rng = np.random.default_rng(900 + k)
        N = max(rows, cols)
        m = rng.integers(0, max(N // 2, 1), size=N).astype(np.int32)
        # compress like the solver's maps
        _, m = np.unique(m, return_inverse=True)
        m = m.astype(np.int32)
        r2, c2, w2, ro2, co2 = R.contract(r, co, w, rows, cols, m)
        put(f"contract{k}", map=m, row=r2, col=c2, cost=w2, dims=[ro2, co2])
        mm, nr = R.matching(r, co, w, rows, cols, 0.05)
        put(f"matching{k}", map=mm, nr=[nr])
        wm, wn = R.woc(r, co, w, rows, cols)
        put(f"woc{k}", map=wm, nr=[wn])
        pos = w > 0
        a, b, ww = R.msf(r[pos], co[pos], w[pos])
        put(f"msf{k}", i=r[pos], j=co[pos], w=w[pos], mi=a, mj=b, mw=ww)
        for L in (3, 4, 5):
            t = R.conflicted_cycles(r, co, w, rows, cols, L, tri_factor=50.0)
            put(f"cycles{k}_{L}", tri=t)
        t5 = R.conflicted_cycles(r, co, w, rows, cols, 5, tri_factor=50.0)
        tn = np.unique(np.sort(t5, axis=1), axis=0) if len(t5) else np.zeros((0, 3), np.int32)
        tn = tn[(tn[:, 0] != tn[:, 1]) & (tn[:, 1] != tn[:, 2])] if len(tn) else tn
        if len(tn):
            lb0, lb1, mr, mc, mw = R.mp(r, co, w, rows, cols, tn, 1, 3)
            put(f"mp{k}", tri=tn, lb0=[lb0], lb1=[lb1], row=mr, col=mc, cost=mw)
        lb, dr, dc, dw, dro, dco = R.dual(r, co, w, rows, cols, 5, 10, 50.0, 1)
        put(f"dual{k}", lb=[lb], row=dr, col=dc, cost=dw, dims=[dro, dco])
        for mode in ("P", "PD", "PD+", "D"):
            lab, lbv, _ = R.rama(i, j, c, mode)
            put(f"rama{k}_{mode}", labels=lab, lb=[lbv])

    # full solves with a budget the reference never exhausts (tight parity)
    for k, (i, j, c) in enumerate(graphs):
        for mode in ("PD", "PD+", "D"):
            lab, lbv, _ = R.rama(i, j, c, mode, tri_memory_factor=1000.0)
            put(f"untrunc{k}_{mode}", i=i, j=j, c=c, mode=np.asarray(mode), labels=lab, lb=[lbv])

    # the reference's own run-to-run spread with the default budget (its
    # triangle set depends on thread scheduling once the budget is hit)
    for k in (2, 3, 5):
        i, j, c = graphs[k]
        lbs, objs = [], []
        for _ in range(5):
            lab, lbv, _ = R.rama(i, j, c, "PD")
            lbs.append(lbv)
            keep = lab[i] != lab[j]
            objs.append(float(np.sum(c[keep].astype(np.float64))))
        put(f"spread{k}", lb=lbs, obj=objs)

    # component labels on CSR forests / sparse graphs
    for k in range(4):
        rng = np.random.default_rng(1200 + k)
        n = 30 + 40 * k
        m = n // 2 + 5 * k
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
        put(f"cc{k}", offsets=off, cols=dst.astype(np.int32), labels=R.cc(off, dst.astype(np.int32)))

    np.savez_compressed(out, **F)
    print(f"wrote {len(F)} arrays to {out}")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                                            "ref_fixtures.npz"))
