"""Seeded synthetic multicut instances.

The reference evaluates on public segmentation/clustering datasets that are not
available here; these generators produce instances with the same shapes, sizes
and cost distributions as the benchmark configurations:

* ``grid2d``           64x64 4-neighbour grid, Beta(0.5,0.5) boundary probabilities
* ``grid3d_longrange`` 256x256x64 voxel grid, 6-neighbour + long-range offsets
* ``knn_rgg``          random geometric k-NN graph (k=20 on 1M points)
* ``delaunay``         Delaunay adjacency of random points (region adjacency graphs)
* ``served_pool`` / ``served_stream``  request graphs mixing the above and a
  Poisson arrival stream over them

Every instance is (i, j, costs) with int32 node ids, i != j, each undirected
edge once, and float32 costs; positive cost = attractive.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


def _cost_from_p(p, clip=10.0):
    p = np.clip(p, 1e-12, 1 - 1e-12)
    return np.clip(np.log((1.0 - p) / p), -clip, clip).astype(np.float32)


def grid2d(h=64, w=64, seed=1001):
    """2-D 4-connected grid, ids row-major; p ~ Beta(0.5,0.5) per edge."""
    rng = np.random.default_rng(seed)
    ids = np.arange(h * w, dtype=np.int64).reshape(h, w)
    i = np.concatenate([ids[:, :-1].ravel(), ids[:-1, :].ravel()])
    j = np.concatenate([ids[:, 1:].ravel(), ids[1:, :].ravel()])
    p = rng.beta(0.5, 0.5, size=len(i))
    return i.astype(np.int32), j.astype(np.int32), _cost_from_p(p)


def grid3d_longrange(nx=256, ny=256, nz=64, seed=1002, offsets=((4, 0, 0), (0, 4, 0), (0, 0, 2)),
                     long_scale=0.5):
    """3-D voxel grid with 6-neighbour edges plus long-range offsets.

    b ~ Beta(0.5,0.5) per voxel smoothed by a 3x3x3 box filter; edge
    p = max(b_u, b_v); cost = clip(log((1-p)/p), +-10), long-range x0.5.
    """
    from scipy.ndimage import uniform_filter

    rng = np.random.default_rng(seed)
    b = rng.beta(0.5, 0.5, size=(nx, ny, nz)).astype(np.float64)
    b = uniform_filter(b, size=3, mode="nearest")
    ids = np.arange(nx * ny * nz, dtype=np.int64).reshape(nx, ny, nz)
    I, J, Cs = [], [], []

    def add(dx, dy, dz, scale):
        a = ids[: nx - dx, : ny - dy, : nz - dz]
        c = ids[dx:, dy:, dz:]
        ba = b[: nx - dx, : ny - dy, : nz - dz]
        bc = b[dx:, dy:, dz:]
        p = np.maximum(ba, bc).ravel()
        I.append(a.ravel().astype(np.int32))
        J.append(c.ravel().astype(np.int32))
        Cs.append((_cost_from_p(p) * np.float32(scale)).astype(np.float32))

    for d in ((1, 0, 0), (0, 1, 0), (0, 0, 1)):
        add(*d, 1.0)
    for d in offsets:
        add(*d, long_scale)
    return np.concatenate(I), np.concatenate(J), np.concatenate(Cs)


def knn_rgg(n=1_000_000, k=20, seed=1003, mean=0.3, std=1.0):
    """k nearest neighbours of n uniform points in the unit square, symmetrised."""
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    pts = rng.random((n, 2))
    tree = cKDTree(pts)
    _, nb = tree.query(pts, k=k + 1, workers=-1)
    src = np.repeat(np.arange(n, dtype=np.int64), k)
    dst = nb[:, 1:].ravel().astype(np.int64)
    lo, hi = np.minimum(src, dst), np.maximum(src, dst)
    key = np.unique(lo * n + hi)
    i = (key // n).astype(np.int32)
    j = (key % n).astype(np.int32)
    c = rng.normal(mean, std, size=len(i)).astype(np.float32)
    return i, j, c


def delaunay(npts, rng, mean=0.2, std=1.0, frac_neg=0.05, neg=-5.0):
    """Delaunay adjacency of npts uniform points; costs N(mean,std), a fraction set to `neg`."""
    from scipy.spatial import Delaunay

    pts = rng.random((npts, 2))
    tri = Delaunay(pts).simplices.astype(np.int64)
    e = np.concatenate([tri[:, [0, 1]], tri[:, [0, 2]], tri[:, [1, 2]]])
    lo, hi = e.min(axis=1), e.max(axis=1)
    key = np.unique(lo * npts + hi)
    i = (key // npts).astype(np.int32)
    j = (key % npts).astype(np.int32)
    c = rng.normal(mean, std, size=len(i)).astype(np.float32)
    c[rng.random(len(i)) < frac_neg] = np.float32(neg)
    return i, j, c


@dataclass
class Batch:
    """Disjoint union of instances with per-instance offsets (int32 node ids
    local to each instance; edge_offsets/node_offsets index the packed arrays)."""

    i: np.ndarray
    j: np.ndarray
    c: np.ndarray
    edge_offsets: np.ndarray  # int64, len = count + 1
    node_counts: np.ndarray   # int32, nodes per instance (max id + 1)

    @property
    def count(self):
        return len(self.node_counts)

    def instance(self, k):
        a, b = self.edge_offsets[k], self.edge_offsets[k + 1]
        return self.i[a:b], self.j[a:b], self.c[a:b]


def pack(instances):
    sizes = [len(x[2]) for x in instances]
    off = np.zeros(len(instances) + 1, np.int64)
    off[1:] = np.cumsum(sizes)
    nodes = np.array([int(max(x[0].max(initial=-1), x[1].max(initial=-1)) + 1) for x in instances], np.int32)
    return Batch(np.concatenate([x[0] for x in instances]).astype(np.int32),
                 np.concatenate([x[1] for x in instances]).astype(np.int32),
                 np.concatenate([x[2] for x in instances]).astype(np.float32), off, nodes)


def delaunay_batch(count=512, nmin=500, nmax=20000, seed=1004):
    """`count` Delaunay region-adjacency graphs, n log-uniform in [nmin, nmax]."""
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(math.log(nmin), math.log(nmax), size=count)).astype(np.int64)
    return pack([delaunay(int(n), rng) for n in ns])


def random_graph(n, avg_deg, seed, neg_frac=0.4, scale=1.0):
    """Erdos-Renyi-like simple graph for small parity cases."""
    rng = np.random.default_rng(seed)
    m = int(n * avg_deg / 2)
    a = rng.integers(0, n, size=3 * m + 8)
    b = rng.integers(0, n, size=3 * m + 8)
    keep = a != b
    lo, hi = np.minimum(a[keep], b[keep]), np.maximum(a[keep], b[keep])
    key = np.unique(lo.astype(np.int64) * n + hi)[:m]
    rng.shuffle(key)
    i = (key // n).astype(np.int32)
    j = (key % n).astype(np.int32)
    c = (rng.normal(0.0, 1.0, size=len(i)) * scale).astype(np.float32)
    c[rng.random(len(i)) < neg_frac] *= -1
    # make sure node n-1 has an edge so the label count is n
    return i, j, c


def served_instance(rng, max_edges=None):
    """One request graph of the served mix: a grid cube (side 16..128,
    6-neighbour), a Delaunay graph (1e3..2e6 edges, log-uniform) or a k-NN
    graph (k = 10, 1e4..5e5 nodes, log-uniform), each kind with probability
    1/3; costs N(0.2, 1) with 5% of the edges at -5.  `max_edges` bounds the
    size (quick tests) by drawing smaller parameters, not by cutting edges."""
    kind = int(rng.integers(0, 3))
    lim = float("inf") if max_edges is None else float(max_edges)
    if kind == 0:
        hi = int(min(128, max(16, (lim / 3) ** (1 / 3))))
        return _cube(int(rng.integers(16, hi + 1)), rng)
    if kind == 1:
        ne = math.exp(rng.uniform(math.log(1e3), math.log(min(2e6, max(lim, 1e3)))))
        return delaunay(max(int(ne / 3), 16), rng)
    nn = int(math.exp(rng.uniform(math.log(1e4), math.log(min(5e5, max(lim / 7, 1e4))))))
    return _knn_small(nn, 10, rng)


def served_pool(size=48, seed=1005, max_edges=None):
    """`size` distinct request graphs of the served mix (see served_instance)."""
    rng = np.random.default_rng(seed)
    return [served_instance(rng, max_edges) for _ in range(size)]


def served_stream(num_requests=10000, rate=1000.0, pool_size=48, seed=1006):
    """A Poisson arrival stream over a pool of request graphs: a list of
    (arrival time in seconds, mode, pool index).  Modes P/PD/D at 50/40/10%."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=num_requests))
    modes = rng.choice(["P", "PD", "D"], size=num_requests, p=[0.5, 0.4, 0.1])
    idx = rng.integers(0, pool_size, size=num_requests)
    return [(float(t[k]), str(modes[k]), int(idx[k])) for k in range(num_requests)]


def _cube(side, rng):
    ids = np.arange(side ** 3, dtype=np.int64).reshape(side, side, side)
    I, J = [], []
    for d in ((1, 0, 0), (0, 1, 0), (0, 0, 1)):
        a = ids[: side - d[0], : side - d[1], : side - d[2]]
        b = ids[d[0]:, d[1]:, d[2]:]
        I.append(a.ravel())
        J.append(b.ravel())
    i = np.concatenate(I).astype(np.int32)
    j = np.concatenate(J).astype(np.int32)
    c = rng.normal(0.2, 1.0, size=len(i)).astype(np.float32)
    c[rng.random(len(i)) < 0.05] = np.float32(-5.0)
    return i, j, c


def _knn_small(n, k, rng):
    from scipy.spatial import cKDTree

    pts = rng.random((n, 2))
    _, nb = cKDTree(pts).query(pts, k=k + 1)
    src = np.repeat(np.arange(n, dtype=np.int64), k)
    dst = nb[:, 1:].ravel().astype(np.int64)
    lo, hi = np.minimum(src, dst), np.maximum(src, dst)
    key = np.unique(lo * n + hi)
    i = (key // n).astype(np.int32)
    j = (key % n).astype(np.int32)
    c = rng.normal(0.2, 1.0, size=len(i)).astype(np.float32)
    c[rng.random(len(i)) < 0.05] = np.float32(-5.0)
    return i, j, c
