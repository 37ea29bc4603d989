// graph.cuh -- the device graph store (directed COO, row<col, sorted by
// (row,col)) and its coarsening.  Restates dCOO (include/dCOO.h:13-121,
// src/dCOO.cu:14-172) with one radix sort of packed (row,col) keys per
// coarsening and a deterministic segmented sum of parallel edges.
#pragma once
#include "prims.cuh"

namespace rama {

struct Graph {
    int32_t *row, *col;
    float *cost;
    int64_t n;
    int32_t rows, cols;  // dCOO::rows_ / cols_
    float cmin;          // smallest cost of an edge with row != col (NaN: not known)
    __device__ __forceinline__ int32_t max_dim() const { return rows > cols ? rows : cols; }
};

__device__ __forceinline__ float unknown_cost() { return __int_as_float(0x7fc00000); }

// Scratch arrays of a new graph, allocated in the temporaries.
template <class Team>
__device__ Graph graph_alloc(const Team &t, Scratch &sc, int64_t n)
{
    Graph g;
    g.row = sc.arena.take<int32_t>(n + 1);
    g.col = sc.arena.take<int32_t>(n + 1);
    g.cost = sc.arena.take<float>(n + 1);
    g.n = n;
    g.rows = g.cols = 0;
    g.cmin = unknown_cost();
    return g;
}

// Move a graph built in the temporaries into the top slot of the arena
// (the slot ends at the arena's end; the old graph there is dead).  Fails
// (team-uniformly) if the slot would overlap live temporaries.
template <class Team>
__device__ Graph graph_commit(const Team &t, Scratch &sc, const Graph &src)
{
    Arena &a = sc.arena;
    uint64_t bytes = (uint64_t)(src.n + 1) * 12 + 3 * 256;
    uint64_t top = (a.cap - bytes) & ~uint64_t(255);
    Graph g = src;
    if (a.failed || bytes > a.cap || top < a.lo) {
        a.failed = 1;
        return src;
    }
    g.row = reinterpret_cast<int32_t *>(a.base + top);
    g.col = reinterpret_cast<int32_t *>(a.base + top + ((uint64_t)(src.n + 1) * 4 + 255) / 256 * 256);
    g.cost = reinterpret_cast<float *>(a.base + top + 2 * (((uint64_t)(src.n + 1) * 4 + 255) / 256 * 256));
    // source lies in the temporaries, strictly below `top`: no overlap
    for (int64_t e = t.rank(); e < src.n; e += t.size()) {
        g.row[e] = src.row[e];
        g.col[e] = src.col[e];
        g.cost[e] = src.cost[e];
    }
    a.top = top;
    t.sync();
    return g;
}

// dims as in dCOO::init (src/dCOO.cu:47-51): rows = last row + 1,
// cols = max col + 1 (0 for an empty graph); in the same pass, the smallest
// cost of an edge that is not a self-loop (dCOO::min of the graph once its
// diagonal is removed; the cycle search's threshold, src/conflicted_cycles_cuda.cu:170-174)
template <class Team>
__device__ void graph_set_dims(const Team &t, Scratch &sc, char *sm, Graph &g)
{
    if (g.n == 0) {
        g.rows = g.cols = 0;
        g.cmin = unknown_cost();
        return;
    }
    int32_t mc = -1;
    float mn = 3.4e38f;
    team_maxi_minf(
        t, sc, sm, g.n, -1, 3.4e38f, [&](int64_t e) { return g.col[e]; },
        [&](int64_t e) { return g.row[e] != g.col[e] ? g.cost[e] : 3.4e38f; }, mc, mn);
    g.cols = mc + 1;
    g.rows = uread(&g.row[g.n - 1]) + 1;
    g.cmin = mn;
}

__device__ __forceinline__ uint64_t pack_key(int32_t a, int32_t b, int nbits)
{
    return ((uint64_t)(uint32_t)a << nbits) | (uint32_t)b;
}

// dCOO ctor with unsorted input (src/dCOO.cu:38-45): endpoints ordered,
// sorted by (row,col), stable.  Inputs are (i, j, c) of length n.
// By buckets of the smaller endpoint: the bucket sort orders each bucket by
// (larger endpoint, edge index) and carries the cost bits and the bucket
// along, and the sorted edges are written straight into the graph slot.
// Buckets of more than BUCKET_MAX edges go through a stable radix sort of
// their packed (min, max) keys inside the bucket sort; edge lists of 2^31 or
// more take graph_from_edges_sorted (one radix sort of every edge's keys).
template <class Team>
__device__ Graph graph_from_edges_sorted(const Team &t, Scratch &sc, char *sm, const int32_t *i, const int32_t *j,
                                         const float *c, int64_t n);

template <class Team>
__device__ Graph graph_from_edges(const Team &t, Scratch &sc, char *sm, const int32_t *i, const int32_t *j,
                                  const float *c, int64_t n)
{
    if (n == 0 || n >= (int64_t(1) << 31)) return graph_from_edges_sorted(t, sc, sm, i, j, c, n);
    Graph out;
    out.n = n;
    out.rows = out.cols = 0;
    out.cmin = unknown_cost();
    const int32_t mx = team_max<Team, int32_t>(t, sc, sm, n, 0, [&](int64_t e) { return i[e] > j[e] ? i[e] : j[e]; });
    const int nbh = bits_for((uint64_t)(mx > 0 ? mx : 1));
    uint64_t m = sc.arena.mark();
    int2 *lohi = sc.arena.take<int2>(n + 1);
    uint64_t *sk = sc.arena.take<uint64_t>(n + 1);
    int32_t *sbits = sc.arena.take<int32_t>(n + 1);
    int32_t *sbk = sc.arena.take<int32_t>(n + 1);
    int32_t *bst = sc.arena.take<int32_t>((int64_t)mx + 2);
    if (!sc.arena.ok()) return out;
    const bool done = team_bucket_sort_ex(
        t, sc, sm, n, mx + 1,
        [&](int64_t e) -> int64_t {
            const int32_t a = i[e], b = j[e];
            const int32_t lo = a < b ? a : b, hi = a < b ? b : a;
            return ((int64_t)hi << 32) | (uint32_t)lo;
        },
        [&](int64_t e) { return lohi[e].x; },
        [&](int64_t e) -> uint64_t { return ((uint64_t)(uint32_t)lohi[e].y << 32) | (uint64_t)e; },
        [&](int64_t e) { return __float_as_int(c[e]); }, sk, sbits, bst, sbk, -1,
        [&](int64_t e) -> uint64_t { return ((uint64_t)(uint32_t)lohi[e].x << nbh) | (uint32_t)lohi[e].y; },
        2 * nbh, [&](int64_t e, int64_t w) { lohi[e] = make_int2((int32_t)(uint32_t)w, (int32_t)(w >> 32)); });
    if (!done) return out;
    Arena &ar = sc.arena;
    const uint64_t bytes = (uint64_t)(n + 1) * 12 + 3 * 256;
    const uint64_t top = (ar.cap - bytes) & ~uint64_t(255);
    if (ar.failed || bytes > ar.cap || top < ar.lo) {
        ar.failed = 1;
        return out;
    }
    const uint64_t words = ((uint64_t)(n + 1) * 4 + 255) / 256 * 256;
    Graph g;
    g.row = reinterpret_cast<int32_t *>(ar.base + top);
    g.col = reinterpret_cast<int32_t *>(ar.base + top + words);
    g.cost = reinterpret_cast<float *>(ar.base + top + 2 * words);
    g.n = n;
    team_for_batched(
        t, n, [&](int64_t p) { return make_int3(sbk[p], (int32_t)(sk[p] >> 32), sbits[p]); },
        [&](int64_t p, int3 v) {
            g.row[p] = v.x;
            g.col[p] = v.y;
            g.cost[p] = __int_as_float(v.z);
        });
    t.sync();
    graph_set_dims(t, sc, sm, g);
    ar.top = top;
    sc.arena.release(m);
    sc.alg_bytes += 24.0 * (double)n;
    return g;
}

template <class Team>
__device__ Graph graph_from_edges_sorted(const Team &t, Scratch &sc, char *sm, const int32_t *i, const int32_t *j,
                                         const float *c, int64_t n)
{
    Graph out;
    out.n = n;
    out.rows = out.cols = 0;
    int32_t mx = team_max<Team, int32_t>(t, sc, sm, n, 0, [&](int64_t e) { return i[e] > j[e] ? i[e] : j[e]; });
    const int nb = bits_for((uint64_t)mx);
    uint64_t m = sc.arena.mark();
    uint64_t *k1 = sc.arena.take<uint64_t>(n + 1), *k2 = sc.arena.take<uint64_t>(n + 1);
    float *v1 = sc.arena.take<float>(n + 1), *v2 = sc.arena.take<float>(n + 1);
    Graph g = graph_alloc(t, sc, n);
    if (!sc.arena.ok()) return out;
    // sort by (min, max) endpoint, stably: bucket by the smaller endpoint and
    // order each bucket by (larger endpoint, edge index); hub rows of more
    // than BUCKET_MAX edges: LSD radix sort
    bool done = false;
    {
        uint64_t bm = sc.arena.mark();
        int32_t *bst = sc.arena.take<int32_t>((int64_t)mx + 2);
        int32_t *bidx = sc.arena.take<int32_t>(n + 1);
        if (sc.arena.ok() && n < (int64_t(1) << 31)) {
            done = team_bucket_sort(
                t, sc, sm, n, mx + 1, [&](int64_t e) { return i[e] < j[e] ? i[e] : j[e]; },
                [&](int64_t e) -> uint64_t {
                    return ((uint64_t)(uint32_t)(i[e] < j[e] ? j[e] : i[e]) << 32) | (uint64_t)e;
                },
                k2, bidx, bst);
            if (done) {
                for (int64_t b = t.rank(); b <= mx; b += t.size())
                    for (int32_t p = bst[b]; p < bst[b + 1]; ++p)
                        k1[p] = pack_key((int32_t)b, (int32_t)(k2[p] >> 32), nb);
                for (int64_t p = t.rank(); p < n; p += t.size()) v1[p] = c[bidx[p]];
                t.sync();
            }
        }
        sc.arena.release(bm);
    }
    if (!done) {
        for (int64_t e = t.rank(); e < n; e += t.size()) {
            int32_t a = i[e], b = j[e];
            k1[e] = pack_key(a < b ? a : b, a < b ? b : a, nb);
            v1[e] = c[e];
        }
        t.sync();
        team_sort_pairs(t, sc, sm, k1, v1, k2, v2, n, 2 * nb);
    }
    const uint64_t mask = (nb == 0) ? 0 : ((uint64_t(1) << nb) - 1);
    for (int64_t e = t.rank(); e < n; e += t.size()) {
        g.row[e] = (int32_t)(k1[e] >> nb);
        g.col[e] = (int32_t)(k1[e] & mask);
        g.cost[e] = v1[e];
    }
    t.sync();
    graph_set_dims(t, sc, sm, g);
    Graph r = graph_commit(t, sc, g);
    sc.arena.release(m);
    sc.alg_bytes += 24.0 * (double)n;
    return r;
}

// dCOO::contract_cuda (src/dCOO.cu:57-95) followed by has_bad_contractions
// (src/rama_cuda.cu:18-30) and remove_diagonal (src/dCOO.cu:106-116).
// Parallel edges are summed in sorted (stable) order with RSUM.
// Returns the new graph (committed to the top slot); *bad is set if a
// self-loop of negative cost appeared.  Dims are taken before the diagonal
// is removed, as the reference does.
// The edges keyed by their contracted endpoints, sorted: k1[p] = (lo, hi)
// packed with nb bits each, v1[p] = the edge's cost, in (lo, hi) order and,
// for equal keys, in edge order (the order a stable sort leaves; it fixes the
// summation order of parallel edges).  The edges are bucketed by their new
// row lo and each row is ordered by (hi, edge index); rows of more than
// BUCKET_MAX edges send the whole list through the LSD radix sort instead.
// k1/v1 (and the spare k2/v2) hold n + 1 entries; the result ends in k1/v1.
template <class Team>
__device__ void contract_sorted_keys(const Team &t, Scratch &sc, char *sm, const Graph &A, const int32_t *map,
                                     int32_t map_max, int nb, uint64_t *&k1, float *&v1, uint64_t *&k2, float *&v2)
{
    const int64_t n = A.n;
    bool done = false;
    uint64_t m = sc.arena.mark();
    int32_t *bst = sc.arena.take<int32_t>((int64_t)map_max + 2);
    int32_t *bidx = sc.arena.take<int32_t>(n + 1);
    if (sc.arena.ok() && n < (int64_t(1) << 31)) {
        done = team_bucket_sort(
            t, sc, sm, n, map_max + 1,
            [&](int64_t e) {
                const int32_t a = map[A.row[e]], b = map[A.col[e]];
                return a < b ? a : b;
            },
            [&](int64_t e) -> uint64_t {
                const int32_t a = map[A.row[e]], b = map[A.col[e]];
                return ((uint64_t)(uint32_t)(a < b ? b : a) << 32) | (uint64_t)e;
            },
            k2, bidx, bst);
        if (done) {
            for (int64_t b = t.rank(); b <= map_max; b += t.size())
                for (int32_t p = bst[b]; p < bst[b + 1]; ++p) k1[p] = pack_key((int32_t)b, (int32_t)(k2[p] >> 32), nb);
            for (int64_t p = t.rank(); p < n; p += t.size()) v1[p] = A.cost[bidx[p]];
            t.sync();
        }
    }
    sc.arena.release(m);
    if (done) return;
    for (int64_t e = t.rank(); e < n; e += t.size()) {
        int32_t a = map[A.row[e]], b = map[A.col[e]];
        k1[e] = pack_key(a < b ? a : b, a < b ? b : a, nb);
        v1[e] = A.cost[e];
    }
    t.sync();
    team_sort_pairs(t, sc, sm, k1, v1, k2, v2, n, 2 * nb);
}

template <class Team>
__device__ Graph graph_contract_sorted(const Team &t, Scratch &sc, char *sm, const Graph &A, const int32_t *map,
                                       int32_t map_max, int *bad)
{
    const int64_t n = A.n;
    const int nb = bits_for((uint64_t)(map_max > 0 ? map_max : 0));
    uint64_t m = sc.arena.mark();
    uint64_t *k1 = sc.arena.take<uint64_t>(n + 1), *k2 = sc.arena.take<uint64_t>(n + 1);
    float *v1 = sc.arena.take<float>(n + 1), *v2 = sc.arena.take<float>(n + 1);
    int64_t *runpos = sc.arena.take<int64_t>(n + 2);
    int32_t *badflag = sc.arena.take<int32_t>(2);
    Graph out = A;
    if (!sc.arena.ok()) return out;
    if (t.rank() == 0) badflag[0] = 0;
    contract_sorted_keys(t, sc, sm, A, map, map_max, nb, k1, v1, k2, v2);
    // run heads -> run index
    const int64_t nruns = team_compact(
        t, sc, sm, n, [&](int64_t k) { return k == 0 || k1[k] != k1[k - 1]; },
        [&](int64_t k, int64_t r) { runpos[r] = k; });
    if (t.rank() == 0) runpos[nruns] = n;
    t.sync();
    Graph g = graph_alloc(t, sc, nruns);
    int32_t *longq = sc.arena.take<int32_t>(nruns + 1);
    int32_t *nlong = sc.arena.take<int32_t>(2);
    if (!sc.arena.ok()) return out;
    const uint64_t mask = (nb == 0) ? 0 : ((uint64_t(1) << nb) - 1);
    if (t.rank() == 0) nlong[0] = 0;
    t.sync();
    for (int64_t r = t.rank(); r < nruns; r += t.size()) {
        int64_t s = runpos[r], e = runpos[r + 1];
        uint64_t key = k1[s];
        g.row[r] = (int32_t)(key >> nb);
        g.col[r] = (int32_t)(key & mask);
        if (e - s <= 32) {
            g.cost[r] = rsum_serial((int)(e - s), [&](int k) { return v1[s + k]; });
        } else {
            int q = atomicAdd(nlong, 1);
            longq[q] = (int32_t)r;
        }
    }
    t.sync();
    const int32_t nl = uread(nlong);
    for (int64_t q = team_warp(t); q < nl; q += team_nwarps(t)) {
        int64_t r = longq[q];
        int64_t s = runpos[r], e = runpos[r + 1];
        float v = rsum_warp(e - s, [&](int64_t k) { return v1[s + k]; });
        if (lane_id() == 0) g.cost[r] = v;
    }
    t.sync();
    g.n = nruns;
    graph_set_dims(t, sc, sm, g);
    // bad contractions + stable removal of the diagonal
    for (int64_t r = t.rank(); r < nruns; r += t.size())
        if (g.row[r] == g.col[r] && g.cost[r] < 0.0f) badflag[0] = 1;
    Graph h = graph_alloc(t, sc, nruns);
    if (!sc.arena.ok()) return out;
    const int64_t nk = team_compact(
        t, sc, sm, nruns, [&](int64_t r) { return g.row[r] != g.col[r]; },
        [&](int64_t r, int64_t p) {
            h.row[p] = g.row[r];
            h.col[p] = g.col[r];
            h.cost[p] = g.cost[r];
        });
    *bad = uread(badflag);
    h.n = nk;
    h.rows = g.rows;
    h.cols = g.cols;
    h.cmin = g.cmin;
    Graph res = graph_commit(t, sc, h);
    sc.arena.release(m);
    sc.alg_bytes += 20.0 * (double)n + 12.0 * (double)nruns;
    return res;
}

// The contraction (dCOO::contract_cuda + has_bad_contractions +
// remove_diagonal) by buckets of the new row:
//   1. each edge's contracted endpoints (lo, hi) are computed once, with its
//      slot in bucket lo;
//   2. the bucket sort orders every bucket by (hi, edge index), carrying the
//      edge's cost bits and its bucket along (no gather afterwards);
//   3. one scan over the sorted edges finds the heads of the runs of equal
//      (lo, hi) and numbers the runs that are not self-loops; the head's
//      thread sums its run (RSUM in edge order; runs of more than 32 by a
//      warp afterwards) and writes the edge straight into the graph slot at
//      the top of the arena (the old graph there is dead by then), or checks
//      a self-loop's sum for a bad contraction;
//   4. one pass over the new edges gives the largest column and the smallest
//      cost; the rows are the last bucket + 1 (dims are taken before the
//      diagonal goes, as the reference does).
// Buckets of more than BUCKET_MAX edges are sorted by a stable radix sort of
// their packed (lo, hi) keys inside the bucket sort; graph_contract_sorted
// (one radix sort of every edge's packed keys) remains for edge lists of
// 2^31 edges or more.  Both give the same graph bit for bit.
template <class Team>
__device__ Graph graph_contract(const Team &t, Scratch &sc, char *sm, const Graph &A, const int32_t *map,
                                int32_t map_max, int *bad)
{
    const int64_t n = A.n;
    Graph out = A;
    if (n == 0 || n >= (int64_t(1) << 31)) return graph_contract_sorted(t, sc, sm, A, map, map_max, bad);
    const int32_t nbk = map_max + 1;
    const int nbh = bits_for((uint64_t)(map_max > 0 ? map_max : 1));
    uint64_t m = sc.arena.mark();
    int2 *lohi = sc.arena.take<int2>(n + 1);
    uint64_t *sk = sc.arena.take<uint64_t>(n + 1);
    int32_t *sbits = sc.arena.take<int32_t>(n + 1);
    int32_t *sbk = sc.arena.take<int32_t>(n + 1);
    int32_t *bst = sc.arena.take<int32_t>((int64_t)nbk + 2);
    int4 *longq = sc.arena.take<int4>(n / 33 + 2);
    // [0] bad, [1] long runs, [2] largest self-loop column
    int32_t *fl = sc.arena.take<int32_t>(8);
    if (!sc.arena.ok()) return out;
    if (t.rank() == 0) {
        fl[0] = 0;
        fl[1] = 0;
        fl[2] = -1;
    }
    const bool done = team_bucket_sort_ex(
        t, sc, sm, n, nbk,
        [&](int64_t e) -> int64_t {
            const int32_t a = map[A.row[e]], b = map[A.col[e]];
            const int32_t lo = a < b ? a : b, hi = a < b ? b : a;
            return ((int64_t)hi << 32) | (uint32_t)lo;
        },
        [&](int64_t e) { return lohi[e].x; },
        [&](int64_t e) -> uint64_t { return ((uint64_t)(uint32_t)lohi[e].y << 32) | (uint64_t)e; },
        [&](int64_t e) { return __float_as_int(A.cost[e]); }, sk, sbits, bst, sbk, PH_CSORT_SLOT,
        [&](int64_t e) -> uint64_t { return ((uint64_t)(uint32_t)lohi[e].x << nbh) | (uint32_t)lohi[e].y; },
        2 * nbh, [&](int64_t e, int64_t w) { lohi[e] = make_int2((int32_t)(uint32_t)w, (int32_t)(w >> 32)); });
    if (!done) {
        sc.arena.release(m);
        return graph_contract_sorted(t, sc, sm, A, map, map_max, bad);
    }
    // the new graph's slot, sized for at most n edges; it ends at the arena's
    // end, so it lies within the old graph's slot (n is the old edge count)
    Arena &ar = sc.arena;
    const uint64_t bytes = (uint64_t)(n + 1) * 12 + 3 * 256;
    const uint64_t top = (ar.cap - bytes) & ~uint64_t(255);
    if (ar.failed || bytes > ar.cap || top < ar.lo) {
        ar.failed = 1;
        return out;
    }
    // temporaries taken from here on stay below the new slot (when the old
    // graph does not live in the slot, as in a single step, the arena's top
    // is its end)
    if (top < ar.top) ar.top = top;
    const uint64_t words = ((uint64_t)(n + 1) * 4 + 255) / 256 * 256;
    Graph h;
    h.row = reinterpret_cast<int32_t *>(ar.base + top);
    h.col = reinterpret_cast<int32_t *>(ar.base + top + words);
    h.cost = reinterpret_cast<float *>(ar.base + top + 2 * words);
    // 3. heads of the runs: one scan counts every run (high 32 bits) and the
    //    runs that are not self-loops (low 32 bits), writes the row and column
    //    of each new edge and notes each run's start and output slot (-1: a
    //    self-loop).  Then a pass over the runs sums each one, its end being
    //    the next run's start: runs of up to 32 edges by one thread, longer
    //    ones by a warp afterwards.
    auto head = [&](int64_t p) {
        return p == 0 || sbk[p] != sbk[p - 1] || (sk[p] >> 32) != (sk[p - 1] >> 32);
    };
    // lohi is dead after the sort: its two halves hold the runs' starts and slots
    int32_t *runstart = reinterpret_cast<int32_t *>(lohi);
    int32_t *runk = runstart + (n + 1);
    // the largest self-loop column, per thread first: one atomic per warp
    // afterwards instead of one per self-loop run on a single word
    int32_t dloc = -1;
    const int64_t packed = team_scan<Team, int64_t>(
        t, sc, sm, n,
        [&](int64_t p) -> int64_t {
            if (!head(p)) return 0;
            return (int64_t(1) << 32) | ((int32_t)(sk[p] >> 32) != sbk[p] ? 1 : 0);
        },
        [&](int64_t p, int64_t pre, int64_t v) {
            if (!v) return;
            const int64_t k = pre & 0xffffffffll, r = pre >> 32;
            const int32_t b = sbk[p], hi = (int32_t)(sk[p] >> 32);
            runstart[r] = (int32_t)p;
            if (v & 1) {
                runk[r] = (int32_t)k;
                h.row[k] = b;
                h.col[k] = hi;
            } else {
                runk[r] = -1;
                dloc = hi > dloc ? hi : dloc;
            }
        });
    const int64_t nk = packed & 0xffffffffll, nruns = packed >> 32;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const int32_t x = __shfl_xor_sync(FULL, dloc, o);
        dloc = x > dloc ? x : dloc;
    }
    if (lane_id() == 0 && dloc >= 0) atomicMax(&fl[2], dloc);
    const float *cost_sorted = reinterpret_cast<const float *>(sbits);
    // a run's sum goes to its edge; a self-loop's negative sum is a bad contraction
    auto finish = [&](int32_t k, float sum) {
        if (k >= 0)
            h.cost[k] = sum;
        else if (sum < 0.0f)
            fl[0] = 1;
    };
    {
        // four runs a thread at a time: starts and slots, then the sums
        constexpr int U = 4;
        const int64_t S = t.size();
        int64_t r0 = t.rank();
        auto one = [&](int64_t r, int32_t s, int32_t e, int32_t k) {
            const int32_t len = e - s;
            if (len <= RSUM_THREAD_MAX)
                finish(k, rsum_upto8(cost_sorted + s, len));
            else if (len <= 32)
                finish(k, rsum_upto32(cost_sorted + s, len));
            else
                longq[atomicAdd(&fl[1], 1)] = make_int4(s, e, k, 0);
        };
        for (; r0 + (U - 1) * S < nruns; r0 += U * S) {
            int32_t s[U], e[U], k[U];
#pragma unroll
            for (int j = 0; j < U; ++j) {
                const int64_t r = r0 + j * S;
                s[j] = runstart[r];
                e[j] = r + 1 < nruns ? runstart[r + 1] : (int32_t)n;
                k[j] = runk[r];
            }
#pragma unroll
            for (int j = 0; j < U; ++j) one(r0 + j * S, s[j], e[j], k[j]);
        }
        for (; r0 < nruns; r0 += S)
            one(r0, runstart[r0], r0 + 1 < nruns ? runstart[r0 + 1] : (int32_t)n, runk[r0]);
    }
    t.sync();
    // runs of 33..RSUM_CHUNK edges: a warp each.  Longer runs (a cluster's
    // self-loop run can hold a large part of the graph): their chunks of
    // RSUM_CHUNK edges are shared out over every warp of the team, then a warp
    // per run sums its chunk sums -- the same sum as rsum_warp.
    const int32_t nl = uread(&fl[1]);
    int64_t nchunks = 0;
    int32_t *coff = nullptr;
    double *chunk_sum = nullptr;
    if (nl > 0) {
        coff = sc.arena.take<int32_t>((int64_t)nl + 1);
        if (!sc.arena.ok()) return out;
        nchunks = team_scan<Team, int64_t>(
            t, sc, sm, nl,
            [&](int64_t q) -> int64_t {
                const int64_t len = longq[q].y - longq[q].x;
                return len > RSUM_CHUNK ? (len + RSUM_CHUNK - 1) / RSUM_CHUNK : 0;
            },
            [&](int64_t q, int64_t pre, int64_t) { coff[q] = (int32_t)pre; });
        chunk_sum = sc.arena.take<double>(nchunks + 1);
        if (!sc.arena.ok()) return out;
    }
    for (int64_t w = team_warp(t); w < nl + nchunks; w += team_nwarps(t)) {
        if (w < nl) {
            const int4 L = longq[w];
            if (L.y - L.x <= RSUM_CHUNK) {
                const float v = (float)rsum_chunk_warp(L.y - L.x, [&](int64_t x) { return cost_sorted[L.x + x]; });
                if (lane_id() == 0) finish(L.z, v);
            }
        } else {
            // chunk g belongs to the last run q with coff[q] <= g
            const int64_t g = w - nl;
            int32_t lo = 0, hi = nl - 1;
            while (lo < hi) {
                const int32_t mid = (lo + hi + 1) >> 1;
                if (coff[mid] <= g)
                    lo = mid;
                else
                    hi = mid - 1;
            }
            const int4 L = longq[lo];
            const int64_t base = L.x + (g - coff[lo]) * RSUM_CHUNK;
            const int64_t len = L.y - base < RSUM_CHUNK ? L.y - base : RSUM_CHUNK;
            const double d = rsum_chunk_warp(len, [&](int64_t x) { return cost_sorted[base + x]; });
            if (lane_id() == 0) chunk_sum[g] = d;
        }
    }
    t.sync();
    if (nchunks > 0) {
        for (int64_t w = team_warp(t); w < nl; w += team_nwarps(t)) {
            const int4 L = longq[w];
            const int64_t len = L.y - L.x;
            if (len <= RSUM_CHUNK) continue;
            const int64_t c0 = coff[w], nc = (len + RSUM_CHUNK - 1) / RSUM_CHUNK;
            double acc = 0.0;  // lane l: chunks l, l + 32, ... in order
            for (int64_t c = lane_id(); c < nc; c += 32) acc = __dadd_rn(acc, chunk_sum[c0 + c]);
            const float v = (float)rsum_lane_tree(acc);
            if (lane_id() == 0) finish(L.z, v);
        }
        t.sync();
    }
    prof_mark(t, sc, PH_CONTRACT_RUNS);
    *bad = uread(&fl[0]);
    // 4. dims and the smallest cost (every new edge has row < col)
    int32_t mc = -1;
    float mn = 3.4e38f;
    team_maxi_minf(
        t, sc, sm, nk, -1, 3.4e38f, [&](int64_t e) { return h.col[e]; }, [&](int64_t e) { return h.cost[e]; }, mc,
        mn);
    const int32_t dmax = uread(&fl[2]);
    h.n = nk;
    h.rows = uread(&sbk[n - 1]) + 1;
    h.cols = (mc > dmax ? mc : dmax) + 1;
    h.cmin = nk > 0 ? mn : unknown_cost();
    ar.top = top;
    sc.arena.release(m);
    sc.alg_bytes += 20.0 * (double)n + 12.0 * (double)nk;
    return h;
}

// compute_sanitized_graph (include/rama_utils.h:429-466): drop duplicate
// edges (the first occurrence in stable (min,max) order survives), then
// renumber the nodes that have edges to 0..k-1.  Outputs live in the
// temporaries; idmap (size = max id + 1) maps original ids to new ones.
template <class Team>
__device__ int64_t sanitize_edges(const Team &t, Scratch &sc, char *sm, const int32_t *I, const int32_t *J,
                                  const float *Cc, int64_t n, int32_t *&si, int32_t *&sj, float *&sw, int32_t *&idmap,
                                  int32_t &idsize)
{
    int32_t mx = team_max<Team, int32_t>(t, sc, sm, n, 0, [&](int64_t e) { return I[e] > J[e] ? I[e] : J[e]; });
    idsize = mx + 1;
    const int nb = bits_for((uint64_t)mx);
    si = sc.arena.take<int32_t>(n + 1);
    sj = sc.arena.take<int32_t>(n + 1);
    sw = sc.arena.take<float>(n + 1);
    idmap = sc.arena.take<int32_t>((int64_t)idsize + 1);
    uint64_t m = sc.arena.mark();
    uint64_t *k1 = sc.arena.take<uint64_t>(n + 1), *k2 = sc.arena.take<uint64_t>(n + 1);
    float *v1 = sc.arena.take<float>(n + 1), *v2 = sc.arena.take<float>(n + 1);
    if (!sc.arena.ok()) return 0;
    for (int64_t e = t.rank(); e < n; e += t.size()) {
        int32_t a = I[e], b = J[e];
        k1[e] = pack_key(a < b ? a : b, a < b ? b : a, nb);
        v1[e] = Cc[e];
    }
    for (int64_t v = t.rank(); v < idsize; v += t.size()) idmap[v] = 0;
    t.sync();
    team_sort_pairs(t, sc, sm, k1, v1, k2, v2, n, 2 * nb);
    const uint64_t mask = (nb == 0) ? 0 : ((uint64_t(1) << nb) - 1);
    const int64_t u = team_compact(
        t, sc, sm, n, [&](int64_t k) { return k == 0 || k1[k] != k1[k - 1]; },
        [&](int64_t k, int64_t p) {
            int32_t a = (int32_t)(k1[k] >> nb), b = (int32_t)(k1[k] & mask);
            si[p] = a;
            sj[p] = b;
            sw[p] = v1[k];
            idmap[a] = 1;
            idmap[b] = 1;
        });
    team_scan<Team, int64_t>(
        t, sc, sm, idsize, [&](int64_t v) -> int64_t { return idmap[v]; },
        [&](int64_t v, int64_t pre, int64_t) { idmap[v] = (int32_t)pre; });
    for (int64_t e = t.rank(); e < u; e += t.size()) {
        si[e] = idmap[si[e]];
        sj[e] = idmap[sj[e]];
    }
    t.sync();
    sc.arena.release(m);
    return u;
}

// Stable contraction WITHOUT diagonal removal (the raw contract_cuda result,
// for parity tests); result lives in the temporaries.
template <class Team>
__device__ Graph graph_contract_raw(const Team &t, Scratch &sc, char *sm, const Graph &A, const int32_t *map,
                                    int32_t map_max)
{
    const int64_t n = A.n;
    const int nb = bits_for((uint64_t)(map_max > 0 ? map_max : 0));
    uint64_t *k1 = sc.arena.take<uint64_t>(n + 1), *k2 = sc.arena.take<uint64_t>(n + 1);
    float *v1 = sc.arena.take<float>(n + 1), *v2 = sc.arena.take<float>(n + 1);
    int64_t *runpos = sc.arena.take<int64_t>(n + 2);
    Graph out = A;
    if (!sc.arena.ok()) return out;
    contract_sorted_keys(t, sc, sm, A, map, map_max, nb, k1, v1, k2, v2);
    const int64_t nruns = team_compact(
        t, sc, sm, n, [&](int64_t k) { return k == 0 || k1[k] != k1[k - 1]; },
        [&](int64_t k, int64_t r) { runpos[r] = k; });
    if (t.rank() == 0) runpos[nruns] = n;
    t.sync();
    Graph g = graph_alloc(t, sc, nruns);
    if (!sc.arena.ok()) return out;
    const uint64_t mask = (nb == 0) ? 0 : ((uint64_t(1) << nb) - 1);
    for (int64_t r = t.rank(); r < nruns; r += t.size()) {
        int64_t s = runpos[r], e = runpos[r + 1];
        uint64_t key = k1[s];
        g.row[r] = (int32_t)(key >> nb);
        g.col[r] = (int32_t)(key & mask);
        g.cost[r] = (e - s <= 32) ? rsum_serial((int)(e - s), [&](int k) { return v1[s + k]; }) : 0.0f;
    }
    t.sync();
    for (int64_t r = team_warp(t); r < nruns; r += team_nwarps(t)) {
        int64_t s = runpos[r], e = runpos[r + 1];
        if (e - s <= 32) continue;
        float v = rsum_warp(e - s, [&](int64_t k) { return v1[s + k]; });
        if (lane_id() == 0) g.cost[r] = v;
    }
    t.sync();
    g.n = nruns;
    graph_set_dims(t, sc, sm, g);
    return g;
}

// ---------------------------------------------------------------------------
// Symmetric CSR of a (row,col)-sorted directed edge list restricted to the
// edges where keep(e) holds: row v lists its neighbours u<v (increasing u)
// then w>v (increasing w) -- the (row,col) order of the doubled list
// (to_undirected + coo_sorting, include/rama_utils.h:107-131, 287-294).
// Built with one stable radix sort of the kept edges by column.
// ---------------------------------------------------------------------------
struct Csr {
    int32_t nrows;
    int32_t *off;  // nrows + 1
    int32_t *adj;  // 2m
    float *w;      // 2m
    int32_t *eid;  // 2m: index of the directed edge (in the kept order) -- optional
    int64_t m2;
};

template <class Team, class Keep>
__device__ Csr build_symmetric_csr(const Team &t, Scratch &sc, char *sm, const Graph &A, int32_t nrows, Keep keep,
                                   bool with_eid, int64_t *kept_idx_out = nullptr)
{
    Csr C;
    C.nrows = nrows;
    C.m2 = 0;
    // 1. compact kept edges (their order stays (row,col)-sorted)
    int64_t *kidx = kept_idx_out ? kept_idx_out : sc.arena.take<int64_t>(A.n + 1);
    int32_t *deg = sc.arena.take<int32_t>((int64_t)nrows + 1);
    C.off = sc.arena.take<int32_t>((int64_t)nrows + 2);
    if (!sc.arena.ok()) return C;
    for (int64_t v = t.rank(); v <= nrows; v += t.size()) deg[v] = 0;
    const int64_t m = team_compact(t, sc, sm, A.n, keep, [&](int64_t e, int64_t p) { kidx[p] = e; });
    C.m2 = 2 * m;
    C.adj = sc.arena.take<int32_t>(2 * m + 1);
    C.w = sc.arena.take<float>(2 * m + 1);
    C.eid = with_eid ? sc.arena.take<int32_t>(2 * m + 1) : nullptr;
    uint64_t mk = sc.arena.mark();
    uint64_t *k1 = sc.arena.take<uint64_t>(m + 1), *k2 = sc.arena.take<uint64_t>(m + 1);
    int32_t *v1 = sc.arena.take<int32_t>(m + 1), *v2 = sc.arena.take<int32_t>(m + 1);
    int32_t *infill = sc.arena.take<int32_t>((int64_t)nrows + 1);
    int32_t *colstart = sc.arena.take<int32_t>((int64_t)nrows + 1);
    int32_t *rowstart = sc.arena.take<int32_t>((int64_t)nrows + 1);
    if (!sc.arena.ok()) return C;
    // 2. degrees (in + out) and in-degrees (number of u<v entries per row)
    for (int64_t v = t.rank(); v <= nrows; v += t.size()) infill[v] = 0;
    t.sync();
    for (int64_t p = t.rank(); p < m; p += t.size()) {
        int64_t e = kidx[p];
        atomicAdd(&deg[A.row[e]], 1);
        atomicAdd(&deg[A.col[e]], 1);
        atomicAdd(&infill[A.col[e]], 1);
        k1[p] = (uint64_t)(uint32_t)A.col[e];
        v1[p] = (int32_t)p;
    }
    t.sync();
    team_scan<Team, int64_t>(
        t, sc, sm, (int64_t)nrows, [&](int64_t v) -> int64_t { return deg[v]; },
        [&](int64_t v, int64_t pre, int64_t) { C.off[v] = (int32_t)pre; });
    // first position of each column among the column-sorted kept edges, and
    // of each row among the (row-sorted) kept edges
    team_scan<Team, int64_t>(
        t, sc, sm, (int64_t)nrows, [&](int64_t v) -> int64_t { return infill[v]; },
        [&](int64_t v, int64_t pre, int64_t) { colstart[v] = (int32_t)pre; });
    team_scan<Team, int64_t>(
        t, sc, sm, (int64_t)nrows, [&](int64_t v) -> int64_t { return deg[v] - infill[v]; },
        [&](int64_t v, int64_t pre, int64_t) { rowstart[v] = (int32_t)pre; });
    if (t.rank() == 0) C.off[nrows] = (int32_t)(2 * m);
    t.sync();
    // 3. kept edges in column order, rows increasing within a column (a
    //    bucket sort by column of the kept positions, which are in row order;
    //    columns of more than BUCKET_MAX entries: a stable radix sort) ->
    //    the reverse entries
    int32_t *bst = sc.arena.take<int32_t>((int64_t)nrows + 2);
    if (sc.arena.ok() && m < (int64_t(1) << 31) &&
        team_bucket_sort(
            t, sc, sm, m, nrows, [&](int64_t p) { return A.col[kidx[p]]; }, [&](int64_t p) { return (uint64_t)p; },
            k2, v2, bst)) {
        for (int64_t q = t.rank(); q < m; q += t.size()) {
            const int64_t p = (int64_t)k2[q];
            const int64_t e = kidx[p];
            const int32_t c = A.col[e];
            const int64_t dst = (int64_t)C.off[c] + (q - bst[c]);
            C.adj[dst] = A.row[e];
            C.w[dst] = A.cost[e];
            if (with_eid) C.eid[dst] = (int32_t)p;
        }
    } else {
        team_sort_pairs(t, sc, sm, k1, v1, k2, v2, m, bits_for((uint64_t)(nrows > 0 ? nrows : 1)));
        for (int64_t q = t.rank(); q < m; q += t.size()) {
            int32_t c = (int32_t)k1[q];
            int64_t p = v1[q];
            int64_t e = kidx[p];
            int64_t dst = (int64_t)C.off[c] + (q - colstart[c]);
            C.adj[dst] = A.row[e];
            C.w[dst] = A.cost[e];
            if (with_eid) C.eid[dst] = (int32_t)p;
        }
    }
    // forward entries: the kept edges of row r are contiguous in kidx order
    for (int64_t p = t.rank(); p < m; p += t.size()) {
        int64_t e = kidx[p];
        int32_t r = A.row[e];
        int64_t dst = (int64_t)C.off[r] + infill[r] + (p - rowstart[r]);
        C.adj[dst] = A.col[e];
        C.w[dst] = A.cost[e];
        if (with_eid) C.eid[dst] = (int32_t)p;
    }
    t.sync();
    sc.arena.release(mk);
    return C;
}

// lower bound of the directed graph: sum of min(0, c) (get_lb,
// include/rama_utils.h:179-190), CSUM
template <class Team>
__device__ double graph_lb(const Team &t, Scratch &sc, const Graph &A)
{
    return team_csum(t, sc, A.n, [&](int64_t e) -> float {
        const float c = A.cost[e];
        return c < 0.0f ? c : 0.0f;
    });
}

// compress_label_sequence (include/rama_utils.h:160-177)
template <class Team>
__device__ void compress_labels(const Team &t, Scratch &sc, char *sm, const int32_t *data, int64_t n,
                                int32_t max_label, int32_t *out)
{
    uint64_t m = sc.arena.mark();
    int32_t *mask = sc.arena.take<int32_t>((int64_t)max_label + 2);
    if (!sc.arena.ok()) return;
    for (int64_t l = t.rank(); l <= max_label; l += t.size()) mask[l] = 0;
    t.sync();
    for (int64_t k = t.rank(); k < n; k += t.size()) mask[data[k]] = 1;
    t.sync();
    team_scan<Team, int64_t>(
        t, sc, sm, (int64_t)max_label + 1, [&](int64_t l) -> int64_t { return mask[l]; },
        [&](int64_t l, int64_t pre, int64_t) { mask[l] = (int32_t)pre; });
    for (int64_t k = t.rank(); k < n; k += t.size()) out[k] = mask[data[k]];
    t.sync();
    sc.arena.release(m);
}

}  // namespace rama
