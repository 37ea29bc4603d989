// woc.cuh -- conflict-free contraction set from a maximum spanning forest
// (src/edge_contractions_woc.cu:10-423, src/edge_contractions_woc_thrust.cu:
// 95-599) with a Boruvka forest (external/cudaMST/gpuMST/gpuMST.cu:106-388).
//
// The reference removes conflicted cycles by growing BFS frontiers from both
// ends of every repulsive edge along the forest, one layer per step, and
// cutting the weakest forest edge on a path when the two frontiers meet.  In a
// forest the frontiers of a repulsive edge meet exactly at the step where the
// two depths add up to the length of its unique forest path.  This file
// therefore roots the forest once per epoch (between two forest changes),
// computes every repulsive edge's path length, and replays the reference's
// step schedule (row step, column step, threshold every 5 iterations)
// without materialising frontiers: same cuts, memory O(N + R).
#pragma once
#include "graph.cuh"

namespace rama {

// ---------------------------------------------------------------------------
// Boruvka maximum spanning forest over m edges (i,j,w), w > 0.  Each super
// vertex picks the lexicographic minimum of (-w, target super vertex, id);
// mutual picks keep the smaller vertex as root; roots are renumbered by rank.
// chosen[e] = 1 for forest edges.
// ---------------------------------------------------------------------------
template <class Team, class EI, class EJ, class EW>
__device__ bool team_msf(const Team &t, Scratch &sc, char *sm, int64_t m, int32_t nv0, EI ei, EJ ej, EW ew,
                         uint8_t *chosen)
{
    uint64_t mark = sc.arena.mark();
    const int64_t n2 = 2 * m;
    int32_t *u = sc.arena.take<int32_t>(n2 + 1), *v = sc.arena.take<int32_t>(n2 + 1);
    int32_t *id = sc.arena.take<int32_t>(n2 + 1);
    uint32_t *wk = sc.arena.take<uint32_t>(n2 + 1);
    int32_t *u2 = sc.arena.take<int32_t>(n2 + 1), *v2 = sc.arena.take<int32_t>(n2 + 1);
    int32_t *id2 = sc.arena.take<int32_t>(n2 + 1);
    uint32_t *wk2 = sc.arena.take<uint32_t>(n2 + 1);
    unsigned long long *best = sc.arena.take<unsigned long long>((int64_t)nv0 + 1);
    int32_t *bid = sc.arena.take<int32_t>((int64_t)nv0 + 1);
    int32_t *succ = sc.arena.take<int32_t>((int64_t)nv0 + 1);
    int32_t *succ2 = sc.arena.take<int32_t>((int64_t)nv0 + 1);
    int32_t *newid = sc.arena.take<int32_t>((int64_t)nv0 + 1);
    int32_t *flags = sc.arena.take<int32_t>(64 * 64);
    if (!sc.arena.ok()) return false;
    for (int64_t e = t.rank(); e < m; e += t.size()) {
        int32_t a = ei(e), b = ej(e);
        uint32_t k = float_ordered(-ew(e));
        u[e] = a;
        v[e] = b;
        u[e + m] = b;
        v[e + m] = a;
        wk[e] = wk[e + m] = k;
        id[e] = id[e + m] = (int32_t)e;
        chosen[e] = 0;
    }
    for (int k = t.rank(); k < 64 * 64; k += t.size()) flags[k] = 0;
    t.sync();
    int64_t ne = n2;
    int32_t nv = nv0;
    bool ok = true;
    for (int level = 0; level < 64 && ne > 0; ++level) {
        for (int64_t x = t.rank(); x < nv; x += t.size()) {
            best[x] = ~0ull;
            bid[x] = 0x7fffffff;
        }
        t.sync();
        for (int64_t e = t.rank(); e < ne; e += t.size())
            atomicMin(&best[u[e]], ((unsigned long long)wk[e] << 32) | (uint32_t)v[e]);
        t.sync();
        for (int64_t e = t.rank(); e < ne; e += t.size())
            if ((((unsigned long long)wk[e] << 32) | (uint32_t)v[e]) == best[u[e]]) atomicMin(&bid[u[e]], id[e]);
        t.sync();
        for (int64_t x = t.rank(); x < nv; x += t.size())
            succ[x] = best[x] == ~0ull ? (int32_t)x : (int32_t)(best[x] & 0xffffffffu);
        t.sync();
        // remove_circles (:106-121) and save forest edges
        for (int64_t x = t.rank(); x < nv; x += t.size()) {
            int32_t s = succ[x], ss = succ[s];
            int32_t r = (s > (int32_t)x && ss == (int32_t)x) ? (int32_t)x : s;
            succ2[x] = r;
            if (r != (int32_t)x) chosen[bid[x]] = 1;
        }
        t.sync();
        // merge_vertices (:123-147): pointer jumping to the roots
        int jumps = 0;
        for (; jumps < 62; ++jumps) {
            for (int64_t x = t.rank(); x < nv; x += t.size()) {
                int32_t s = succ2[x];
                int32_t ss = ((volatile int32_t *)succ2)[s];
                if (ss != s) {
                    succ2[x] = ss;
                    flags[level * 64 + jumps] = 1;
                }
            }
            t.sync();
            if (!uread(&flags[level * 64 + jumps])) break;
        }
        if (jumps == 62) ok = false;
        // renumber roots by rank (sort + mark_segments + scan, :285-298)
        const int64_t nroots = team_compact(
            t, sc, sm, nv, [&](int64_t x) { return succ2[x] == (int32_t)x; },
            [&](int64_t x, int64_t p) { newid[x] = (int32_t)p; });
        for (int64_t x = t.rank(); x < nv; x += t.size()) succ[x] = newid[succ2[x]];
        t.sync();
        // keep edges between different super vertices, relabelled (:300-334)
        const int64_t ne2 = team_compact(
            t, sc, sm, ne, [&](int64_t e) { return succ[u[e]] != succ[v[e]]; },
            [&](int64_t e, int64_t p) {
                u2[p] = succ[u[e]];
                v2[p] = succ[v[e]];
                wk2[p] = wk[e];
                id2[p] = id[e];
            });
        int32_t *tp;
        tp = u; u = u2; u2 = tp;
        tp = v; v = v2; v2 = tp;
        tp = id; id = id2; id2 = tp;
        uint32_t *tw = wk; wk = wk2; wk2 = tw;
        ne = ne2;
        nv = (int32_t)nroots;
    }
    if (ne > 0) ok = false;
    sc.arena.release(mark);
    return ok;
}

// ---------------------------------------------------------------------------
struct Forest {
    int32_t nn;
    int64_t m2;
    int32_t *r, *c;
    float *w;
    int32_t *r2, *c2;  // ping-pong
    float *w2;
    int32_t *off;
    int64_t R;
    int32_t *rr, *rc, *rr2, *rc2;
    int32_t *lab;
    uint8_t *inv;
    int32_t *par, *dep, *plen;
    float *pw;
    int32_t *front, *front2, *cnt;
    int version;
};

template <class Team>
__device__ void forest_offsets(const Team &t, Forest &F)
{
    team_offsets(t, F.m2, F.nn, [&](int64_t k) { return F.r[k]; }, F.off);
}

__device__ __forceinline__ int32_t forest_find(const Forest &F, int32_t a, int32_t b)
{
    int32_t lo = F.off[a], hi = F.off[a + 1];
    while (lo < hi) {
        int32_t m = (lo + hi) >> 1;
        if (F.c[m] < b)
            lo = m + 1;
        else
            hi = m;
    }
    return lo;
}

// drop the undirected edges whose entry is flagged in F.inv (both
// directions); returns whether anything was removed.  F.inv is cleared.
template <class Team>
__device__ bool forest_remove_flagged(const Team &t, Scratch &sc, char *sm, Forest &F)
{
    for (int64_t k = t.rank(); k < F.m2; k += t.size()) {
        if (F.inv[k] == 1) {
            int32_t q = forest_find(F, F.c[k], F.r[k]);
            F.inv[q] = 2;  // mark the reverse entry (2: reverse-only mark)
        }
    }
    t.sync();
    const int64_t kept = team_compact(
        t, sc, sm, F.m2, [&](int64_t k) { return F.inv[k] == 0; },
        [&](int64_t k, int64_t p) {
            F.r2[p] = F.r[k];
            F.c2[p] = F.c[k];
            F.w2[p] = F.w[k];
        });
    const bool any = kept != F.m2;
    int32_t *tp;
    tp = F.r; F.r = F.r2; F.r2 = tp;
    tp = F.c; F.c = F.c2; F.c2 = tp;
    float *tw = F.w; F.w = F.w2; F.w2 = tw;
    F.m2 = kept;
    for (int64_t k = t.rank(); k < F.m2; k += t.size()) F.inv[k] = 0;
    forest_offsets(t, F);
    if (any) F.version++;
    return any;
}

// filter_by_cc (src/edge_contractions_woc.cu:257-276)
template <class Team>
__device__ int64_t forest_filter_by_cc(const Team &t, Scratch &sc, char *sm, Forest &F)
{
    team_cc(t, sc, F.nn, F.m2, [&](int64_t k) { return F.r[k]; }, [&](int64_t k) { return F.c[k]; }, F.lab);
    const int64_t R = team_compact(
        t, sc, sm, F.R, [&](int64_t k) { return F.lab[F.rr[k]] == F.lab[F.rc[k]]; },
        [&](int64_t k, int64_t p) {
            F.rr2[p] = F.rr[k];
            F.rc2[p] = F.rc[k];
        });
    int32_t *tp;
    tp = F.rr; F.rr = F.rr2; F.rr2 = tp;
    tp = F.rc; F.rc = F.rc2; F.rc2 = tp;
    F.R = R;
    return R;
}

__device__ __forceinline__ int32_t first_common_pos(const Forest &F, int32_t a, int32_t b, int32_t &pa, int32_t &pb)
{
    int32_t x = F.off[a], y = F.off[b], xe = F.off[a + 1], ye = F.off[b + 1];
    while (x < xe && y < ye) {
        int32_t na = F.c[x], nb = F.c[y];
        if (na == nb) {
            pa = x;
            pb = y;
            return na;
        }
        x += (na < nb);
        y += (nb < na);
    }
    return -1;
}

// check_triangles_cuda (src/edge_contractions_woc.cu:10-37)
template <class Team>
__device__ bool forest_check_triangles(const Team &t, Scratch &sc, char *sm, Forest &F)
{
    if (F.R == 0) return false;
    for (int64_t k = t.rank(); k < F.R; k += t.size()) {
        int32_t p1, p2;
        if (first_common_pos(F, F.rr[k], F.rc[k], p1, p2) < 0) continue;
        F.inv[F.w[p1] < F.w[p2] ? p1 : p2] = 1;
    }
    t.sync();
    return forest_remove_flagged(t, sc, sm, F);
}

// check_quadrangles_cuda (src/edge_contractions_woc.cu:39-79)
template <class Team>
__device__ bool forest_check_quadrangles(const Team &t, Scratch &sc, char *sm, Forest &F)
{
    if (F.R == 0) return false;
    for (int64_t k = t.rank(); k < F.R; k += t.size()) {
        int32_t v1 = F.rr[k], v2 = F.rc[k];
        for (int32_t e1 = F.off[v1]; e1 < F.off[v1 + 1]; ++e1) {
            int32_t n1 = F.c[e1];
            int32_t p1, p2;
            if (first_common_pos(F, n1, v2, p1, p2) < 0) continue;
            float a = F.w[e1], b = F.w[p1], c = F.w[p2];
            F.inv[(a < b && a < c) ? e1 : (b < c ? p1 : p2)] = 1;
        }
    }
    t.sync();
    return forest_remove_flagged(t, sc, sm, F);
}

// check_pentagons_cuda (src/edge_contractions_woc.cu:81-139): for every
// repulsive edge (v1, v2) and every pair of forest neighbours n1 of v1, n2 of
// v2 with n1 != n2, the first common neighbour mid of n1 and n2 closes the
// 5-cycle v1-n1-mid-n2-v2; the weakest of its four forest edges is cut (the
// reference's comparison order).  The reference ships this step disabled;
// here it runs when the option asks for it.
template <class Team>
__device__ bool forest_check_pentagons(const Team &t, Scratch &sc, char *sm, Forest &F)
{
    if (F.R == 0) return false;
    for (int64_t k = t.rank(); k < F.R; k += t.size()) {
        const int32_t v1 = F.rr[k], v2 = F.rc[k];
        for (int32_t e2 = F.off[v2]; e2 < F.off[v2 + 1]; ++e2) {
            const int32_t n2 = F.c[e2];
            for (int32_t e1 = F.off[v1]; e1 < F.off[v1 + 1]; ++e1) {
                const int32_t n1 = F.c[e1];
                if (n1 == n2) continue;
                int32_t p1, p2;
                if (first_common_pos(F, n1, n2, p1, p2) < 0) continue;
                const float a = F.w[e1], b = F.w[e2], c1 = F.w[p1], c2 = F.w[p2];
                int32_t cut;
                if (a < b)
                    cut = (a < c1 && a < c2) ? e1 : (c1 < c2 ? p1 : p2);
                else
                    cut = (b < c1 && b < c2) ? e2 : (c1 < c2 ? p1 : p2);
                F.inv[cut] = 1;
            }
        }
    }
    t.sync();
    return forest_remove_flagged(t, sc, sm, F);
}

// filter_by_thresholding (src/edge_contractions_woc_thrust.cu:522-542)
template <class Team>
__device__ bool forest_threshold(const Team &t, Scratch &sc, char *sm, Forest &F)
{
    const double S = team_csum(t, sc, F.m2, [&](int64_t k) -> float {
        const float x = F.w[k];
        return x >= 0.0f ? x : 0.0f;
    });
    const int64_t cnt = team_sum<Team, int64_t>(t, sc, sm, F.m2, [&](int64_t k) -> int64_t { return F.w[k] >= 0.0f; });
    const float thr = (0.9f * (float)S) / (float)cnt;
    for (int64_t k = t.rank(); k < F.m2; k += t.size()) F.inv[k] = F.w[k] < thr ? 3 : 0;
    t.sync();
    return forest_remove_flagged(t, sc, sm, F);
}

// roots = component minima; level-synchronous BFS gives parent, depth and
// the weight of the edge to the parent.  In a forest every vertex is found
// by exactly one frontier vertex, so the BFS needs no atomics on par[].
template <class Team>
__device__ bool forest_root(const Team &t, Scratch &sc, char *sm, Forest &F)
{
    for (int64_t v = t.rank(); v < F.nn; v += t.size()) {
        F.par[v] = -2;
        F.dep[v] = 0;
        F.pw[v] = 0.0f;
    }
    t.sync();
    int64_t nf = team_compact(
        t, sc, sm, F.nn, [&](int64_t v) { return F.lab[v] == (int32_t)v && F.off[v + 1] > F.off[v]; },
        [&](int64_t v, int64_t p) {
            F.front[p] = (int32_t)v;
            F.par[v] = -1;
        });
    for (int lvl = 0; nf > 0; ++lvl) {
        if (lvl > F.nn) return false;
        int32_t *cntp = F.cnt + (lvl & 1) * 2;
        if (t.rank() == 0) F.cnt[((lvl + 1) & 1) * 2] = 0;
        for (int64_t q = t.rank(); q < nf; q += t.size()) {
            int32_t x = F.front[q];
            for (int32_t k = F.off[x]; k < F.off[x + 1]; ++k) {
                int32_t y = F.c[k];
                if (F.par[y] != -2) continue;
                F.par[y] = x;
                F.dep[y] = F.dep[x] + 1;
                F.pw[y] = F.w[k];
                int32_t p = atomicAdd(cntp, 1);
                F.front2[p] = y;
            }
        }
        t.sync();
        nf = uread(cntp);
        int32_t *tf = F.front;
        F.front = F.front2;
        F.front2 = tf;
        t.sync();
        if (t.rank() == 0) cntp[0] = 0;
    }
    return true;
}

// Walks v1 and v2 up to their meeting point in the rooted forest; la / lb =
// edges walked on each side.  Returns false if the walk leaves the forest
// (an unreached vertex or different trees), never reading outside par[].
__device__ __forceinline__ bool forest_meet(const Forest &F, int32_t a, int32_t b, int32_t &la, int32_t &lb)
{
    la = lb = 0;
    for (int32_t s = 0; s <= F.nn && a >= 0 && b >= 0 && F.dep[a] > F.dep[b]; ++s) {
        a = F.par[a];
        ++la;
    }
    for (int32_t s = 0; s <= F.nn && a >= 0 && b >= 0 && F.dep[b] > F.dep[a]; ++s) {
        b = F.par[b];
        ++lb;
    }
    for (int32_t s = 0; s <= F.nn && a >= 0 && b >= 0 && a != b; ++s) {
        a = F.par[a];
        b = F.par[b];
        ++la;
        ++lb;
    }
    return a >= 0 && b >= 0 && a == b;
}

template <class Team>
__device__ int32_t forest_path_lengths(const Team &t, Scratch &sc, char *sm, Forest &F)
{
    for (int64_t k = t.rank(); k < F.R; k += t.size()) {
        int32_t la, lb;
        F.plen[k] = forest_meet(F, F.rr[k], F.rc[k], la, lb) ? la + lb : 0x3fffffff;
    }
    t.sync();
    return team_min<Team, int32_t>(t, sc, sm, F.R, 0x7fffffff, [&](int64_t k) { return F.plen[k]; });
}

// Cut the bottleneck of every repulsive edge whose path has dr+dc edges: the
// first minimum met from v1 over the first dr path edges against the first
// minimum met from v2 over the last dc (reduce_intersecting_paths,
// src/edge_contractions_woc_thrust.cu:201-216: the v1 side wins only when
// strictly smaller).
template <class Team>
__device__ bool forest_resolve(const Team &t, Scratch &sc, char *sm, Forest &F, int32_t dr, int32_t dc)
{
    const int32_t s = dr + dc;
    for (int64_t k = t.rank(); k < F.R; k += t.size()) {
        if (F.plen[k] != s) continue;
        const int32_t v1 = F.rr[k], v2 = F.rc[k];
        int32_t la = 0, lb = 0;
        if (!forest_meet(F, v1, v2, la, lb)) continue;
        const int32_t L = la + lb;
        // row half: path[q], q in [0,dr); path[q] is v1's up edge q (q<la) or
        // v2's up edge L-1-q (q>=la)
        float brow = 3.402823466e38f, bcol = 3.402823466e38f;
        int32_t crow = -1, ccol = -1;  // child vertex of the chosen edge
        {
            int32_t x = v1;
            for (int32_t q = 0; q < la && q < dr; ++q) {
                if (F.pw[x] < brow) {
                    brow = F.pw[x];
                    crow = x;
                }
                x = F.par[x];
            }
            if (dr > la) {  // j = L-1-q in [L-dr, lb), scanned in descending j
                float bb = 3.402823466e38f;
                int32_t cb = -1;
                int32_t y = v2;
                for (int32_t j = 0; j < lb; ++j) {
                    if (j >= L - dr && F.pw[y] <= bb) {
                        bb = F.pw[y];
                        cb = y;
                    }
                    y = F.par[y];
                }
                if (bb < brow) {
                    brow = bb;
                    crow = cb;
                }
            }
        }
        {
            int32_t y = v2;
            for (int32_t j = 0; j < lb && j < dc; ++j) {
                if (F.pw[y] < bcol) {
                    bcol = F.pw[y];
                    ccol = y;
                }
                y = F.par[y];
            }
            if (dc > lb) {  // q = L-1-j' in [L-dc, la), scanned in descending q
                float bb = 3.402823466e38f;
                int32_t cb = -1;
                int32_t x = v1;
                for (int32_t q = 0; q < la; ++q) {
                    if (q >= L - dc && F.pw[x] <= bb) {
                        bb = F.pw[x];
                        cb = x;
                    }
                    x = F.par[x];
                }
                if (bb < bcol) {
                    bcol = bb;
                    ccol = cb;
                }
            }
        }
        int32_t child = (brow < bcol) ? crow : ccol;
        if (child < 0) child = crow >= 0 ? crow : ccol;
        if (child < 0) continue;
        F.inv[forest_find(F, child, F.par[child])] = 1;
    }
    t.sync();
    return forest_remove_flagged(t, sc, sm, F);
}

// edge_contractions_woc ctor + find_contraction_mapping.  map_out gets
// max_dim(A) entries; returns the number of directed forest entries left
// (0 = nothing to contract).
template <class Team>
__device__ int32_t woc_contraction_map(const Team &t, Scratch &sc, char *sm, const Graph &A, int32_t *map_out,
                                       int32_t *map_size, int *err, bool pentagons = false)
{
    Forest F;
    F.nn = A.max_dim();
    F.version = 0;
    *map_size = 0;
    uint64_t mark = sc.arena.mark();
    int64_t *pidx = sc.arena.take<int64_t>(A.n + 1);
    F.rr = sc.arena.take<int32_t>(A.n + 1);
    F.rc = sc.arena.take<int32_t>(A.n + 1);
    F.rr2 = sc.arena.take<int32_t>(A.n + 1);
    F.rc2 = sc.arena.take<int32_t>(A.n + 1);
    if (!sc.arena.ok()) return 0;
    // 1. partition at cost > 0 (:345-375)
    const int64_t P = team_compact(
        t, sc, sm, A.n, [&](int64_t e) { return A.cost[e] > 0.0f; }, [&](int64_t e, int64_t p) { pidx[p] = e; });
    F.R = team_compact(
        t, sc, sm, A.n, [&](int64_t e) { return !(A.cost[e] > 0.0f); },
        [&](int64_t e, int64_t p) {
            F.rr[p] = A.row[e];
            F.rc[p] = A.col[e];
        });
    if (P == 0) {
        sc.arena.release(mark);
        return 0;
    }
    // 2. maximum spanning forest of the attractive edges
    const int32_t nv0 = 1 + team_max<Team, int32_t>(t, sc, sm, P, 0, [&](int64_t p) { return A.col[pidx[p]]; });
    uint8_t *chosen = sc.arena.take<uint8_t>(P + 1);
    if (!sc.arena.ok()) return 0;
    if (!team_msf(t, sc, sm, P, nv0, [&](int64_t p) { return A.row[pidx[p]]; },
                  [&](int64_t p) { return A.col[pidx[p]]; }, [&](int64_t p) { return A.cost[pidx[p]]; }, chosen)) {
        *err |= ERR_ITER_LIMIT;
    }
    prof_mark(t, sc, PH_WOC_MSF);
    // 3. forest as a symmetric (row,col)-sorted list + CSR
    uint8_t *ekeep = sc.arena.take<uint8_t>(A.n + 1);
    if (!sc.arena.ok()) return 0;
    for (int64_t e = t.rank(); e < A.n; e += t.size()) ekeep[e] = 0;
    t.sync();
    for (int64_t p = t.rank(); p < P; p += t.size())
        if (chosen[p]) ekeep[pidx[p]] = 1;
    t.sync();
    Csr C = build_symmetric_csr(t, sc, sm, A, F.nn, [&](int64_t e) { return ekeep[e] != 0; }, false);
    F.m2 = C.m2;
    F.off = C.off;
    F.c = C.adj;
    F.w = C.w;
    F.r = sc.arena.take<int32_t>(F.m2 + 1);
    F.r2 = sc.arena.take<int32_t>(F.m2 + 1);
    F.c2 = sc.arena.take<int32_t>(F.m2 + 1);
    F.w2 = sc.arena.take<float>(F.m2 + 1);
    F.inv = sc.arena.take<uint8_t>(F.m2 + 1);
    F.lab = sc.arena.take<int32_t>((int64_t)F.nn + 1);
    F.par = sc.arena.take<int32_t>((int64_t)F.nn + 1);
    F.dep = sc.arena.take<int32_t>((int64_t)F.nn + 1);
    F.pw = sc.arena.take<float>((int64_t)F.nn + 1);
    F.front = sc.arena.take<int32_t>((int64_t)F.nn + 1);
    F.front2 = sc.arena.take<int32_t>((int64_t)F.nn + 1);
    F.cnt = sc.arena.take<int32_t>(8);
    F.plen = sc.arena.take<int32_t>(F.R + 1);
    if (!sc.arena.ok()) return 0;
    for (int64_t v = t.rank(); v < F.nn; v += t.size())
        for (int32_t k = F.off[v]; k < F.off[v + 1]; ++k) F.r[k] = (int32_t)v;
    for (int64_t k = t.rank(); k < F.m2; k += t.size()) F.inv[k] = 0;
    if (t.rank() < 8) F.cnt[t.rank()] = 0;
    t.sync();
    prof_mark(t, sc, PH_WOC_CSR);
    if (F.m2 == 0) {
        sc.arena.release(mark);
        return 0;
    }
    // 4. find_contraction_mapping (src/edge_contractions_woc.cu:387-423)
    forest_filter_by_cc(t, sc, sm, F);
    if (forest_check_triangles(t, sc, sm, F)) forest_filter_by_cc(t, sc, sm, F);
    forest_check_quadrangles(t, sc, sm, F);
    if (pentagons) forest_check_pentagons(t, sc, sm, F);  // the commented-out call at :414
    if (F.m2 == 0) {
        sc.arena.release(mark);
        return 0;
    }
    // 5. edge_contractions_woc_thrust::find_contraction_mapping (:544-599)
    int64_t R = forest_filter_by_cc(t, sc, sm, F);
    prof_mark(t, sc, PH_WOC_CHECKS);
    int32_t dr = 0, dc = 0, itr = 0;
    int32_t lmin = -1;           // shortest path length of this epoch (-1: stale)
    int thr_noop_version = -1;   // forest version at which thresholding was a no-op
    for (int guard = 0; R > 0 && F.m2 > 0; ++guard) {
        if (guard > (1 << 26)) {
            *err |= ERR_ITER_LIMIT;
            break;
        }
        if (itr % 5 == 0 && thr_noop_version != F.version) {
            if (forest_threshold(t, sc, sm, F)) {
                R = forest_filter_by_cc(t, sc, sm, F);
                dr = dc = 0;
                lmin = -1;
            } else {
                thr_noop_version = F.version;
            }
            prof_mark(t, sc, PH_WOC_CHECKS);
        }
        if (R == 0 || F.m2 == 0) break;
        for (int side = 0; side < 2; ++side) {
            if (side == 0)
                ++dr;
            else
                ++dc;
            if (lmin < 0) {
                if (!forest_root(t, sc, sm, F)) *err |= ERR_ITER_LIMIT;
                prof_mark(t, sc, PH_WOC_ROOT);
                lmin = forest_path_lengths(t, sc, sm, F);
                prof_mark(t, sc, PH_WOC_PATHS);
            }
            if (dr + dc == lmin) {
                const bool cut = forest_resolve(t, sc, sm, F, dr, dc);
                prof_mark(t, sc, PH_WOC_PATHS);
                if (cut) {
                    R = forest_filter_by_cc(t, sc, sm, F);
                    dr = dc = 0;
                    lmin = -1;
                    prof_mark(t, sc, PH_WOC_CHECKS);
                }
            }
            if (side == 0 && (R == 0 || F.m2 == 0)) break;
        }
        if (R == 0 || F.m2 == 0) break;
        ++itr;
    }
    compress_labels(t, sc, sm, F.lab, F.nn, F.nn - 1, map_out);
    *map_size = F.nn;
    const int32_t nr = (int32_t)F.m2;
    sc.arena.release(mark);
    return nr;
}

}  // namespace rama
