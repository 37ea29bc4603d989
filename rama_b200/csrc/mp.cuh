// mp.cuh -- triangle message passing (src/multicut_message_passing.cu:15-360)
// and the dual solver loop (src/dual_solver.cu:7-63).
//
// Layout (all SoA in the arena): triangles t1<t2<t3 sorted and unique; their
// edge indices e12/e13/e23 into the merged edge list (the graph's edges plus
// the triangle chords it lacks, cost 0).  The messages a triangle sends to
// its edges go to `slot`, which holds each edge's incoming messages
// contiguously in incidence order (triangle order); pos[3t + corner] is the
// slot of triangle t's message to that corner's edge.  Each edge then takes
// the RSUM of its run of slots, which replaces the reference's float
// atomicAdd by a deterministic sum.
#pragma once
#include "cycles.cuh"

namespace rama {

struct Mp {
    int64_t T, E;
    int32_t *t1, *t2, *t3;
    int32_t *e12, *e13, *e23;
    float *c12, *c13, *c23;
    float *slot;  // 3T: incoming messages, edge by edge in incidence order
    int32_t *pos;  // 3T: slot of triangle t's message to corner c at 3t + c
    int32_t *row, *col;
    float *cost;
    float *share;      // E: cost / number of incident triangles (covered edges)
    int32_t *inc_off;  // E + 1: first slot of each edge
    int32_t *longe;    // edges with more than RSUM_THREAD_MAX incident triangles
    int64_t nlong;
    int32_t rows, cols;
};

// position of (a,b) in a (row,col)-sorted list with row offsets `off`
__device__ __forceinline__ int64_t find_edge(const int32_t *off, const int32_t *col, int32_t a, int32_t b)
{
    int32_t lo = off[a], hi = off[a + 1];
    while (lo < hi) {
        int32_t m = (lo + hi) >> 1;
        if (col[m] < b)
            lo = m + 1;
        else
            hi = m;
    }
    return (lo < off[a + 1] && col[lo] == b) ? lo : -1;
}

// find_edge of three (a, b) pairs at once: the three binary searches step in
// lockstep, so each step's loads are in flight together
__device__ __forceinline__ void find_edges3(const int32_t *off, const int32_t *col, const int32_t (&a)[3],
                                           const int32_t (&b)[3], int32_t (&out)[3])
{
    int32_t lo[3], hi[3], end[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        lo[k] = off[a[k]];
        hi[k] = end[k] = off[a[k] + 1];
    }
    for (int step = 0; step < 32; ++step) {
        int32_t m[3], c[3];
        bool any = false;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            m[k] = (lo[k] + hi[k]) >> 1;
            c[k] = lo[k] < hi[k] ? col[m[k]] : 0;
        }
#pragma unroll
        for (int k = 0; k < 3; ++k)
            if (lo[k] < hi[k]) {
                any = true;
                if (c[k] < b[k])
                    lo[k] = m[k] + 1;
                else
                    hi[k] = m[k];
            }
        if (!any) break;
    }
    int32_t c[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) c[k] = lo[k] < end[k] ? col[lo[k]] : 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) out[k] = (lo[k] < end[k] && c[k] == b[k]) ? lo[k] : -1;
}

// number of entries of row a with col < b, plus all rows < a
__device__ __forceinline__ int64_t lower_edge(const int32_t *off, const int32_t *col, int32_t a, int32_t b)
{
    int32_t lo = off[a], hi = off[a + 1];
    while (lo < hi) {
        int32_t m = (lo + hi) >> 1;
        if (col[m] < b)
            lo = m + 1;
        else
            hi = m;
    }
    return lo;
}

// multicut_message_passing ctor (:65-176)
template <class Team>
__device__ bool mp_build(const Team &t, Scratch &sc, char *sm, const Graph &A, TriBuf &tb, Mp &mp)
{
    int32_t nmax = A.max_dim();
    // normalize_triangles (:79)
    const int64_t T = tri_normalize(t, sc, sm, tb.t1, tb.t2, tb.t3, tb.num, nmax);
    prof_mark(t, sc, PH_MP_NORM);
    if (!sc.arena.ok()) return false;
    mp.T = T;
    mp.t1 = tb.t1;
    mp.t2 = tb.t2;
    mp.t3 = tb.t3;
    // row offsets of A over [0, nmax]
    int32_t *aoff = sc.arena.take<int32_t>((int64_t)nmax + 2);
    uint64_t *nk1 = sc.arena.take<uint64_t>(3 * T + 1), *nk2 = sc.arena.take<uint64_t>(3 * T + 1);
    int32_t *nv1 = sc.arena.take<int32_t>(3 * T + 1), *nv2 = sc.arena.take<int32_t>(3 * T + 1);
    if (!sc.arena.ok()) return false;
    team_offsets(t, A.n, nmax, [&](int64_t e) { return A.row[e]; }, aoff);
    const int nb = bits_for((uint64_t)(nmax > 0 ? nmax : 1));
    // chords not in A: the three sides of each triangle are looked up
    // together, and the compaction reads the flags (nv2 is free until the
    // chord sort)
    uint8_t *absent = reinterpret_cast<uint8_t *>(nv2);
    for (int64_t k = t.rank(); k < T; k += t.size()) {
        const int32_t a[3] = {mp.t1[k], mp.t1[k], mp.t2[k]};
        const int32_t b[3] = {mp.t2[k], mp.t3[k], mp.t3[k]};
        int32_t f[3];
        find_edges3(aoff, A.col, a, b, f);
#pragma unroll
        for (int s = 0; s < 3; ++s) absent[3 * k + s] = f[s] < 0;
    }
    t.sync();
    const int64_t nn = team_compact(
        t, sc, sm, 3 * T, [&](int64_t q) { return absent[q] != 0; },
        [&](int64_t q, int64_t p) {
            int64_t k = q / 3;
            int s = (int)(q % 3);
            int32_t a = s == 2 ? mp.t2[k] : mp.t1[k];
            int32_t b = s == 0 ? mp.t2[k] : mp.t3[k];
            nk1[p] = pack_key(a, b, nb);
            nv1[p] = 0;
        });
    {
        // sort the chords (a, b): bucket by a, order by b (equal chords are
        // merged below, so their order does not matter); rows of more than
        // BUCKET_MAX chords: LSD radix sort
        const uint64_t cmask = (nb == 0) ? 0 : ((uint64_t(1) << nb) - 1);
        uint64_t bm = sc.arena.mark();
        int32_t *bst = sc.arena.take<int32_t>((int64_t)nmax + 2);
        bool done = false;
        if (sc.arena.ok() && nn < (int64_t(1) << 31)) {
            // the payload of each chord is its row, so every sorted position
            // rebuilds its key from its own entries
            auto row = [&](int64_t q) { return (int32_t)(nk1[q] >> nb); };
            done = team_bucket_sort_ex(
                t, sc, sm, nn, nmax + 1, row, row, [&](int64_t q) { return nk1[q] & cmask; }, row, nk2, nv2, bst);
            if (done) {
                team_for_batched(
                    t, nn, [&](int64_t p) { return ((uint64_t)(uint32_t)nv2[p] << nb) | nk2[p]; },
                    [&](int64_t p, uint64_t key) { nk1[p] = key; });
                t.sync();
            }
        }
        sc.arena.release(bm);
        if (!done) team_sort_pairs(t, sc, sm, nk1, nv1, nk2, nv2, nn, 2 * nb);
    }
    uint64_t *nu = nk2;  // unique chords
    const int64_t nu_n = team_compact(
        t, sc, sm, nn, [&](int64_t k) { return k == 0 || nk1[k] != nk1[k - 1]; },
        [&](int64_t k, int64_t p) { nu[p] = nk1[k]; });
    // merged edge list (set_union_by_key, :130-158)
    const int64_t E = A.n + nu_n;
    mp.E = E;
    mp.row = sc.arena.take<int32_t>(E + 1);
    mp.col = sc.arena.take<int32_t>(E + 1);
    mp.cost = sc.arena.take<float>(E + 1);
    if (!sc.arena.ok()) return false;
    const uint64_t mask = (nb == 0) ? 0 : ((uint64_t(1) << nb) - 1);
    // row offsets of the chords: an edge counts the chords before it among
    // those of its own row
    // (counted per row and scanned: chords leave long runs of empty rows)
    int32_t *coff = sc.arena.take<int32_t>((int64_t)nmax + 2);
    if (!sc.arena.ok()) return false;
    for (int64_t v = t.rank(); v <= nmax; v += t.size()) coff[v] = 0;
    t.sync();
    for (int64_t k = t.rank(); k < nu_n; k += t.size()) atomicAdd(&coff[(int32_t)(nu[k] >> nb)], 1);
    t.sync();
    team_scan<Team, int64_t>(
        t, sc, sm, (int64_t)nmax + 1, [&](int64_t v) -> int64_t { return coff[v]; },
        [&](int64_t v, int64_t pre, int64_t) { coff[v] = (int32_t)pre; });
    for (int64_t e = t.rank(); e < A.n; e += t.size()) {
        const int32_t r = A.row[e];
        uint64_t key = pack_key(r, A.col[e], nb);
        int64_t lo = coff[r], hi = coff[r + 1];  // chords < key: all of rows < r, then within row r
        while (lo < hi) {
            int64_t m = (lo + hi) >> 1;
            if (nu[m] < key)
                lo = m + 1;
            else
                hi = m;
        }
        int64_t p = e + lo;
        mp.row[p] = A.row[e];
        mp.col[p] = A.col[e];
        mp.cost[p] = A.cost[e];
    }
    for (int64_t k = t.rank(); k < nu_n; k += t.size()) {
        int32_t a = (int32_t)(nu[k] >> nb), b = (int32_t)(nu[k] & mask);
        int64_t p = k + lower_edge(aoff, A.col, a, b);
        mp.row[p] = a;
        mp.col[p] = b;
        mp.cost[p] = 0.0f;
    }
    t.sync();
    prof_mark(t, sc, PH_MP_CHORDS);
    // merged row offsets, correspondences (compute_triangle_edge_correspondence, :15-62)
    int32_t *moff = aoff;  // reuse
    team_offsets(t, E, nmax, [&](int64_t e) { return mp.row[e]; }, moff);
    mp.e12 = sc.arena.take<int32_t>(T + 1);
    mp.e13 = sc.arena.take<int32_t>(T + 1);
    mp.e23 = sc.arena.take<int32_t>(T + 1);
    mp.c12 = sc.arena.take<float>(T + 1);
    mp.c13 = sc.arena.take<float>(T + 1);
    mp.c23 = sc.arena.take<float>(T + 1);
    mp.slot = sc.arena.take<float>(3 * T + 1);
    mp.pos = sc.arena.take<int32_t>(3 * T + 1);
    mp.inc_off = sc.arena.take<int32_t>(E + 2);
    uint64_t ik = sc.arena.mark();
    uint64_t *q1 = sc.arena.take<uint64_t>(3 * T + 1), *q2 = sc.arena.take<uint64_t>(3 * T + 1);
    int32_t *w1 = sc.arena.take<int32_t>(3 * T + 1), *w2 = sc.arena.take<int32_t>(3 * T + 1);
    if (!sc.arena.ok()) return false;
    for (int64_t k = t.rank(); k < T; k += t.size()) {
        const int32_t a = mp.t1[k], b = mp.t2[k], c = mp.t3[k];
        const int32_t from[3] = {a, a, b}, to[3] = {b, c, c};
        int32_t f[3];
        find_edges3(moff, mp.col, from, to, f);
        const int32_t x = f[0], y = f[1], z = f[2];
        mp.e12[k] = x;
        mp.e13[k] = y;
        mp.e23[k] = z;
        mp.c12[k] = mp.c13[k] = mp.c23[k] = 0.0f;
        q1[3 * k] = (uint64_t)x;
        q1[3 * k + 1] = (uint64_t)y;
        q1[3 * k + 2] = (uint64_t)z;
        w1[3 * k] = (int32_t)(3 * k);
        w1[3 * k + 1] = (int32_t)(3 * k + 1);
        w1[3 * k + 2] = (int32_t)(3 * k + 2);
    }
    t.sync();
    // incidence order: (edge, 3t + corner) sorted by edge, then by 3t + corner;
    // the rank of each (triangle, corner) in that order is its slot
    if (3 * T < (int64_t(1) << 31) &&
        team_bucket_sort(
            t, sc, sm, 3 * T, (int32_t)E, [&](int64_t q) { return (int32_t)q1[q]; },
            [&](int64_t q) { return (uint64_t)q; }, q2, w2, mp.inc_off)) {
        for (int64_t q = t.rank(); q < 3 * T; q += t.size()) mp.pos[w2[q]] = (int32_t)q;
        t.sync();
    } else {
        int32_t *incp = w1;
        uint64_t *qk = q1;
        team_sort_pairs(t, sc, sm, qk, incp, q2, w2, 3 * T, bits_for((uint64_t)(E > 0 ? E : 1)));
        for (int64_t q = t.rank(); q < 3 * T; q += t.size()) mp.pos[incp[q]] = (int32_t)q;
        team_offsets(t, 3 * T, (int32_t)E, [&](int64_t k) { return (int32_t)qk[k]; }, mp.inc_off);
    }
    sc.arena.release(ik);
    prof_mark(t, sc, PH_MP_INCID);
    // each covered edge's share of its cost, and the edges whose incoming
    // messages a whole warp sums
    mp.share = sc.arena.take<float>(E + 1);
    mp.longe = sc.arena.take<int32_t>(E + 1);
    if (!sc.arena.ok()) return false;
    mp.nlong = team_compact(
        t, sc, sm, E, [&](int64_t e) { return mp.inc_off[e + 1] - mp.inc_off[e] > RSUM_THREAD_MAX; },
        [&](int64_t e, int64_t p) { mp.longe[p] = (int32_t)e; });
    for (int64_t e = t.rank(); e < E; e += t.size()) {
        const int32_t n = mp.inc_off[e + 1] - mp.inc_off[e];
        mp.share[e] = n > 0 ? __fdiv_rn(mp.cost[e], (float)n) : 0.0f;
    }
    t.sync();
    mp.rows = A.rows;
    mp.cols = A.cols;
    return true;
}

// triangle_lb_func (:186-199)
__device__ __forceinline__ float tri_lb(float c12, float c13, float c23)
{
    float lb = 0.0f;
    lb = fminf(lb, __fadd_rn(c12, c13));
    lb = fminf(lb, __fadd_rn(c12, c23));
    lb = fminf(lb, __fadd_rn(c13, c23));
    lb = fminf(lb, __fadd_rn(__fadd_rn(c12, c13), c23));
    return lb;
}

// lower_bound (:201-216), CSUM for both parts
template <class Team>
__device__ double mp_lower_bound(const Team &t, Scratch &sc, const Mp &mp)
{
    double le = team_csum(t, sc, mp.E, [&](int64_t e) -> float {
        const float c = mp.cost[e];
        return c < 0.0f ? c : 0.0f;
    });
    double lt = team_csum(t, sc, mp.T, [&](int64_t k) -> float { return tri_lb(mp.c12[k], mp.c13[k], mp.c23[k]); });
    return le + lt;
}

// decrease_triangle_costs_func::min_marginal (:275-280)
__device__ __forceinline__ float min_marginal(float x, float y, float z)
{
    float mm1 = fminf(__fadd_rn(__fadd_rn(x, y), z), fminf(__fadd_rn(x, y), __fadd_rn(x, z)));
    float yz = __fadd_rn(y, z);
    float mm0 = (0.0 < (double)yz) ? 0.0f : yz;
    return __fsub_rn(mm1, mm0);
}

__device__ __forceinline__ float sub_scaled(float a, double s, float mm)
{
    return (float)__dsub_rn((double)a, __dmul_rn(s, (double)mm));
}
__device__ __forceinline__ float add_scaled(float a, double s, float mm)
{
    return (float)__dadd_rn((double)a, __dmul_rn(s, (double)mm));
}

// one iteration (:350-354): send_messages_to_triplets (:241-269) fused with
// the six min-marginal moves of send_messages_to_edges (:271-348); then each
// covered edge takes the RSUM of its incoming messages.
template <class Team>
__device__ void mp_iteration(const Team &t, const Mp &mp)
{
    const double third = 1.0 / 3.0, half = 1.0 / 2.0;
    // the six moves of one triangle, from its three costs (the edges' shares
    // added); writes the triangle's costs and its messages to the edges
    auto moves = [&](int64_t k, float t12, float t13, float t23) {
        float e12 = 0.0f, e13 = 0.0f, e23 = 0.0f;
        {
            float mm = min_marginal(t12, t13, t23);
            t12 = sub_scaled(t12, third, mm);
            e12 = add_scaled(e12, third, mm);
        }
        {
            float mm = min_marginal(t13, t12, t23);
            t13 = sub_scaled(t13, half, mm);
            e13 = add_scaled(e13, half, mm);
        }
        {
            float mm = min_marginal(t23, t12, t13);
            t23 = __fsub_rn(t23, mm);
            e23 = __fadd_rn(e23, mm);
        }
        {
            float mm = min_marginal(t12, t13, t23);
            t12 = sub_scaled(t12, half, mm);
            e12 = add_scaled(e12, half, mm);
        }
        {
            float mm = min_marginal(t13, t12, t23);
            t13 = __fsub_rn(t13, mm);
            e13 = __fadd_rn(e13, mm);
        }
        {
            float mm = min_marginal(t12, t13, t23);
            t12 = __fsub_rn(t12, mm);
            e12 = __fadd_rn(e12, mm);
        }
        mp.c12[k] = t12;
        mp.c13[k] = t13;
        mp.c23[k] = t23;
        mp.slot[mp.pos[3 * k]] = e12;
        mp.slot[mp.pos[3 * k + 1]] = e13;
        mp.slot[mp.pos[3 * k + 2]] = e23;
    };
    {
        // two triangles a thread at a time: their loads and the gathers of
        // the edges' shares are in flight together
        const int64_t S = t.size();
        int64_t k = t.rank();
        for (; k + S < mp.T; k += 2 * S) {
            const int64_t k2 = k + S;
            const int32_t a12 = mp.e12[k], a13 = mp.e13[k], a23 = mp.e23[k];
            const int32_t b12 = mp.e12[k2], b13 = mp.e13[k2], b23 = mp.e23[k2];
            const float ac12 = mp.c12[k], ac13 = mp.c13[k], ac23 = mp.c23[k];
            const float bc12 = mp.c12[k2], bc13 = mp.c13[k2], bc23 = mp.c23[k2];
            const float as12 = mp.share[a12], as13 = mp.share[a13], as23 = mp.share[a23];
            const float bs12 = mp.share[b12], bs13 = mp.share[b13], bs23 = mp.share[b23];
            moves(k, __fadd_rn(ac12, as12), __fadd_rn(ac13, as13), __fadd_rn(ac23, as23));
            moves(k2, __fadd_rn(bc12, bs12), __fadd_rn(bc13, bs13), __fadd_rn(bc23, bs23));
        }
        for (; k < mp.T; k += S)
            moves(k, __fadd_rn(mp.c12[k], mp.share[mp.e12[k]]), __fadd_rn(mp.c13[k], mp.share[mp.e13[k]]),
                  __fadd_rn(mp.c23[k], mp.share[mp.e23[k]]));
    }
    t.sync();
    // covered edges: c = 0 + RSUM(messages); long runs by a warp
    {
        // four edges a thread at a time: offsets, then the messages, then
        // the stores
        constexpr int U = 4;
        const int64_t S = t.size();
        int64_t e0 = t.rank();
        for (; e0 + (U - 1) * S < mp.E; e0 += U * S) {
            int32_t s[U], n[U];
            float c[U];
#pragma unroll
            for (int k = 0; k < U; ++k) {
                s[k] = mp.inc_off[e0 + k * S];
                n[k] = mp.inc_off[e0 + k * S + 1] - s[k];
            }
#pragma unroll
            for (int k = 0; k < U; ++k)
                c[k] = (n[k] == 0 || n[k] > RSUM_THREAD_MAX) ? 0.0f : __fadd_rn(0.0f, rsum_upto8(mp.slot + s[k], n[k]));
#pragma unroll
            for (int k = 0; k < U; ++k)
                if (n[k] != 0 && n[k] <= RSUM_THREAD_MAX) {
                    mp.cost[e0 + k * S] = c[k];
                    mp.share[e0 + k * S] = __fdiv_rn(c[k], (float)n[k]);
                }
        }
        for (; e0 < mp.E; e0 += S) {
            const int32_t s = mp.inc_off[e0], n = mp.inc_off[e0 + 1] - s;
            if (n == 0 || n > RSUM_THREAD_MAX) continue;
            const float c = __fadd_rn(0.0f, rsum_upto8(mp.slot + s, n));
            mp.cost[e0] = c;
            mp.share[e0] = __fdiv_rn(c, (float)n);
        }
    }
    for (int64_t q = team_warp(t); q < mp.nlong; q += team_nwarps(t)) {
        const int32_t e = mp.longe[q];
        const int32_t s = mp.inc_off[e], n = mp.inc_off[e + 1] - s;
        const float c = __fadd_rn(0.0f, rsum_warp(n, [&](int64_t k) { return mp.slot[s + k]; }));
        if (lane_id() == 0) {
            mp.cost[e] = c;
            mp.share[e] = __fdiv_rn(c, (float)n);
        }
    }
    t.sync();
}

// dual_update_cycle_length (src/dual_solver.cu:7-35).  On success the graph
// in the top slot is replaced by the reparametrised one.
template <class Team>
__device__ double dual_update_cycle_length(const Team &t, Scratch &sc, char *sm, Graph &A, int c, int num_iter,
                                           float tri_factor, float tol, int64_t *num_tri, bool *failed,
                                           bool *no_cycles)
{
    uint64_t m = sc.arena.mark();
    TriBuf tb;
    prof_mark(t, sc, PH_OTHER);
    conflicted_cycles(t, sc, sm, A, c, tri_factor, tol, tb);
    prof_mark(t, sc, PH_CYC_SEARCH);
    *failed = !sc.arena.ok();
    if (*failed) {
        sc.arena.release(m);
        return 0.0;
    }
    *num_tri = tb.count;
    *no_cycles = tb.none != 0;
    if (tb.count == 0) {
        sc.arena.release(m);
        return graph_lb(t, sc, A);
    }
    Mp mp;
    if (!mp_build(t, sc, sm, A, tb, mp)) {
        *failed = true;
        sc.arena.release(m);
        return 0.0;
    }
    prof_mark(t, sc, PH_MP_BUILD);
    double prev = 0.0;
    for (int it = 0; it < num_iter; ++it) {
        double lb = mp_lower_bound(t, sc, mp);
        sc.alg_bytes += 4.0 * (double)mp.E + 12.0 * (double)mp.T;
        if (it > 0 && (lb - prev) < 1e-3) break;
        mp_iteration(t, mp);
        sc.alg_bytes += 84.0 * (double)mp.T + 12.0 * (double)mp.E;
        prev = lb;
    }
    const double fin = mp_lower_bound(t, sc, mp);
    prof_mark(t, sc, PH_MP_ITER);
    Graph g;
    g.row = mp.row;
    g.col = mp.col;
    g.cost = mp.cost;
    g.n = mp.E;
    graph_set_dims(t, sc, sm, g);
    Graph ng = graph_commit(t, sc, g);
    prof_mark(t, sc, PH_DUAL_COMMIT);
    *failed = !sc.arena.ok();
    if (!*failed) A = ng;
    sc.arena.release(m);
    return fin;
}

// dual_solver (src/dual_solver.cu:37-63); an arena overflow plays the role of
// the reference's bad_alloc: the trivial bound of the current graph is
// returned and the graph keeps its last committed state.
template <class Team>
__device__ double dual_solver(const Team &t, Scratch &sc, char *sm, Graph &A, int max_len, int num_iter,
                              float tri_factor, int num_outer, float tol, int64_t *num_tri_last, int *oom)
{
    if (num_tri_last) *num_tri_last = 0;
    if (max_len < 3 || num_iter == 0 || num_outer == 0) return graph_lb(t, sc, A);
    double prev = 0.0, fin = 0.0;
    int64_t nt = 0;
    for (int o = 0; o < num_outer; ++o) {
        for (int c = 3; c <= max_len; ++c) {
            bool failed = false, none = false;
            fin = dual_update_cycle_length(t, sc, sm, A, c, num_iter, tri_factor, tol, &nt, &failed, &none);
            if (failed) {
                sc.arena.failed = 0;
                if (oom) *oom = 1;
                return graph_lb(t, sc, A);
            }
            // the graph is unchanged and no repulsive edge can close a cycle:
            // the longer cycle lengths find nothing either (nt == 0 ends the
            // outer loop too)
            if (none) break;
        }
        if (nt == 0 || (o > 0 && (fin - prev) < 1e-3)) break;
        prev = fin;
    }
    if (num_tri_last) *num_tri_last = nt;
    return fin;
}

}  // namespace rama
