// cycles.cuh -- conflicted 3/4/5-cycle search on the CSR of attractive edges
// (src/conflicted_cycles_cuda.cu:13-343).  Each conflicted cycle is emitted
// as triangles.  Expansions (a rep edge; a rep edge and a neighbour; a rep
// edge and two neighbours) are taken in canonical order in chunks of 2^24,
// each emitting its triangles in the reference's order; a chunk whose
// emissions exceed the room left in the budget keeps them round-robin: the
// first K emissions of every expansion (K as large as fits) and one more for
// the first expansions that have one, until the budget is full.  Computed by
// count -> K -> scan -> write.
#pragma once
#include "graph.cuh"

namespace rama {

struct TriBuf {
    int32_t *t1, *t2, *t3;  // capacity budget + 1
    int64_t budget;
    int64_t count;  // the reference's triangle counter (budget+1 once overflowed)
    int64_t num;    // valid entries: min(count, budget)
    int none;       // no repulsive edge has an attractive edge at both ends: no cycle of any length
};

__device__ __forceinline__ int count_common(const int32_t *adj, int32_t a0, int32_t a1, int32_t b0, int32_t b1)
{
    int c = 0;
    while (a0 < a1 && b0 < b1) {
        int32_t x = adj[a0], y = adj[b0];
        c += (x == y);
        a0 += (x <= y);
        b0 += (y <= x);
    }
    return c;
}

// calls f(mid) for the common neighbours in ascending order while f returns true
template <class F>
__device__ __forceinline__ void for_common(const int32_t *adj, int32_t a0, int32_t a1, int32_t b0, int32_t b1, F f)
{
    while (a0 < a1 && b0 < b1) {
        int32_t x = adj[a0], y = adj[b0];
        if (x == y && !f(x)) return;
        a0 += (x <= y);
        b0 += (y <= x);
    }
}

__device__ __forceinline__ void write_tri(TriBuf &tb, int64_t pos, int32_t a, int32_t b, int32_t c)
{
    if (pos >= tb.budget) return;
    int32_t lo = min(a, min(b, c)), hi = max(a, max(b, c));
    int32_t md = max(min(a, b), min(max(a, b), c));
    tb.t1[pos] = lo;
    tb.t2[pos] = md;
    tb.t3[pos] = hi;
}

// remove degenerate triangles, sort lexicographically, unique (the first n
// entries of the buffer); returns the new count
template <class Team>
__device__ int64_t tri_normalize(const Team &t, Scratch &sc, char *sm, int32_t *t1, int32_t *t2, int32_t *t3, int64_t n,
                                 int32_t nmax)
{
    if (n == 0) return 0;
    const int nb = bits_for((uint64_t)(nmax > 0 ? nmax : 1));
    uint64_t m = sc.arena.mark();
    uint64_t *k1 = sc.arena.take<uint64_t>(n + 1), *k2 = sc.arena.take<uint64_t>(n + 1);
    uint64_t *u1 = sc.arena.take<uint64_t>(n + 1), *u2 = sc.arena.take<uint64_t>(n + 1);
    int32_t *tlo = sc.arena.take<int32_t>(n + 1);
    if (!sc.arena.ok()) return 0;
    const uint64_t mask = (nb == 0) ? 0 : ((uint64_t(1) << nb) - 1);
    // drop degenerate triangles; key the rest by lo and (md, hi)
    const int64_t w = team_compact(
        t, sc, sm, n, [&](int64_t k) { return !(t1[k] == t2[k] || t1[k] == t3[k] || t2[k] == t3[k]); },
        [&](int64_t k, int64_t p) {
            int32_t a = t1[k], b = t2[k], c = t3[k];
            int32_t lo = min(a, min(b, c)), hi = max(a, max(b, c));
            int32_t md = max(min(a, b), min(max(a, b), c));
            tlo[p] = lo;
            u1[p] = pack_key(md, hi, nb);
        });
    // sort by (lo, md, hi): bucket by lo (identical triangles may end in any
    // order among themselves, they are merged below) ...
    bool done = false;
    {
        uint64_t bm = sc.arena.mark();
        int32_t *bst = sc.arena.take<int32_t>((int64_t)nmax + 2);
        int32_t *bidx = sc.arena.take<int32_t>(w + 1);
        if (sc.arena.ok() && w < (int64_t(1) << 31)) {
            // the payload of each triangle is its lo, so every sorted position
            // rebuilds its keys from its own entries
            auto lo = [&](int64_t i) { return tlo[i]; };
            done = team_bucket_sort_ex(
                t, sc, sm, w, nmax + 1, lo, lo, [&](int64_t i) { return u1[i]; }, lo, k2, bidx, bst);
            if (done) {
                team_for_batched(
                    t, w, [&](int64_t p) { return make_longlong2((long long)bidx[p], (long long)k2[p]); },
                    [&](int64_t p, longlong2 v) {
                        const uint64_t mh = (uint64_t)v.y;
                        k1[p] = pack_key((int32_t)v.x, (int32_t)(mh >> nb), nb);
                        u2[p] = mh & mask;
                    });
                t.sync();
                uint64_t *tp = u1;
                u1 = u2;
                u2 = tp;
            }
        }
        sc.arena.release(bm);
    }
    if (!done) {
        // ... or by LSD radix: stable sort by hi carrying (lo, md), then by (lo, md) carrying hi
        for (int64_t k = t.rank(); k < w; k += t.size()) {
            const uint64_t mh = u1[k];
            k1[k] = mh & mask;
            u1[k] = pack_key(tlo[k], (int32_t)(mh >> nb), nb);
        }
        t.sync();
        team_sort_pairs(t, sc, sm, k1, u1, k2, u2, w, nb);
        for (int64_t k = t.rank(); k < w; k += t.size()) {
            uint64_t tmp = u1[k];
            u1[k] = k1[k];  // hi becomes the value
            k1[k] = tmp;
        }
        t.sync();
        team_sort_pairs(t, sc, sm, k1, u1, k2, u2, w, 2 * nb);
    }
    const int64_t u = team_compact(
        t, sc, sm, w, [&](int64_t k) { return k == 0 || k1[k] != k1[k - 1] || u1[k] != u1[k - 1]; },
        [&](int64_t k, int64_t p) {
            t1[p] = (int32_t)(k1[k] >> nb);
            t2[p] = (int32_t)(k1[k] & mask);
            t3[p] = (int32_t)u1[k];
        });
    sc.arena.release(m);
    return u;
}

// Expansion stage over X expansions (X given as an exclusive scan xo[R+1]
// over rep edges; xo == nullptr means one expansion per rep edge).  For each
// expansion: count(x) emissions, then write them at `count + prefix`.
// Processed in chunks so that a filled budget stops the work early.
__device__ __forceinline__ int64_t expansion_owner(const int64_t *xo, int64_t R, int64_t x)
{
    if (!xo) return x;
    int64_t lo = 0, hi = R;  // largest r with xo[r] <= x
    while (lo < hi) {
        int64_t mid = (lo + hi + 1) >> 1;
        if (xo[mid] <= x)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// emit(r, loc, pos, keep) writes the first `keep` emissions of an expansion
// at pos, pos + 1, ...
template <class Team, class Count, class Emit>
__device__ void expansion_stage(const Team &t, Scratch &sc, char *sm, TriBuf &tb, const int64_t *xo, int64_t R,
                                int64_t X, Count cnt, Emit emit)
{
    const int64_t CH = int64_t(1) << 24;
    const int64_t KALL = int64_t(1) << 40;  // no truncation: every emission is kept
    uint64_t m = sc.arena.mark();
    int32_t *ccount = sc.arena.take<int32_t>(CH < X ? CH : X + 1);
    int64_t *cbase = sc.arena.take<int64_t>((CH < X ? CH : X) + 1);
    if (!sc.arena.ok()) return;
    for (int64_t x0 = 0; x0 < X && tb.count <= tb.budget; x0 += CH) {
        const int64_t xn = (X - x0) < CH ? (X - x0) : CH;
        // count
        // a warp takes 32 consecutive expansions: one search for the owner of
        // the first, then each lane steps forward to its own
        for (int64_t qb = (int64_t)team_warp(t) * 32; qb < xn; qb += (int64_t)team_nwarps(t) * 32) {
            int64_t r0 = lane_id() == 0 ? expansion_owner(xo, R, x0 + qb) : 0;
            r0 = __shfl_sync(FULL, r0, 0);
            const int64_t q = qb + lane_id();
            if (q >= xn) continue;
            const int64_t x = x0 + q;
            int64_t r = xo ? r0 : x;
            if (xo) {
                int steps = 0;  // long runs of rep edges without expansions: search instead
                while (r < R && xo[r + 1] <= x && ++steps <= 64) ++r;
                if (steps > 64) r = expansion_owner(xo, R, x);
            }
            ccount[q] = cnt(r, xo ? x - xo[r] : 0);
        }
        t.sync();
        const int64_t start = tb.count;
        const int64_t rem = tb.budget - start;
        const int64_t tot = team_sum<Team, int64_t>(t, sc, sm, xn, [&](int64_t q) -> int64_t { return ccount[q]; });
        // round-robin when the chunk does not fit: the largest K with
        // sum_q min(count_q, K) <= rem, and `extra` expansions keep one more
        int64_t K = KALL, extra = 0;
        if (tot > rem) {
            const int32_t mx = team_max<Team, int32_t>(t, sc, sm, xn, 0, [&](int64_t q) { return ccount[q]; });
            int64_t lo = 0, hi = mx, slo = 0;
            for (int guard = 0; lo < hi && guard < 40; ++guard) {
                const int64_t k = (lo + hi + 1) >> 1;
                const int64_t s = team_sum<Team, int64_t>(t, sc, sm, xn, [&](int64_t q) -> int64_t {
                    const int64_t c = ccount[q];
                    return c < k ? c : k;
                });
                if (s <= rem) {
                    lo = k;
                    slo = s;
                } else {
                    hi = k - 1;
                }
            }
            K = lo;
            extra = rem - slo;
        }
        // positions: one scan of (kept below K) << 25 | (has more than K);
        // count_q is replaced by the number it keeps
        team_scan<Team, int64_t>(
            t, sc, sm, xn,
            [&](int64_t q) -> int64_t {
                const int64_t c = ccount[q];
                return ((c < K ? c : K) << 25) | (c > K ? 1 : 0);
            },
            [&](int64_t q, int64_t pre, int64_t v) {
                const int64_t pmin = pre >> 25, pbig = pre & ((int64_t(1) << 25) - 1);
                cbase[q] = pmin + (pbig < extra ? pbig : extra);
                ccount[q] = (int32_t)((v >> 25) + ((v & 1) && pbig < extra ? 1 : 0));
            });
        for (int64_t qb = (int64_t)team_warp(t) * 32; qb < xn; qb += (int64_t)team_nwarps(t) * 32) {
            const int64_t q = qb + lane_id();
            const bool work = q < xn && ccount[q] != 0;
            if (!__any_sync(FULL, work)) continue;
            int64_t r0 = lane_id() == 0 ? expansion_owner(xo, R, x0 + qb) : 0;
            r0 = __shfl_sync(FULL, r0, 0);
            if (!work) continue;
            const int64_t x = x0 + q;
            int64_t r = xo ? r0 : x;
            if (xo) {
                int steps = 0;  // long runs of rep edges without expansions: search instead
                while (r < R && xo[r + 1] <= x && ++steps <= 64) ++r;
                if (steps > 64) r = expansion_owner(xo, R, x);
            }
            emit(r, xo ? x - xo[r] : 0, start + cbase[q], (int64_t)ccount[q]);
        }
        t.sync();
        tb.count = tot <= rem ? start + tot : tb.budget + 1;
    }
    sc.arena.release(m);
}

// conflicted_cycles_cuda (:222-343).  Triangles land in tb (allocated here
// in the temporaries); tb.count is the reference's counter.
template <class Team>
__device__ void conflicted_cycles(const Team &t, Scratch &sc, char *sm, const Graph &A, int max_len, float tri_factor,
                                  float tol, TriBuf &tb)
{
    tb.count = 0;
    tb.num = 0;
    tb.budget = 0;
    tb.none = 0;
    tb.t1 = tb.t2 = tb.t3 = nullptr;
    if (max_len < 3 || A.n == 0) return;
    // the smallest cost: known from the pass that built the graph, or one pass
    const float mn = A.cmin == A.cmin
                         ? A.cmin
                         : team_min<Team, float>(t, sc, sm, A.n, 3.4e38f, [&](int64_t e) { return A.cost[e]; });
    const float thresh = mn * tol;          // determine_threshold (:170-174)
    const float pos_tol = -1.0f * thresh;   // create_matrices (:176-220)
    const int32_t N = A.max_dim();
    // Every conflicted cycle closes a repulsive edge (u, v) with a path of
    // attractive edges, so both u and v have an attractive edge.  Repulsive
    // edges without one at either end emit nothing: they are left out of the
    // search (the emission order of the others, and so the budget's
    // truncation, is unchanged), and a graph with none left needs no CSR.
    int64_t *ridx = sc.arena.take<int64_t>(A.n + 1);
    int8_t *haspos = sc.arena.take<int8_t>((int64_t)N + 1);
    if (!sc.arena.ok()) return;
    for (int64_t v = t.rank(); v < N; v += t.size()) haspos[v] = 0;
    t.sync();
    int64_t pc = 0;
    {
        // four edges a thread at a time: costs, then the ends of the
        // attractive ones, then the marks
        constexpr int U = 4;
        const int64_t S = t.size();
        int64_t e0 = t.rank();
        for (; e0 + (U - 1) * S < A.n; e0 += U * S) {
            float c[U];
            int32_t a[U], b[U];
#pragma unroll
            for (int k = 0; k < U; ++k) c[k] = A.cost[e0 + k * S];
#pragma unroll
            for (int k = 0; k < U; ++k)
                if (c[k] > pos_tol) {
                    a[k] = A.row[e0 + k * S];
                    b[k] = A.col[e0 + k * S];
                }
#pragma unroll
            for (int k = 0; k < U; ++k)
                if (c[k] > pos_tol) {
                    haspos[a[k]] = 1;
                    haspos[b[k]] = 1;
                    ++pc;
                }
        }
        for (; e0 < A.n; e0 += S)
            if (A.cost[e0] > pos_tol) {
                haspos[A.row[e0]] = 1;
                haspos[A.col[e0]] = 1;
                ++pc;
            }
    }
    const int64_t P = team_total<Team, int64_t>(t, sc, sm, pc);
    // one pass counts both: the low 32 bits count every repulsive edge (the
    // budget counts them all, :247), the high bits the kept ones; the kept
    // ones are compacted only when there are any
    auto rep_code = [&](int64_t e) -> int64_t {
        if (!(A.cost[e] < thresh)) return 0;
        return (haspos[A.row[e]] && haspos[A.col[e]]) ? (int64_t(1) << 32) + 1 : 1;
    };
    const int64_t packed = team_sum<Team, int64_t>(t, sc, sm, A.n, rep_code);
    const int64_t Rall = packed & 0xffffffffll;
    const int64_t R = packed >> 32;
    sc.alg_bytes += 12.0 * (double)A.n;
    if (P == 0 || R == 0) {
        tb.none = 1;
        prof_mark(t, sc, PH_CYCLES);
        return;
    }
    team_scan<Team, int64_t>(
        t, sc, sm, A.n, [&](int64_t e) -> int64_t { return rep_code(e) >> 32; },
        [&](int64_t e, int64_t pre, int64_t v) {
            if (v) ridx[pre] = e;
        });
    prof_mark(t, sc, PH_CYCLES);
    Csr C = build_symmetric_csr(t, sc, sm, A, N, [&](int64_t e) { return A.cost[e] > pos_tol; }, false);
    prof_mark(t, sc, PH_CSR);
    const int64_t budget = (int64_t)(int32_t)(tri_factor * (float)Rall);  // (:247)
    tb.budget = budget < 0 ? 0 : budget;
    tb.t1 = sc.arena.take<int32_t>(tb.budget + 1);
    tb.t2 = sc.arena.take<int32_t>(tb.budget + 1);
    tb.t3 = sc.arena.take<int32_t>(tb.budget + 1);
    int64_t *xo = sc.arena.take<int64_t>(R + 2);
    if (!sc.arena.ok()) return;
    const int32_t *off = C.off;
    const int32_t *adj = C.adj;
    auto rv1 = [&](int64_t r) { return A.row[ridx[r]]; };
    auto rv2 = [&](int64_t r) { return A.col[ridx[r]]; };
    // ---- 3-cycles: find_triangles_parallel (:31-61)
    {
        TriBuf &T = tb;
        expansion_stage(
            t, sc, sm, T, nullptr, R, R,
            [&](int64_t r, int64_t) {
                int32_t v1 = rv1(r), v2 = rv2(r);
                return count_common(adj, off[v1], off[v1 + 1], off[v2], off[v2 + 1]);
            },
            [&](int64_t r, int64_t, int64_t pos, int64_t keep) {
                int32_t v1 = rv1(r), v2 = rv2(r);
                int64_t e = 0;
                for_common(adj, off[v1], off[v1 + 1], off[v2], off[v2 + 1], [&](int32_t mid) {
                    write_tri(T, pos + e, v1, v2, mid);
                    return ++e < keep;
                });
            });
    }
    // ---- 4-cycles: find_quadrangles_parallel (:63-101)
    if (max_len >= 4 && tb.count < tb.budget) {
        tb.count = tri_normalize(t, sc, sm, tb.t1, tb.t2, tb.t3, tb.count, N);
        const int64_t X = team_scan<Team, int64_t>(
            t, sc, sm, R, [&](int64_t r) -> int64_t { int32_t v1 = rv1(r); return off[v1 + 1] - off[v1]; },
            [&](int64_t r, int64_t pre, int64_t) { xo[r] = pre; });
        if (t.rank() == 0) xo[R] = X;
        t.sync();
        TriBuf &T = tb;
        expansion_stage(
            t, sc, sm, T, xo, R, X,
            [&](int64_t r, int64_t loc) {
                int32_t v1 = rv1(r), v2 = rv2(r);
                int32_t n1 = adj[off[v1] + loc];
                return 2 * count_common(adj, off[n1], off[n1 + 1], off[v2], off[v2 + 1]);
            },
            [&](int64_t r, int64_t loc, int64_t pos, int64_t keep) {
                int32_t v1 = rv1(r), v2 = rv2(r);
                int32_t n1 = adj[off[v1] + loc];
                int64_t e = 0;
                for_common(adj, off[n1], off[n1 + 1], off[v2], off[v2 + 1], [&](int32_t mid) {
                    write_tri(T, pos + e, v1, v2, n1);
                    if (++e >= keep) return false;
                    write_tri(T, pos + e, v2, n1, mid);
                    return ++e < keep;
                });
            });
    }
    // ---- 5-cycles: find_pentagons_parallel (:103-148)
    if (max_len >= 5 && tb.count < tb.budget) {
        tb.count = tri_normalize(t, sc, sm, tb.t1, tb.t2, tb.t3, tb.count, N);
        const int64_t X = team_scan<Team, int64_t>(
            t, sc, sm, R,
            [&](int64_t r) -> int64_t {
                int32_t v1 = rv1(r), v2 = rv2(r);
                return (int64_t)(off[v1 + 1] - off[v1]) * (int64_t)(off[v2 + 1] - off[v2]);
            },
            [&](int64_t r, int64_t pre, int64_t) { xo[r] = pre; });
        if (t.rank() == 0) xo[R] = X;
        t.sync();
        TriBuf &T = tb;
        expansion_stage(
            t, sc, sm, T, xo, R, X,
            [&](int64_t r, int64_t loc) {
                int32_t v1 = rv1(r), v2 = rv2(r);
                int64_t d1 = off[v1 + 1] - off[v1];
                int32_t n1 = adj[off[v1] + (int32_t)(loc % d1)];
                int32_t n2 = adj[off[v2] + (int32_t)(loc / d1)];
                if (n1 == n2) return 0;
                return 3 * count_common(adj, off[n1], off[n1 + 1], off[n2], off[n2 + 1]);
            },
            [&](int64_t r, int64_t loc, int64_t pos, int64_t keep) {
                int32_t v1 = rv1(r), v2 = rv2(r);
                int64_t d1 = off[v1 + 1] - off[v1];
                int32_t n1 = adj[off[v1] + (int32_t)(loc % d1)];
                int32_t n2 = adj[off[v2] + (int32_t)(loc / d1)];
                if (n1 == n2) return;
                int64_t e = 0;
                for_common(adj, off[n1], off[n1 + 1], off[n2], off[n2 + 1], [&](int32_t mid) {
                    write_tri(T, pos + e, v1, v2, n1);
                    if (++e >= keep) return false;
                    write_tri(T, pos + e, v2, n1, mid);
                    if (++e >= keep) return false;
                    write_tri(T, pos + e, v2, mid, n2);
                    return ++e < keep;
                });
            });
    }
    tb.num = tb.count < tb.budget ? tb.count : tb.budget;
    sc.alg_bytes += 8.0 * (double)R + 4.0 * (double)C.m2 + 12.0 * (double)tb.num;
}

}  // namespace rama
