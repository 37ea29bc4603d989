// matching.cuh -- vertex-based matching contraction set
// (src/maximum_matching_vertex_based.cu:10-137, src/rama_cuda.cu:54-62).
#pragma once
#include "graph.cuh"

namespace rama {

// Returns the number of matched vertices; map_out (capacity >= max col + 1)
// receives the compressed contraction map and *M_out its length.
//
// pick_best_neighbour (:10-47) scans a vertex's row of the symmetric CSR and
// keeps the first neighbour of largest cost above the threshold that is
// unmatched.  Rows are sorted by neighbour id, so that is the unmatched
// neighbour with the largest (cost, -id).  Here every edge offers itself to
// both endpoints by a 64-bit atomicMax on (order-preserving cost bits,
// complemented neighbour id), which gives the same choice without building
// the CSR.  The offers of one iteration go to one of two key arrays; the
// match pass reads it and clears the other for the next iteration.
template <class Team>
__device__ int32_t matching_contraction_map(const Team &t, Scratch &sc, char *sm, const Graph &A, float mm,
                                            int32_t *map_out, int32_t *M_out)
{
    int32_t mc = team_max<Team, int32_t>(t, sc, sm, A.n, -1, [&](int64_t e) { return A.col[e]; });
    const int32_t M = mc + 1;
    *M_out = M;
    uint64_t mark = sc.arena.mark();
    int32_t *nm = sc.arena.take<int32_t>((int64_t)M + 1);
    int32_t *matched = sc.arena.take<int32_t>((int64_t)M + 1);
    unsigned long long *offer[2];
    offer[0] = sc.arena.take<unsigned long long>((int64_t)M + 1);
    offer[1] = sc.arena.take<unsigned long long>((int64_t)M + 1);
    int32_t *flags = sc.arena.take<int32_t>(16);
    if (!sc.arena.ok()) return 0;
    for (int64_t v = t.rank(); v < M; v += t.size()) {
        nm[v] = (int32_t)v;
        matched[v] = 0;
        offer[0][v] = 0ull;
        offer[1][v] = 0ull;
    }
    if (t.rank() < 16) flags[t.rank()] = 0;
    // determine_matching_threshold (:76-86): mean of the non-negative costs
    // of the doubled edge list, CSUM over the directed list
    const double S = team_csum(t, sc, A.n, [&](int64_t e) -> double {
        float c = A.cost[e];
        return c >= 0.0f ? (double)c : 0.0;
    });
    const int64_t K = team_sum<Team, int64_t>(t, sc, sm, A.n, [&](int64_t e) -> int64_t { return A.cost[e] >= 0.0f; });
    int32_t prev = 0;
    if (K > 0) {
        const float sum_f = (float)(2.0 * S);
        const float thresh = (mm * sum_f) / (float)(2 * K);
        for (int it = 0; it < 10; ++it) {
            unsigned long long *cur_offer = offer[it & 1], *next_offer = offer[(it + 1) & 1];
            // pick_best_neighbour: every edge above the threshold between two
            // unmatched vertices offers itself to both
            for (int64_t e = t.rank(); e < A.n; e += t.size()) {
                const float c = A.cost[e];
                if (!(c > thresh)) continue;
                const int32_t u = A.row[e], v = A.col[e];
                if (u == v || matched[u] || matched[v]) continue;
                const unsigned long long hi = (unsigned long long)float_ordered(c) << 32;
                atomicMax(&cur_offer[u], hi | (unsigned long long)(~(uint32_t)v));
                atomicMax(&cur_offer[v], hi | (unsigned long long)(~(uint32_t)u));
            }
            t.sync();
            // match_neighbours (:49-74): mutual best offers pair up
            for (int64_t v = t.rank(); v < M; v += t.size()) {
                next_offer[v] = 0ull;
                if (matched[v]) continue;
                const unsigned long long o = cur_offer[v];
                if (!o) continue;
                const int32_t b = (int32_t)(~(uint32_t)(o & 0xffffffffull));
                const unsigned long long ob = cur_offer[b];
                if (ob && (int32_t)(~(uint32_t)(ob & 0xffffffffull)) == (int32_t)v) {
                    if ((int32_t)v < b) {
                        nm[b] = (int32_t)v;
                        matched[v] = 1;
                        matched[b] = 1;
                        flags[it] = 1;
                    }
                }
            }
            t.sync();
            sc.alg_bytes += 20.0 * (double)A.n + 24.0 * (double)M;
            int32_t cur = team_sum<Team, int32_t>(t, sc, sm, M, [&](int64_t v) { return matched[v]; });
            float rel = (float)(cur - prev) / ((float)prev + 1.0f);
            prev = cur;
            if (!uread(&flags[it]) || (double)rel < 0.1) break;
            // vertices matched in this iteration must not take offers of the
            // next one: the offer pass reads `matched` after this sync
        }
    }
    compress_labels(t, sc, sm, nm, M, M - 1, map_out);
    sc.arena.release(mark);
    return prev;
}

}  // namespace rama
