// matching.cuh -- vertex-based matching contraction set
// (src/maximum_matching_vertex_based.cu:10-137, src/rama_cuda.cu:54-62).
#pragma once
#include "graph.cuh"

namespace rama {

// Returns the number of matched vertices; map_out (capacity >= max col + 1)
// receives the compressed contraction map and *M_out its length.
template <class Team>
__device__ int32_t matching_contraction_map(const Team &t, Scratch &sc, char *sm, const Graph &A, float mm,
                                            int32_t *map_out, int32_t *M_out)
{
    int32_t mc = team_max<Team, int32_t>(t, sc, sm, A.n, -1, [&](int64_t e) { return A.col[e]; });
    const int32_t M = mc + 1;
    *M_out = M;
    uint64_t mark = sc.arena.mark();
    int32_t *nm = sc.arena.take<int32_t>((int64_t)M + 1);
    int32_t *best = sc.arena.take<int32_t>((int64_t)M + 1);
    int32_t *matched = sc.arena.take<int32_t>((int64_t)M + 1);
    int32_t *flags = sc.arena.take<int32_t>(16);
    if (!sc.arena.ok()) return 0;
    for (int64_t v = t.rank(); v < M; v += t.size()) {
        nm[v] = (int32_t)v;
        best[v] = -1;
        matched[v] = 0;
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
        Csr C = build_symmetric_csr(t, sc, sm, A, M, [](int64_t) { return true; }, false);
        if (!sc.arena.ok()) return 0;
        for (int it = 0; it < 10; ++it) {
            // pick_best_neighbour / get_best_neighbour (:10-47)
            for (int64_t v = t.rank(); v < M; v += t.size()) {
                if (matched[v]) continue;
                float mx = thresh;
                int32_t id = -1;
                for (int32_t k = C.off[v]; k < C.off[v + 1]; ++k) {
                    float cv = C.w[k];
                    int32_t nb = C.adj[k];
                    if (cv <= mx || matched[nb] || nb == v) continue;
                    mx = cv;
                    id = nb;
                }
                best[v] = id;
            }
            t.sync();
            // match_neighbours (:49-74)
            for (int64_t v = t.rank(); v < M; v += t.size()) {
                if (((volatile int32_t *)matched)[v]) continue;
                int32_t b = best[v];
                if (b == -1 || ((volatile int32_t *)matched)[b]) continue;
                if (best[b] == (int32_t)v) {
                    int32_t hi = b > (int32_t)v ? b : (int32_t)v, lo = b > (int32_t)v ? (int32_t)v : b;
                    nm[hi] = lo;
                    matched[v] = 1;
                    matched[b] = 1;
                    flags[it] = 1;
                }
            }
            t.sync();
            sc.alg_bytes += 12.0 * (double)C.m2 + 16.0 * (double)M;
            int32_t cur = team_sum<Team, int32_t>(t, sc, sm, M, [&](int64_t v) { return matched[v]; });
            float rel = (float)(cur - prev) / ((float)prev + 1.0f);
            prev = cur;
            if (!uread(&flags[it]) || (double)rel < 0.1) break;
        }
    }
    compress_labels(t, sc, sm, nm, M, M - 1, map_out);
    sc.arena.release(mark);
    return prev;
}

}  // namespace rama
