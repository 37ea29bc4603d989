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
//
// Only edges above the threshold between two unmatched vertices can offer:
// the first iteration reads every edge and appends those to a candidate list,
// and each later iteration reads the list and appends its still-unmatched
// edges to the next one.  The vertices that received an offer go to a
// touched list, and only they are matched, cleared and counted.  Lists are
// appended with warp-aggregated atomics, so their order varies, but an
// atomicMax and the per-vertex match do not depend on the order: the map is
// the same as with full passes.
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
    int32_t *flags = sc.arena.take<int32_t>(64);  // [16 + 4k]: list sizes and new pairs of iteration k
    if (!sc.arena.ok()) return 0;
    for (int64_t v = t.rank(); v < M; v += t.size()) {
        nm[v] = (int32_t)v;
        matched[v] = 0;
        offer[0][v] = 0ull;
        offer[1][v] = 0ull;
    }
    if (t.rank() < 64) flags[t.rank()] = 0;
    // determine_matching_threshold (:76-86): mean of the non-negative costs
    // of the doubled edge list, CSUM over the directed list
    int64_t K = 0;
    const float *cost = A.cost;
    auto nonneg = [cost](int64_t e) -> float {
        const float c = cost[e];
        return c >= 0.0f ? c : 0.0f;
    };
    auto counted = [cost](int64_t e) { return cost[e] >= 0.0f; };
    double S;
    if constexpr (std::is_same<Team, GridTeam>::value)
        S = team_csum_count_outlined(t, sc, A.n, nonneg, counted, &K);
    else
        S = team_csum_count(t, sc, A.n, nonneg, counted, &K);
    int32_t prev = 0;
    if (K > 0) {
        const float sum_f = (float)(2.0 * S);
        const float thresh = (mm * sum_f) / (float)(2 * K);
        // candidate edges (u, v, order-preserving cost bits), two lists
        uint64_t lm = sc.arena.mark();
        const int64_t cap = A.n + 1;
        int2 *cand[2];
        uint32_t *cbits[2];
        cand[0] = sc.arena.take<int2>(cap);
        cand[1] = sc.arena.take<int2>(cap);
        cbits[0] = sc.arena.take<uint32_t>(cap);
        cbits[1] = sc.arena.take<uint32_t>(cap);
        int32_t *touched[2];
        touched[0] = sc.arena.take<int32_t>((int64_t)M + 1);
        touched[1] = sc.arena.take<int32_t>((int64_t)M + 1);
        if (!sc.arena.ok()) {
            sc.arena.release(mark);
            return 0;
        }
        prof_mark(t, sc, PH_MATCHING);
        int64_t ncand = 0;      // entries of the list read by this iteration
        int32_t ntouch_prev = 0;  // vertices touched by the previous iteration
        for (int it = 0; it < 10; ++it) {
            const int cur = it & 1, nxt = cur ^ 1;
            unsigned long long *cur_offer = offer[cur], *next_offer = offer[nxt];
            int32_t *cnt_next = flags + 16 + 4 * (it & 7);  // [0]: next list, [1]: touched, [2]: pairs
            int32_t *cnt_clear = flags + 16 + 4 * ((it + 1) & 7);
            // pick_best_neighbour: every live candidate offers itself to both
            // ends and stays a candidate for the next iteration.  A lane takes
            // MI edges at once (independent loads, gathers and atomics in
            // flight together); the CTA reserves list space for a tile of
            // blockDim * MI edges with one atomic per list.
            constexpr int MI = 4;
            int32_t *wsum = reinterpret_cast<int32_t *>(sm);  // per warp: list count, touched count; then bases
            auto offer_tile = [&](const int32_t (&u)[MI], const int32_t (&v)[MI], const uint32_t (&hb)[MI],
                                  const bool (&live)[MI]) {
                bool fu[MI], fv[MI];
#pragma unroll
                for (int k = 0; k < MI; ++k) {
                    fu[k] = fv[k] = false;
                    if (live[k]) {
                        const unsigned long long hi = (unsigned long long)hb[k] << 32;
                        fu[k] = atomicMax(&cur_offer[u[k]], hi | (unsigned long long)(~(uint32_t)v[k])) == 0ull;
                        fv[k] = atomicMax(&cur_offer[v[k]], hi | (unsigned long long)(~(uint32_t)u[k])) == 0ull;
                    }
                }
                int nl = 0, nt = 0;
#pragma unroll
                for (int k = 0; k < MI; ++k) {
                    nl += live[k];
                    nt += fu[k] + fv[k];
                }
                // lane prefixes by a warp scan of (touched << 16 | list)
                const int packed = (nt << 16) | nl;
                const int incl = warp_incl_scan(packed);
                const int w = warp_in_block(), nw = blockDim.x >> 5;
                if (lane_id() == 31) wsum[w] = incl;
                __syncthreads();
                if (threadIdx.x == 0) {
                    int tl = 0, tt = 0;
                    for (int q = 0; q < nw; ++q) {
                        const int x = wsum[q];
                        wsum[32 + q] = tl;
                        wsum[64 + q] = tt;
                        tl += x & 0xffff;
                        tt += x >> 16;
                    }
                    wsum[96] = tl ? atomicAdd(&cnt_next[0], tl) : 0;
                    wsum[97] = tt ? atomicAdd(&cnt_next[1], tt) : 0;
                }
                __syncthreads();
                int lbase = wsum[96] + wsum[32 + w] + ((incl - packed) & 0xffff);
                int tbase = wsum[97] + wsum[64 + w] + ((incl - packed) >> 16);
                __syncthreads();  // wsum is rewritten by the next tile
#pragma unroll
                for (int k = 0; k < MI; ++k) {
                    if (live[k]) {
                        cand[nxt][lbase] = make_int2(u[k], v[k]);
                        cbits[nxt][lbase] = hb[k];
                        ++lbase;
                    }
                    if (fu[k]) touched[cur][tbase++] = u[k];
                    if (fv[k]) touched[cur][tbase++] = v[k];
                }
            };
            // block-uniform loops over tiles (every thread takes part in the
            // tile's reservation)
            const int64_t TILE = (int64_t)blockDim.x * MI;
            const int64_t wofs = (int64_t)warp_in_block() * 32 * MI;
            if (it == 0) {
                // a lane takes MI = 4 consecutive edges: one 128-bit load per
                // array when the arrays are 16-byte aligned (the graph slot is)
                const bool vec = ((reinterpret_cast<uintptr_t>(A.row) | reinterpret_cast<uintptr_t>(A.col) |
                                   reinterpret_cast<uintptr_t>(A.cost)) & 15) == 0;
                for (int64_t tile = (int64_t)t.block() * TILE; tile < A.n; tile += (int64_t)t.nblocks() * TILE) {
                    int32_t u[MI], v[MI];
                    uint32_t hb[MI];
                    bool live[MI];
                    float c[MI];
                    const int64_t e0 = tile + wofs + (int64_t)lane_id() * MI;
                    if (vec && e0 + MI <= A.n) {
                        const float4 c4 = *reinterpret_cast<const float4 *>(A.cost + e0);
                        const int4 r4 = *reinterpret_cast<const int4 *>(A.row + e0);
                        const int4 l4 = *reinterpret_cast<const int4 *>(A.col + e0);
                        c[0] = c4.x, c[1] = c4.y, c[2] = c4.z, c[3] = c4.w;
                        u[0] = r4.x, u[1] = r4.y, u[2] = r4.z, u[3] = r4.w;
                        v[0] = l4.x, v[1] = l4.y, v[2] = l4.z, v[3] = l4.w;
#pragma unroll
                        for (int k = 0; k < MI; ++k) live[k] = c[k] > thresh;
                    } else {
#pragma unroll
                        for (int k = 0; k < MI; ++k) {
                            const int64_t e = e0 + k;
                            c[k] = e < A.n ? A.cost[e] : 0.0f;
                            live[k] = e < A.n && c[k] > thresh;
                            u[k] = live[k] ? A.row[e] : 0;
                            v[k] = live[k] ? A.col[e] : 0;
                        }
                    }
#pragma unroll
                    for (int k = 0; k < MI; ++k) {
                        hb[k] = float_ordered(c[k]);
                        live[k] = live[k] && u[k] != v[k];
                    }
                    offer_tile(u, v, hb, live);
                }
            } else {
                const int2 *L = cand[cur];
                const uint32_t *LB = cbits[cur];
                for (int64_t tile = (int64_t)t.block() * TILE; tile < ncand; tile += (int64_t)t.nblocks() * TILE) {
                    int32_t u[MI], v[MI];
                    uint32_t hb[MI];
                    bool live[MI];
#pragma unroll
                    for (int k = 0; k < MI; ++k) {
                        const int64_t q = tile + wofs + k * 32 + lane_id();
                        int2 uv = make_int2(0, 0);
                        hb[k] = 0;
                        if (q < ncand) {
                            uv = L[q];
                            hb[k] = LB[q];
                        }
                        u[k] = uv.x;
                        v[k] = uv.y;
                        live[k] = q < ncand;
                    }
                    int32_t mu[MI], mv[MI];
#pragma unroll
                    for (int k = 0; k < MI; ++k) {
                        mu[k] = live[k] ? matched[u[k]] : 1;
                        mv[k] = live[k] ? matched[v[k]] : 1;
                    }
#pragma unroll
                    for (int k = 0; k < MI; ++k) live[k] = live[k] && !mu[k] && !mv[k];
                    offer_tile(u, v, hb, live);
                }
            }
            if (t.rank() < 3) cnt_clear[t.rank()] = 0;  // counters of the next iteration
            t.sync();
            const int64_t nread = it == 0 ? A.n : ncand;
            const int32_t ntouch = uread(&cnt_next[1]);
            ncand = uread(&cnt_next[0]);
            // match_neighbours (:49-74): mutual best offers pair up; the other
            // offer buffer is cleared where the previous iteration wrote it
            const int32_t *T0 = touched[cur];
            const int32_t *Tp = touched[nxt];
            for (int64_t k = t.rank(); k < ntouch_prev; k += t.size()) next_offer[Tp[k]] = 0ull;
            // (the pairs are counted at their smaller end, one atomic per warp)
            int32_t mine = 0;
            auto offered = [](unsigned long long o) { return (int32_t)(~(uint32_t)(o & 0xffffffffull)); };
            auto pair_up = [&](int32_t v, int32_t b, unsigned long long ob) {
                if (ob && offered(ob) == v && v < b) {
                    nm[b] = v;
                    matched[v] = 1;
                    matched[b] = 1;
                    ++mine;
                }
            };
            {
                // four touched vertices a thread at a time: their chains of
                // loads (vertex, its offer, the partner's offer) overlap
                constexpr int U = 4;
                const int64_t S = t.size();
                int64_t k0 = t.rank();
                for (; k0 + (U - 1) * S < ntouch; k0 += U * S) {
                    int32_t v[U], b[U];
                    unsigned long long ob[U];
#pragma unroll
                    for (int k = 0; k < U; ++k) v[k] = T0[k0 + k * S];
#pragma unroll
                    for (int k = 0; k < U; ++k) b[k] = offered(cur_offer[v[k]]);
#pragma unroll
                    for (int k = 0; k < U; ++k) ob[k] = cur_offer[b[k]];
#pragma unroll
                    for (int k = 0; k < U; ++k) pair_up(v[k], b[k], ob[k]);
                }
                for (; k0 < ntouch; k0 += S) {
                    const int32_t v = T0[k0];
                    const int32_t b = offered(cur_offer[v]);
                    pair_up(v, b, cur_offer[b]);
                }
            }
            mine = warp_sum(mine);
            if (lane_id() == 0 && mine) atomicAdd(&cnt_next[2], mine);
            t.sync();
            sc.alg_bytes += 12.0 * (double)nread + 24.0 * (double)ntouch;
            const int32_t pairs = uread(&cnt_next[2]);
            const int32_t curm = prev + 2 * pairs;
            float rel = (float)(curm - prev) / ((float)prev + 1.0f);
            prev = curm;
            ntouch_prev = ntouch;
            if (it == 0) prof_mark(t, sc, PH_MATCH_FIRST);
            if (pairs == 0 || (double)rel < 0.1) break;
            // vertices matched in this iteration take no offers in the next:
            // the next offer pass reads `matched` after this sync
        }
        sc.arena.release(lm);
        prof_mark(t, sc, PH_MATCH_ITER);
    }
    // compress_label_sequence (include/rama_utils.h:160-177) of nm: the labels
    // in use are exactly the roots (nm[v] == v; a matched vertex points to its
    // smaller partner, which is a root), so a root's new label is its rank
    // among the roots
    int32_t *rank = reinterpret_cast<int32_t *>(offer[0]);  // the offers are dead by now
    team_scan<Team, int64_t>(
        t, sc, sm, M, [&](int64_t v) -> int64_t { return nm[v] == (int32_t)v ? 1 : 0; },
        [&](int64_t v, int64_t pre, int64_t) { rank[v] = (int32_t)pre; });
    team_for_batched(
        t, M, [&](int64_t v) { return rank[nm[v]]; }, [&](int64_t v, int32_t r) { map_out[v] = r; });
    t.sync();
    prof_mark(t, sc, PH_MATCH_LABELS);
    sc.arena.release(mark);
    return prev;
}

}  // namespace rama
