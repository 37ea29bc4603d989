// solver.cuh -- the whole multicut solve of one instance by one team
// (src/rama_cuda.cu:64-212).  Runs on the device end to end: no host
// round-trips between rounds.
#pragma once
#include "matching.cuh"
#include "mp.cuh"
#include "woc.cuh"

namespace rama {

struct Options {
    int32_t max_cycle_length_lb;
    int32_t num_dual_itr_lb;
    int32_t max_cycle_length_primal;
    int32_t num_dual_itr_primal;
    int32_t num_outer_itr_dual;
    float mean_multiplier_mm;
    float matching_thresh_crossover_ratio;
    float tri_memory_factor;
    int32_t only_compute_lb;
    int32_t max_time_sec;
    int32_t dump_timeline;
    int32_t verbose;
    int32_t sanitize_graph;
    int32_t woc_pentagons;
};

// One instance: inputs, outputs and statistics (device memory).
struct Instance {
    Options opts;
    const int32_t *i, *j;
    const float *c;
    int64_t n;
    int32_t *labels;
    int64_t labels_cap;
    int32_t *timeline;       // optional: rounds x num_labels
    int64_t timeline_cap;    // entries
    int64_t *prof;           // optional: PH_COUNT nanosecond counters, then PH_COUNT byte counters
    char *ws;                // workspace slice of this instance (CTA solves)
    uint64_t ws_bytes;
    // outputs
    int64_t num_labels;
    double lb;
    int32_t status;
    int32_t rounds;
    int32_t matching_rounds;
    int32_t mst_rounds;
    int32_t timeline_rounds;
    int32_t dual_oom;
    int64_t triangles_initial;
    int64_t arena_peak;
    int64_t arena_want;      // workspace bytes a refused allocation needed (0: none refused)
    int64_t edges_after_dual;
    double alg_bytes;
};

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

template <class Team>
__device__ void solve_instance(const Team &t, char *sm, Scratch sc, Instance *io)
{
    const Options o = io->opts;
    if (t.rank() == 0) *sc.err = 0;  // the first team primitive below syncs before any reader
    sc.prof = io->prof;
    if (sc.prof && t.leader()) sc.tlast = prof_now();
    const int64_t n = io->n;
    const int32_t *I = io->i, *J = io->j;
    const float *Cc = io->c;
    int32_t status = ERR_NONE;
    int32_t rounds = 0, mrounds = 0, wrounds = 0, tl_rounds = 0;
    int oom = 0;
    int64_t ntri = 0;
    double lb = 0.0;
    int64_t num_labels = 0;
    int64_t eafter = 0;
    uint64_t *slot = reinterpret_cast<uint64_t *>(sc.arena.take<uint64_t>(4));
    const int64_t bad_in = team_sum<Team, int64_t>(t, sc, sm, n, [&](int64_t e) -> int64_t {
        int32_t a = I[e], b = J[e];
        return (a < 0 || b < 0 || a == b) ? 1 : 0;
    });
    if (!sc.arena.ok()) status |= ERR_ARENA;
    if (bad_in) status |= ERR_INVALID_ARG;
    int32_t *idmap = nullptr;
    int32_t idsize = 0;
    int64_t nin = n;
    if (status == ERR_NONE && n > 0 && o.sanitize_graph) {
        int32_t *si, *sj;
        float *sw;
        nin = sanitize_edges(t, sc, sm, I, J, Cc, n, si, sj, sw, idmap, idsize);
        I = si;
        J = sj;
        Cc = sw;
        if (!sc.arena.ok()) status |= ERR_ARENA;
    }
    if (status == ERR_NONE && n > 0) {
        uint64_t t0 = 0;
        if (t.rank() == 0) slot[0] = global_ns();
        Graph A = graph_from_edges(t, sc, sm, I, J, Cc, nin);
        prof_mark(t, sc, PH_INIT);
        t0 = uread(&slot[0]);
        if (!sc.arena.ok()) status |= ERR_ARENA;
        if (status == ERR_NONE) {
            lb = dual_solver(t, sc, sm, A, o.max_cycle_length_lb, o.num_dual_itr_lb, o.tri_memory_factor,
                             o.num_outer_itr_dual, 1e-4f, &ntri, &oom);
            eafter = A.n;
            const int32_t N0 = A.max_dim();
            if (!o.only_compute_lb) {
                // persistent per-solve arrays sit below every later mark
                int32_t *nm = sc.arena.take<int32_t>((int64_t)N0 + 1);
                int32_t *map = sc.arena.take<int32_t>((int64_t)N0 + 1);
                if (!sc.arena.ok()) status |= ERR_ARENA;
                for (int64_t v = t.rank(); v < N0 && status == ERR_NONE; v += t.size()) nm[v] = (int32_t)v;
                t.sync();
                bool try_mm = !(o.matching_thresh_crossover_ratio > 1.0f);
                for (int64_t iter = 0; status == ERR_NONE && A.n > 0; ++iter) {
                    if (iter > (1 << 22)) {
                        status |= ERR_ITER_LIMIT;
                        break;
                    }
                    if (iter > 0)
                        dual_solver(t, sc, sm, A, o.max_cycle_length_primal, o.num_dual_itr_primal, 1.0f, 1, 1e-4f,
                                    nullptr, &oom);
                    int32_t msize = 0, nr = 0;
                    int werr = 0;
                    if (try_mm) {
                        nr = matching_contraction_map(t, sc, sm, A, o.mean_multiplier_mm, map, &msize);
                        prof_mark(t, sc, PH_MATCHING);
                        ++mrounds;
                        if ((float)nr < (float)A.rows * o.matching_thresh_crossover_ratio) try_mm = false;
                    } else {
                        nr = woc_contraction_map(t, sc, sm, A, map, &msize, &werr, o.woc_pentagons != 0);
                        prof_mark(t, sc, PH_WOC);
                        ++wrounds;
                        status |= werr;
                    }
                    if (!sc.arena.ok()) {
                        status |= ERR_ARENA;
                        break;
                    }
                    if (nr == 0) break;
                    int bad = 0;
                    A = graph_contract(t, sc, sm, A, map, msize - 1, &bad);
                    prof_mark(t, sc, PH_CONTRACT);
                    if (!sc.arena.ok()) {
                        status |= ERR_ARENA;
                        break;
                    }
                    if (bad) {
                        status |= ERR_BAD_CONTRACTION;
                        break;
                    }
                    // map_node_labels (src/rama_cuda.cu:32-52)
                    team_for_batched(
                        t, N0,
                        [&](int64_t v) {
                            const int32_t m = nm[v];
                            return m < msize ? map[m] : m;
                        },
                        [&](int64_t v, int32_t m) { nm[v] = m; });
                    t.sync();
                    prof_mark(t, sc, PH_OTHER);
                    ++rounds;
                    if (o.dump_timeline && io->timeline &&
                        (int64_t)(tl_rounds + 1) * N0 <= io->timeline_cap) {
                        for (int64_t v = t.rank(); v < N0; v += t.size())
                            io->timeline[(int64_t)tl_rounds * N0 + v] = nm[v];
                        ++tl_rounds;
                    }
                    if (o.max_time_sec >= 0) {
                        if (t.rank() == 0) slot[1] = global_ns();
                        t.sync();
                        uint64_t now = uread(&slot[1]);
                        t.sync();
                        if ((int64_t)((now - t0) / 1000000000ull) > (int64_t)o.max_time_sec) break;
                    }
                }
                if (status == ERR_NONE && idmap) {
                    // desanitize_node_labels (include/rama_utils.h:468-493): -1 for ids without edges
                    if (idsize > io->labels_cap)
                        status |= ERR_INVALID_ARG;
                    else {
                        for (int64_t v = t.rank(); v < idsize; v += t.size()) {
                            int32_t cur = idmap[v];
                            bool present = (v == idsize - 1) || cur != idmap[v + 1];
                            io->labels[v] = present ? nm[cur] : -1;
                        }
                        num_labels = idsize;
                    }
                } else if (status == ERR_NONE) {
                    if (N0 > io->labels_cap)
                        status |= ERR_INVALID_ARG;
                    else {
                        for (int64_t v = t.rank(); v < N0; v += t.size()) io->labels[v] = nm[v];
                        num_labels = N0;
                    }
                }
            }
        }
    }
    t.sync();
    if (__ldcg(sc.err)) status |= ERR_ITER_LIMIT;
    if (t.leader()) {
        io->status = status;
        io->lb = lb;
        io->num_labels = num_labels;
        io->rounds = rounds;
        io->matching_rounds = mrounds;
        io->mst_rounds = wrounds;
        io->timeline_rounds = tl_rounds;
        io->dual_oom = oom;
        io->triangles_initial = ntri;
        io->arena_peak = (int64_t)sc.arena.peak;
        io->arena_want = (int64_t)sc.arena.want;
        io->edges_after_dual = eafter;
        io->alg_bytes = sc.alg_bytes;
    }
}

}  // namespace rama
