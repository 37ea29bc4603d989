// step.cuh -- single solver steps on one team, for parity tests and profiling
// (rama_step, include/rama_b200.h).
#pragma once
#include "kernels.cuh"

namespace rama {

template <class Team>
__device__ void copy_graph_out(const Team &t, const Graph &g, rama_step_args *a)
{
    if (g.n <= a->out_cap)
        for (int64_t e = t.rank(); e < g.n; e += t.size()) {
            a->out_row[e] = g.row[e];
            a->out_col[e] = g.col[e];
            a->out_cost[e] = g.cost[e];
        }
    if (t.leader()) {
        a->out_n = g.n;
        a->out_rows = g.rows;
        a->out_cols = g.cols;
        if (g.n > a->out_cap) a->status |= ERR_INVALID_ARG;
    }
}

template <class Team>
__device__ void run_step(const Team &t, char *sm, Scratch sc, rama_step_args *a)
{
    if (t.rank() == 0) *sc.err = 0;
    t.sync();
    Graph A;
    A.row = const_cast<int32_t *>(a->row);
    A.col = const_cast<int32_t *>(a->col);
    A.cost = const_cast<float *>(a->cost);
    A.n = a->n;
    A.rows = a->rows;
    A.cols = a->cols;
    A.cmin = unknown_cost();
    const int op = a->op;
    if (op == RAMA_STEP_INIT) {
        Graph g = graph_from_edges(t, sc, sm, a->i, a->j, a->c, a->m);
        if (sc.arena.ok()) copy_graph_out(t, g, a);
    } else if (op == RAMA_STEP_CONTRACT) {
        int32_t mx = team_max<Team, int32_t>(t, sc, sm, a->map_size, 0, [&](int64_t k) { return a->map[k]; });
        Graph g = graph_contract_raw(t, sc, sm, A, a->map, mx);
        if (sc.arena.ok()) copy_graph_out(t, g, a);
    } else if (op == RAMA_STEP_COARSEN) {
        int32_t mx = team_max<Team, int32_t>(t, sc, sm, a->map_size, 0, [&](int64_t k) { return a->map[k]; });
        int bad = 0;
        Graph g = graph_contract(t, sc, sm, A, a->map, mx, &bad);
        if (sc.arena.ok()) copy_graph_out(t, g, a);
        if (t.leader()) a->out_nr = bad;
    } else if (op == RAMA_STEP_MATCHING) {
        int32_t M = 0;
        int32_t nr = matching_contraction_map(t, sc, sm, A, a->mean_multiplier_mm, a->out_map, &M);
        if (t.leader()) {
            a->out_nr = nr;
            a->out_count = M;
        }
    } else if (op == RAMA_STEP_WOC) {
        int32_t sz = 0;
        int err = 0;
        int32_t nr = woc_contraction_map(t, sc, sm, A, a->out_map, &sz, &err, a->max_cycle_length >= 5);
        if (t.leader()) {
            a->out_nr = nr;
            a->out_count = sz;
            a->status |= err;
        }
    } else if (op == RAMA_STEP_MSF) {
        int32_t mx = team_max<Team, int32_t>(t, sc, sm, a->m, 0, [&](int64_t e) { return max(a->i[e], a->j[e]); });
        bool ok = team_msf(t, sc, sm, a->m, mx + 1, [&](int64_t e) { return a->i[e]; },
                           [&](int64_t e) { return a->j[e]; }, [&](int64_t e) { return a->c[e]; }, a->out_flags);
        if (t.leader() && !ok) a->status |= ERR_ITER_LIMIT;
    } else if (op == RAMA_STEP_CC) {
        const int32_t *off = a->offsets;
        const int32_t nn = a->num_nodes;
        bool ok = team_cc(
            t, sc, nn, a->adj_len,
            [&](int64_t k) {
                int32_t lo = 0, hi = nn - 1;  // row of entry k: last v with off[v] <= k
                while (lo < hi) {
                    int32_t mid = (lo + hi + 1) >> 1;
                    if (off[mid] <= k)
                        lo = mid;
                    else
                        hi = mid - 1;
                }
                return lo;
            },
            [&](int64_t k) { return a->adj[k]; }, a->out_map);
        if (t.leader() && !ok) a->status |= ERR_ITER_LIMIT;
    } else if (op == RAMA_STEP_CYCLES) {
        TriBuf tb;
        conflicted_cycles(t, sc, sm, A, a->max_cycle_length, a->tri_memory_factor, a->tol, tb);
        if (sc.arena.ok()) {
            if (tb.num <= a->out_tri_cap)
                for (int64_t k = t.rank(); k < tb.num; k += t.size()) {
                    a->out_t1[k] = tb.t1[k];
                    a->out_t2[k] = tb.t2[k];
                    a->out_t3[k] = tb.t3[k];
                }
            if (t.leader()) {
                a->out_count = tb.num;
                a->out_raw = tb.count;
                if (tb.num > a->out_tri_cap) a->status |= ERR_INVALID_ARG;
            }
        }
    } else if (op == RAMA_STEP_MP) {
        TriBuf tb;
        tb.budget = a->T;
        tb.count = a->T;
        tb.num = a->T;
        tb.t1 = sc.arena.take<int32_t>(a->T + 1);
        tb.t2 = sc.arena.take<int32_t>(a->T + 1);
        tb.t3 = sc.arena.take<int32_t>(a->T + 1);
        if (sc.arena.ok()) {
            for (int64_t k = t.rank(); k < a->T; k += t.size()) {
                tb.t1[k] = a->t1[k];
                tb.t2[k] = a->t2[k];
                tb.t3[k] = a->t3[k];
            }
            t.sync();
            Mp mp;
            if (mp_build(t, sc, sm, A, tb, mp)) {
                double lb0 = mp_lower_bound(t, sc, mp);
                for (int it = 0; it < a->num_iter; ++it) mp_iteration(t, mp);
                double lb1 = mp_lower_bound(t, sc, mp);
                Graph g;
                g.row = mp.row;
                g.col = mp.col;
                g.cost = mp.cost;
                g.n = mp.E;
                graph_set_dims(t, sc, sm, g);
                copy_graph_out(t, g, a);
                if (t.leader()) {
                    a->out_lb0 = lb0;
                    a->out_lb1 = lb1;
                    a->out_count = mp.T;
                }
            }
        }
    } else if (op == RAMA_STEP_DUAL) {
        int64_t nt = 0;
        int oom = 0;
        double lb = dual_solver(t, sc, sm, A, a->max_cycle_length, a->num_iter, a->tri_memory_factor, a->num_outer,
                                a->tol, &nt, &oom);
        copy_graph_out(t, A, a);
        if (t.leader()) {
            a->out_lb0 = lb;
            a->out_raw = nt;
            a->out_nr = oom;
        }
    } else if (op == RAMA_STEP_CSUM) {
        double s = team_csum(t, sc, a->m, [&](int64_t k) -> float { return a->c[k]; });
        if (t.leader()) a->out_lb0 = s;
    } else if (op == RAMA_STEP_SORT) {
        uint64_t *k1 = sc.arena.take<uint64_t>(a->m + 1), *k2 = sc.arena.take<uint64_t>(a->m + 1);
        int32_t *v1 = sc.arena.take<int32_t>(a->m + 1), *v2 = sc.arena.take<int32_t>(a->m + 1);
        if (sc.arena.ok()) {
            for (int64_t k = t.rank(); k < a->m; k += t.size()) {
                k1[k] = a->keys[k];
                v1[k] = a->i[k];
            }
            t.sync();
            team_sort_pairs(t, sc, sm, k1, v1, k2, v2, a->m, a->key_bits);
            for (int64_t k = t.rank(); k < a->m; k += t.size()) {
                a->out_keys[k] = k1[k];
                a->out_map[k] = v1[k];
            }
        }
    }
    t.sync();
    if (t.leader()) {
        if (!sc.arena.ok()) a->status |= ERR_ARENA;
        if (__ldcg(sc.err)) a->status |= ERR_ITER_LIMIT;
    }
}

}  // namespace rama
