/*
 * rama_oracle.h -- CPU restatement of RAMA's multicut solve (TEST INFRASTRUCTURE).
 *
 * This library is the checker for the CUDA solver in rama_b200/.  It is linked
 * or loaded only by tests/, __graft_entry__.smoke() and the cpu_baseline leg of
 * bench.py; the product path never calls it.
 *
 * It restates, step by step, the algorithm of the reference solver
 * (pawelswoboda/RAMA).  Where the reference is nondeterministic (float
 * atomics, an atomic triangle budget, unordered Thrust/CUB reductions, ties in
 * Boruvka's reduce-by-key) this file fixes ONE canonical order; the CUDA path
 * follows the same order, so the two agree bit for bit.  The canonical choices
 * are listed in rama_oracle.c next to each step, with the reference file:line
 * they restate.
 *
 * Pinning: tests/test_oracle_golden.py checks this oracle against every
 * known-answer test of the reference (its test directory) and against
 * fixtures produced by the reference itself (tests/golden/, made by
 * tests/golden/make_ref_fixtures.py with the reference built from source).
 */
#ifndef RAMA_ORACLE_H
#define RAMA_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Solver options: same fields and meaning as multicut_solver_options
 * (include/multicut_solver_options.h:4-19 in the reference). */
typedef struct {
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
    int32_t woc_pentagons; /* the forest contraction's 5-cycle check, disabled in the reference */
} orc_opts;

/* Directed COO graph (the reference's dCOO, include/dCOO.h:13-70):
 * row < col, sorted by (row, col); rows/cols track rows_/cols_. */
typedef struct {
    int64_t n;
    int32_t *row, *col;
    float *cost;
    int32_t rows, cols;
} orc_graph;

typedef struct {
    int32_t rounds;            /* contraction rounds executed */
    int32_t matching_rounds;
    int32_t mst_rounds;
    int64_t triangles_initial; /* triangles of the initial dual (last cycle length) */
    int32_t status;
    int32_t truncations;       /* cycle searches whose triangle budget overflowed */
} orc_stats;

/* status codes shared with the CUDA library */
enum {
    ORC_OK = 0,
    ORC_ERR_INVALID_ARG = 1,
    ORC_ERR_OOM = 2,
    ORC_ERR_BAD_CONTRACTION = 5
};

/* ---- graph store ---- */
orc_graph *orc_graph_from_edges(int64_t n, const int32_t *i, const int32_t *j, const float *c);
orc_graph *orc_graph_from_sorted(int64_t n, const int32_t *row, const int32_t *col, const float *c);
void orc_graph_free(orc_graph *g);
void orc_graph_info(const orc_graph *g, int64_t *n, int32_t *rows, int32_t *cols);
void orc_graph_copy_out(const orc_graph *g, int32_t *row, int32_t *col, float *cost);
orc_graph *orc_contract(const orc_graph *A, const int32_t *map, int64_t map_size);
int orc_has_bad_contractions(const orc_graph *A);
void orc_remove_diagonal(orc_graph *A);

/* ---- primitives pinned by the reference's unit tests ---- */
void orc_compute_offsets(const int32_t *sorted_ids, int64_t n, int32_t max_value, int32_t *offsets /* max_value+2 */);
void orc_compress_label_sequence(const int32_t *data, int64_t n, int32_t max_label, int32_t *out);
void orc_cc(int32_t num_nodes, const int32_t *offsets, const int32_t *cols, int32_t *labels);
double orc_csum_f32(const float *x, int64_t n);
float orc_rsum_f32(const float *x, int64_t n);

/* ---- contraction-set selection ---- */
/* vertex matching + label compression (rama_cuda.cu:54-62); map has
 * (max col of A)+1 entries. */
int orc_matching(const orc_graph *A, float mean_multiplier_mm, int32_t *map_out, int64_t *map_size, int32_t *nr_matched);
/* maximum spanning forest (Boruvka) over m edges; writes sorted unique edge ids */
int orc_msf(int64_t m, const int32_t *i, const int32_t *j, const float *w, int32_t *ids_out, int64_t *k_out);
/* conflict-free forest contraction (edge_contractions_woc{,_thrust}.cu); map has
 * max(rows,cols) entries; nr = directed forest entries left (0 = stop). */
int orc_woc(const orc_graph *A, int32_t *map_out, int64_t *map_size, int32_t *nr_out);
/* orc_woc with the 5-cycle forest check (check_pentagons_cuda) when pentagons != 0 */
int orc_woc_ex(const orc_graph *A, int32_t *map_out, int64_t *map_size, int32_t *nr_out, int pentagons);

/* ---- conflicted cycles ---- */
/* writes the first min(count, budget) emitted triangles (3 ints each) in
 * canonical order; *raw_count = the reference's triangle counter. */
int orc_conflicted_cycles(const orc_graph *A, int32_t max_cycle_length, float tri_memory_factor, float tol_ratio,
                          int32_t *tri_out, int64_t tri_cap, int64_t *num_out, int64_t *raw_count);

/* FP64 oracle of the dual solver: the same triangle selection, every cost,
 * message and bound in double (for reporting the error of the FP32 messages) */
int orc_dual_lb_f64(int64_t n, const int32_t *i, const int32_t *j, const float *c, int32_t max_len, int32_t num_iter,
                    float tri_factor, int32_t num_outer, float tol, double *lb);

/* ---- message passing ---- */
typedef struct orc_mp orc_mp;
orc_mp *orc_mp_create(const orc_graph *A, const int32_t *t1, const int32_t *t2, const int32_t *t3, int64_t T);
void orc_mp_free(orc_mp *mp);
double orc_mp_lower_bound(orc_mp *mp);
void orc_mp_send_messages_to_triplets(orc_mp *mp);
void orc_mp_send_messages_to_edges(orc_mp *mp);
void orc_mp_iteration(orc_mp *mp);
void orc_mp_info(const orc_mp *mp, int64_t *num_edges, int64_t *num_triangles);
void orc_mp_copy_edges(const orc_mp *mp, int32_t *row, int32_t *col, float *cost, int32_t *counter);
void orc_mp_copy_triangles(const orc_mp *mp, int32_t *t1, int32_t *t2, int32_t *t3, float *c12, float *c13, float *c23,
                           int32_t *e12, int32_t *e13, int32_t *e23);

/* ---- dual solver: replaces *A by the reparametrised graph, returns the LB ---- */
double orc_dual_solver(orc_graph **A, int32_t max_cycle_length, int32_t num_iter, float tri_memory_factor,
                       int32_t num_outer_itr, float tol_ratio, int64_t *num_triangles_last);

/* ---- full solve (rama_cuda.cu:64-193) ---- */
void orc_opts_init(orc_opts *o, const char *mode /* NULL, "PD", "P", "PD+", "D" */);
int orc_solve(int64_t n, const int32_t *i, const int32_t *j, const float *c, const orc_opts *opts,
              int32_t *labels_out, int64_t labels_cap, int64_t *num_labels, double *lb_out, orc_stats *stats);
double orc_objective(int64_t n, const int32_t *i, const int32_t *j, const float *c, const int32_t *labels);

/* ---- sanitize (rama_utils.h:429-493) ---- */
int orc_sanitize(int64_t n, int32_t *i, int32_t *j, float *c, int64_t *n_out, int32_t *ids_mapping_out,
                 int64_t ids_cap, int64_t *ids_size);

/* ---- project-written CPU baseline: greedy additive edge contraction ---- */
int orc_gaec(int64_t n, const int32_t *i, const int32_t *j, const float *c, int32_t num_nodes, int32_t *labels_out);

void orc_free(void *p);

#ifdef __cplusplus
}
#endif
#endif
