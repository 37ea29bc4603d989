/*
 * rama_oracle.c -- CPU restatement of the RAMA multicut solve.
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker for the CUDA solver.  Only
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load it.
 *
 * Every function cites the reference file:line it restates (paths inside the
 * reference project).  The reference leaves several orders to the hardware;
 * this restatement fixes them as follows (the CUDA path uses the same ones):
 *
 *  C1  sorts are stable (LSD radix); the reference's zip-key sorts are merge
 *      sorts, also stable.
 *  C2  sums that the reference does with unordered float reductions (matching
 *      threshold, forest threshold, lower bound, objective) use CSUM: a
 *      compensated FP64 sum over chunks of 4096 elements, 32 lane-strided
 *      partial sums per chunk (TwoSum compensation), a pairwise tree over the
 *      32 lanes, then the same lane/tree scheme over the chunk partials.
 *  C3  sums of parallel edges after contraction and of messages arriving at
 *      an edge use RSUM: FP64, 32 lane-strided partial sums in element order,
 *      pairwise tree over lanes, rounded once to float.
 *  C4  the triangle budget: expansions (a rep edge; a rep edge and a
 *      neighbour; a rep edge and two neighbours) are taken in canonical order
 *      in chunks of 2^24, each emitting its triangles in a fixed order.  A
 *      chunk whose emissions exceed the room left keeps them round-robin:
 *      the first K emissions of every expansion, K as large as fits, and one
 *      more for the first expansions (in order) that have one, until the room
 *      is full.  The reference keeps whichever emissions its atomics admit;
 *      with all its threads resident that is close to round-robin over rep
 *      edges, which keeps some triangles of every conflicted edge.
 *  C5  Boruvka picks per super-vertex the lexicographic minimum of
 *      (-weight, target super-vertex, edge id); the reference's reduce-by-key
 *      only fixes (-weight, target).
 *  C6  divisions are IEEE (the reference builds with -use_fast_math).
 */
#include "rama_oracle.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

/* ------------------------------------------------------------------------ */
/* memory helpers                                                           */
/* ------------------------------------------------------------------------ */
static void *xmalloc(size_t n)
{
    void *p = malloc(n ? n : 1);
    if (!p) {
        fprintf(stderr, "rama oracle: out of memory (%zu bytes)\n", n);
        abort();
    }
    return p;
}
#define NEW(T, n) ((T *)xmalloc(sizeof(T) * (size_t)(n)))

static void *xcalloc(size_t n, size_t s)
{
    void *p = calloc(n ? n : 1, s ? s : 1);
    if (!p) {
        fprintf(stderr, "rama oracle: out of memory\n");
        abort();
    }
    return p;
}

void orc_free(void *p) { free(p); }

static inline int32_t imin(int32_t a, int32_t b) { return a < b ? a : b; }
static inline int32_t imax(int32_t a, int32_t b) { return a > b ? a : b; }

/* ------------------------------------------------------------------------ */
/* C1: stable order of 64-bit keys (LSD radix, 16-bit digits)                */
/* ------------------------------------------------------------------------ */
static int64_t *stable_order_u64(const uint64_t *keys, int64_t n)
{
    int64_t *perm = NEW(int64_t, n);
    int64_t *tmp = NEW(int64_t, n);
    uint64_t any = 0;
    for (int64_t k = 0; k < n; ++k) {
        perm[k] = k;
        any |= keys[k];
    }
    int bits = 0;
    while (bits < 64 && (any >> bits) != 0) bits++;
    int64_t *cnt = NEW(int64_t, 65537);
    for (int shift = 0; shift < bits; shift += 16) {
        memset(cnt, 0, sizeof(int64_t) * 65537);
        for (int64_t k = 0; k < n; ++k) cnt[((keys[perm[k]] >> shift) & 0xFFFF) + 1]++;
        for (int d = 0; d < 65536; ++d) cnt[d + 1] += cnt[d];
        for (int64_t k = 0; k < n; ++k) {
            int64_t p = perm[k];
            tmp[cnt[(keys[p] >> shift) & 0xFFFF]++] = p;
        }
        int64_t *s = perm;
        perm = tmp;
        tmp = s;
    }
    free(cnt);
    free(tmp);
    return perm;
}

static inline uint64_t pack2(int32_t a, int32_t b) { return ((uint64_t)(uint32_t)a << 32) | (uint32_t)b; }

/* ------------------------------------------------------------------------ */
/* C2: CSUM, compensated FP64 (TwoSum) with a fixed reduction tree           */
/* ------------------------------------------------------------------------ */
typedef struct {
    double s, c;
} csum_t;

static inline csum_t cs_merge(csum_t a, csum_t b)
{
    double s = a.s + b.s;
    double bb = s - a.s;
    double e = (a.s - (s - bb)) + (b.s - bb);
    csum_t r;
    r.s = s;
    r.c = (a.c + b.c) + e;
    return r;
}

#define CS_CHUNK 4096
typedef struct {
    csum_t lane[32];
    csum_t *part;
    int64_t nparts, cap;
    int64_t idx;
} csum_acc;

static void cacc_init(csum_acc *a)
{
    memset(a->lane, 0, sizeof(a->lane));
    a->cap = 64;
    a->part = NEW(csum_t, a->cap);
    a->nparts = 0;
    a->idx = 0;
}

static csum_t cs_tree32(csum_t *lane)
{
    for (int off = 1; off < 32; off *= 2)
        for (int l = 0; l < 32; l += 2 * off) lane[l] = cs_merge(lane[l], lane[l + off]);
    return lane[0];
}

static void cacc_flush(csum_acc *a)
{
    csum_t p = cs_tree32(a->lane);
    if (a->nparts == a->cap) {
        a->cap *= 2;
        csum_t *np = NEW(csum_t, a->cap);
        memcpy(np, a->part, sizeof(csum_t) * (size_t)a->nparts);
        free(a->part);
        a->part = np;
    }
    a->part[a->nparts++] = p;
    memset(a->lane, 0, sizeof(a->lane));
}

static inline void cacc_push(csum_acc *a, double x)
{
    int l = (int)((a->idx % CS_CHUNK) & 31);
    csum_t b = {x, 0.0};
    a->lane[l] = cs_merge(a->lane[l], b);
    a->idx++;
    if (a->idx % CS_CHUNK == 0) cacc_flush(a);
}

static double cacc_finish(csum_acc *a)
{
    if (a->idx % CS_CHUNK != 0) cacc_flush(a);
    csum_t lane[32];
    memset(lane, 0, sizeof(lane));
    for (int64_t k = 0; k < a->nparts; ++k) lane[k & 31] = cs_merge(lane[k & 31], a->part[k]);
    csum_t r = cs_tree32(lane);
    free(a->part);
    a->part = NULL;
    return r.s + r.c;
}

double orc_csum_f32(const float *x, int64_t n)
{
    csum_acc a;
    cacc_init(&a);
    for (int64_t k = 0; k < n; ++k) cacc_push(&a, (double)x[k]);
    return cacc_finish(&a);
}

/* C3: RSUM, plain FP64 lane-strided sums + pairwise tree, rounded to float.
 * Up to 4096 values: value k goes to lane k mod 32 (each lane starts at +0.0
 * and adds its values in order), then a pairwise tree over the 32 lanes.
 * More than 4096 values: each chunk of 4096 consecutive values is summed that
 * way (kept in double), and the chunk sums are summed the same way (chunk c
 * to lane c mod 32), so that many warps can share one long sum on the GPU. */
typedef struct {
    double lane[32];
    double chunk_lane[32];
    int64_t idx;
    int64_t chunks;
} rsum_acc;
static inline double racc_tree(double *lane)
{
    for (int off = 1; off < 32; off *= 2)
        for (int l = 0; l < 32; l += 2 * off) lane[l] = lane[l] + lane[l + off];
    return lane[0];
}
static inline void racc_init(rsum_acc *a)
{
    memset(a->lane, 0, sizeof(a->lane));
    memset(a->chunk_lane, 0, sizeof(a->chunk_lane));
    a->idx = 0;
    a->chunks = 0;
}
static inline void racc_push(rsum_acc *a, float x)
{
    a->lane[a->idx & 31] += (double)x;
    a->idx++;
    if ((a->idx & 4095) == 0) {
        a->chunk_lane[a->chunks & 31] += racc_tree(a->lane);
        a->chunks++;
        memset(a->lane, 0, sizeof(a->lane));
    }
}
static inline float racc_finish(rsum_acc *a)
{
    if (a->idx <= 4096) {
        if (a->chunks == 1) return (float)a->chunk_lane[0]; /* exactly 4096 values */
        return (float)racc_tree(a->lane);
    }
    if ((a->idx & 4095) != 0) {
        a->chunk_lane[a->chunks & 31] += racc_tree(a->lane);
        a->chunks++;
    }
    return (float)racc_tree(a->chunk_lane);
}

float orc_rsum_f32(const float *x, int64_t n)
{
    rsum_acc a;
    racc_init(&a);
    for (int64_t k = 0; k < n; ++k) racc_push(&a, x[k]);
    return racc_finish(&a);
}

/* ------------------------------------------------------------------------ */
/* graph store (include/dCOO.h:13-121, src/dCOO.cu:28-152)                   */
/* ------------------------------------------------------------------------ */
static orc_graph *graph_alloc(int64_t n)
{
    orc_graph *g = NEW(orc_graph, 1);
    g->n = n;
    g->row = NEW(int32_t, n);
    g->col = NEW(int32_t, n);
    g->cost = NEW(float, n);
    g->rows = 0;
    g->cols = 0;
    return g;
}

void orc_graph_free(orc_graph *g)
{
    if (!g) return;
    free(g->row);
    free(g->col);
    free(g->cost);
    free(g);
}

static void graph_set_dims(orc_graph *g)
{
    /* dCOO::init (src/dCOO.cu:47-51): cols_ = max col + 1, rows_ = last row + 1 */
    if (g->n == 0) {
        g->rows = g->cols = 0;
        return;
    }
    int32_t mc = 0;
    for (int64_t e = 0; e < g->n; ++e) mc = imax(mc, g->col[e]);
    g->cols = mc + 1;
    g->rows = g->row[g->n - 1] + 1;
}

/* dCOO ctor with is_sorted=false: sort_edge_nodes + coo_sorting
 * (src/dCOO.cu:38-45, include/rama_utils.h:231-294) */
orc_graph *orc_graph_from_edges(int64_t n, const int32_t *i, const int32_t *j, const float *c)
{
    uint64_t *keys = NEW(uint64_t, n);
    for (int64_t e = 0; e < n; ++e) keys[e] = pack2(imin(i[e], j[e]), imax(i[e], j[e]));
    int64_t *perm = stable_order_u64(keys, n);
    orc_graph *g = graph_alloc(n);
    for (int64_t k = 0; k < n; ++k) {
        int64_t p = perm[k];
        g->row[k] = imin(i[p], j[p]);
        g->col[k] = imax(i[p], j[p]);
        g->cost[k] = c[p];
    }
    free(perm);
    free(keys);
    graph_set_dims(g);
    return g;
}

orc_graph *orc_graph_from_sorted(int64_t n, const int32_t *row, const int32_t *col, const float *c)
{
    orc_graph *g = graph_alloc(n);
    memcpy(g->row, row, sizeof(int32_t) * (size_t)n);
    memcpy(g->col, col, sizeof(int32_t) * (size_t)n);
    memcpy(g->cost, c, sizeof(float) * (size_t)n);
    graph_set_dims(g);
    return g;
}

void orc_graph_info(const orc_graph *g, int64_t *n, int32_t *rows, int32_t *cols)
{
    if (n) *n = g->n;
    if (rows) *rows = g->rows;
    if (cols) *cols = g->cols;
}

void orc_graph_copy_out(const orc_graph *g, int32_t *row, int32_t *col, float *cost)
{
    if (row) memcpy(row, g->row, sizeof(int32_t) * (size_t)g->n);
    if (col) memcpy(col, g->col, sizeof(int32_t) * (size_t)g->n);
    if (cost) memcpy(cost, g->cost, sizeof(float) * (size_t)g->n);
}

static int32_t graph_max_dim(const orc_graph *g) { return imax(g->rows, g->cols); }

/* dCOO::contract_cuda (src/dCOO.cu:14-26, 57-95): relabel, sort, sum parallel
 * edges (RSUM, C3).  Self loops (the "diagonal") are kept. */
orc_graph *orc_contract(const orc_graph *A, const int32_t *map, int64_t map_size)
{
    (void)map_size;
    int64_t n = A->n;
    uint64_t *keys = NEW(uint64_t, n);
    for (int64_t e = 0; e < n; ++e) {
        int32_t a = map[A->row[e]], b = map[A->col[e]];
        keys[e] = pack2(imin(a, b), imax(a, b));
    }
    int64_t *perm = stable_order_u64(keys, n);
    int64_t runs = 0;
    for (int64_t k = 0; k < n; ++k)
        if (k == 0 || keys[perm[k]] != keys[perm[k - 1]]) runs++;
    orc_graph *g = graph_alloc(runs);
    int64_t out = -1;
    rsum_acc acc;
    racc_init(&acc);
    for (int64_t k = 0; k < n; ++k) {
        int64_t p = perm[k];
        if (k == 0 || keys[p] != keys[perm[k - 1]]) {
            if (out >= 0) g->cost[out] = racc_finish(&acc);
            out++;
            racc_init(&acc);
            g->row[out] = (int32_t)(keys[p] >> 32);
            g->col[out] = (int32_t)(keys[p] & 0xFFFFFFFFu);
        }
        racc_push(&acc, A->cost[p]);
    }
    if (out >= 0) g->cost[out] = racc_finish(&acc);
    free(perm);
    free(keys);
    graph_set_dims(g); /* out_rows.back()+1 and max(out_cols)+1, diagonal included */
    return g;
}

/* has_bad_contractions (src/rama_cuda.cu:18-30) + dCOO::diagonal (src/dCOO.cu:118-142) */
int orc_has_bad_contractions(const orc_graph *A)
{
    for (int64_t e = 0; e < A->n; ++e)
        if (A->row[e] == A->col[e] && A->cost[e] < 0.0f) return 1;
    return 0;
}

/* dCOO::remove_diagonal (src/dCOO.cu:97-116): stable; dims are kept */
void orc_remove_diagonal(orc_graph *A)
{
    int64_t w = 0;
    for (int64_t e = 0; e < A->n; ++e) {
        if (A->row[e] == A->col[e]) continue;
        A->row[w] = A->row[e];
        A->col[w] = A->col[e];
        A->cost[w] = A->cost[e];
        w++;
    }
    A->n = w;
}

/* compute_offsets (include/rama_utils.h:403-413) */
void orc_compute_offsets(const int32_t *ids, int64_t n, int32_t max_value, int32_t *offsets)
{
    memset(offsets, 0, sizeof(int32_t) * (size_t)(max_value + 2));
    for (int64_t k = 0; k < n; ++k) offsets[ids[k] + 1]++;
    for (int32_t v = 0; v <= max_value; ++v) offsets[v + 1] += offsets[v];
}

/* compress_label_sequence (include/rama_utils.h:160-177) */
void orc_compress_label_sequence(const int32_t *data, int64_t n, int32_t max_label, int32_t *out)
{
    int32_t *mask = (int32_t *)xcalloc((size_t)max_label + 1, sizeof(int32_t));
    for (int64_t k = 0; k < n; ++k) mask[data[k]] = 1;
    int32_t run = 0;
    for (int32_t l = 0; l <= max_label; ++l) {
        int32_t m = mask[l];
        mask[l] = run;
        run += m;
    }
    for (int64_t k = 0; k < n; ++k) out[k] = mask[data[k]];
    free(mask);
}

/* symmetric CSR of a set of directed edges (export_undirected / to_undirected,
 * src/dCOO.cu:164-172, include/rama_utils.h:107-131), rows sorted by column. */
typedef struct {
    int32_t n;       /* number of rows */
    int32_t *off;    /* n+1 */
    int32_t *adj;    /* 2m */
    float *w;        /* 2m */
    int64_t m2;
} csr_t;

static void csr_free(csr_t *c)
{
    free(c->off);
    free(c->adj);
    free(c->w);
}

/* rows i<j of a (row,col)-sorted list: row v lists first the neighbours u<v in
 * increasing u, then the neighbours w>v in increasing w -- the (row,col) sort
 * of the doubled list. */
static void build_symmetric_csr(int32_t nrows, int64_t m, const int32_t *r, const int32_t *c, const float *w, csr_t *out)
{
    out->n = nrows;
    out->m2 = 2 * m;
    out->off = (int32_t *)xcalloc((size_t)nrows + 1, sizeof(int32_t));
    out->adj = NEW(int32_t, 2 * m);
    out->w = NEW(float, 2 * m);
    for (int64_t e = 0; e < m; ++e) {
        out->off[r[e] + 1]++;
        out->off[c[e] + 1]++;
    }
    for (int32_t v = 0; v < nrows; ++v) out->off[v + 1] += out->off[v];
    int32_t *fill = NEW(int32_t, nrows);
    memcpy(fill, out->off, sizeof(int32_t) * (size_t)nrows);
    /* reverse entries (col -> row): scanning the sorted list gives increasing row */
    for (int64_t e = 0; e < m; ++e) {
        int32_t v = c[e];
        out->adj[fill[v]] = r[e];
        out->w[fill[v]] = w[e];
        fill[v]++;
    }
    for (int64_t e = 0; e < m; ++e) {
        int32_t v = r[e];
        out->adj[fill[v]] = c[e];
        out->w[fill[v]] = w[e];
        fill[v]++;
    }
    free(fill);
    /* rows are sorted as long as the input is (row,col)-sorted without
     * duplicates; sort defensively otherwise (stable insertion sort) */
    for (int32_t v = 0; v < nrows; ++v) {
        for (int32_t k = out->off[v] + 1; k < out->off[v + 1]; ++k) {
            int32_t a = out->adj[k];
            float aw = out->w[k];
            int32_t q = k - 1;
            while (q >= out->off[v] && out->adj[q] > a) {
                out->adj[q + 1] = out->adj[q];
                out->w[q + 1] = out->w[q];
                q--;
            }
            out->adj[q + 1] = a;
            out->w[q + 1] = aw;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* connected components: labels = minimum vertex id (ECL-CC semantics,       */
/* external/ECL-CC/ECL-CC_11.cu:58-254)                                      */
/* ------------------------------------------------------------------------ */
static int32_t uf_find(int32_t *p, int32_t x)
{
    int32_t r = x;
    while (p[r] != r) r = p[r];
    while (p[x] != r) {
        int32_t nx = p[x];
        p[x] = r;
        x = nx;
    }
    return r;
}

void orc_cc(int32_t num_nodes, const int32_t *offsets, const int32_t *cols, int32_t *labels)
{
    for (int32_t v = 0; v < num_nodes; ++v) labels[v] = v;
    for (int32_t v = 0; v < num_nodes; ++v) {
        for (int32_t k = offsets[v]; k < offsets[v + 1]; ++k) {
            int32_t a = uf_find(labels, v), b = uf_find(labels, cols[k]);
            if (a == b) continue;
            if (a < b)
                labels[b] = a;
            else
                labels[a] = b;
        }
    }
    for (int32_t v = 0; v < num_nodes; ++v) labels[v] = uf_find(labels, v);
}

/* ------------------------------------------------------------------------ */
/* vertex-based matching (src/maximum_matching_vertex_based.cu:10-137)       */
/* ------------------------------------------------------------------------ */
int orc_matching(const orc_graph *A, float mm, int32_t *map_out, int64_t *map_size, int32_t *nr_matched)
{
    int32_t M = 0;
    for (int64_t e = 0; e < A->n; ++e) M = imax(M, A->col[e] + 1);
    csr_t G;
    build_symmetric_csr(M, A->n, A->row, A->col, A->cost, &G);

    /* determine_matching_threshold (:76-86): mean over the doubled list of the
     * non-negative costs (C2); the doubled sum is 2x the directed one. */
    csum_acc acc;
    cacc_init(&acc);
    int64_t cnt = 0;
    for (int64_t e = 0; e < A->n; ++e) {
        float c = A->cost[e];
        cacc_push(&acc, c >= 0.0f ? (double)c : 0.0);
        cnt += (c >= 0.0f);
    }
    double S = cacc_finish(&acc);
    int32_t *node_mapping = NEW(int32_t, M);
    for (int32_t v = 0; v < M; ++v) node_mapping[v] = v;
    int32_t prev = 0;
    if (cnt > 0) {
        float sum_f = (float)(2.0 * S);
        float thresh = (mm * sum_f) / (float)(2 * cnt);
        int32_t *best = NEW(int32_t, M);
        int32_t *matched = (int32_t *)xcalloc((size_t)M, sizeof(int32_t));
        for (int32_t v = 0; v < M; ++v) best[v] = -1;
        for (int t = 0; t < 10; ++t) {
            int still = 0;
            /* pick_best_neighbour / get_best_neighbour (:10-47) */
            for (int32_t v = 0; v < M; ++v) {
                if (matched[v]) continue;
                float mx = thresh;
                int32_t id = -1;
                for (int32_t k = G.off[v]; k < G.off[v + 1]; ++k) {
                    float cv = G.w[k];
                    int32_t nb = G.adj[k];
                    if (cv <= mx || matched[nb] || nb == v) continue;
                    mx = cv;
                    id = nb;
                }
                best[v] = id;
            }
            /* match_neighbours (:49-74) */
            for (int32_t v = 0; v < M; ++v) {
                if (matched[v]) continue;
                int32_t b = best[v];
                if (b == -1 || matched[b]) continue;
                if (best[b] == v) {
                    node_mapping[imax(b, v)] = imin(b, v);
                    matched[v] = 1;
                    matched[b] = 1;
                    still = 1;
                }
            }
            int32_t cur = 0;
            for (int32_t v = 0; v < M; ++v) cur += matched[v];
            float rel = (float)(cur - prev) / ((float)prev + 1.0f);
            prev = cur;
            if (!still || (double)rel < 0.1) break;
        }
        free(best);
        free(matched);
    }
    /* contraction_mapping_by_maximum_matching (src/rama_cuda.cu:54-62) */
    orc_compress_label_sequence(node_mapping, M, M - 1, map_out);
    *map_size = M;
    *nr_matched = prev;
    free(node_mapping);
    csr_free(&G);
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* maximum spanning forest, Boruvka (external/cudaMST/gpuMST/gpuMST.cu:      */
/* 106-147, 191-339, 364-388) with the C5 tie-break                          */
/* ------------------------------------------------------------------------ */
int orc_msf(int64_t m, const int32_t *i, const int32_t *j, const float *w, int32_t *ids_out, int64_t *k_out)
{
    *k_out = 0;
    if (m == 0) return ORC_OK;
    int64_t ne = 2 * m;
    int32_t *u = NEW(int32_t, ne), *v = NEW(int32_t, ne), *id = NEW(int32_t, ne);
    float *nw = NEW(float, ne);
    int32_t nv = 0;
    for (int64_t e = 0; e < m; ++e) {
        u[e] = i[e];
        v[e] = j[e];
        u[e + m] = j[e];
        v[e + m] = i[e];
        nw[e] = nw[e + m] = -w[e];
        id[e] = id[e + m] = (int32_t)e;
        nv = imax(nv, imax(i[e], j[e]) + 1);
    }
    int32_t *mst = NEW(int32_t, m + 1);
    int64_t nm = 0;
    int32_t *bv = NEW(int32_t, nv), *bid = NEW(int32_t, nv), *succ = NEW(int32_t, nv), *succ2 = NEW(int32_t, nv);
    float *bw = NEW(float, nv);
    int32_t *newid = NEW(int32_t, nv);
    for (int guard = 0; guard < 64 && ne > 0; ++guard) {
        if (ne == 1) {
            mst[nm++] = id[0];
            break;
        }
        for (int32_t x = 0; x < nv; ++x) bv[x] = -1;
        for (int64_t e = 0; e < ne; ++e) {
            int32_t x = u[e];
            int better = 0;
            if (bv[x] < 0)
                better = 1;
            else if (nw[e] < bw[x])
                better = 1;
            else if (nw[e] == bw[x]) {
                if (v[e] < bv[x])
                    better = 1;
                else if (v[e] == bv[x] && id[e] < bid[x])
                    better = 1;
            }
            if (better) {
                bw[x] = nw[e];
                bv[x] = v[e];
                bid[x] = id[e];
            }
        }
        for (int32_t x = 0; x < nv; ++x) succ[x] = bv[x] < 0 ? x : bv[x];
        /* remove_circles (:106-121) */
        for (int32_t x = 0; x < nv; ++x) {
            int32_t s = succ[x], ss = succ[s];
            succ2[x] = (s > x && ss == x) ? x : s;
        }
        for (int32_t x = 0; x < nv; ++x)
            if (succ2[x] != x) mst[nm++] = bid[x];
        /* merge_vertices (:123-147): each vertex points to its root */
        for (int32_t x = 0; x < nv; ++x) {
            int32_t r = succ2[x];
            int lim = 0;
            while (succ2[r] != r && lim++ < (1 << 30)) r = succ2[r];
            succ[x] = r;
        }
        /* new id = rank of the root among roots (sort + mark_segments + scan) */
        int32_t nroots = 0;
        for (int32_t x = 0; x < nv; ++x)
            if (succ[x] == x) newid[x] = nroots++;
        for (int32_t x = 0; x < nv; ++x) succ2[x] = newid[succ[x]];
        int64_t w2 = 0;
        for (int64_t e = 0; e < ne; ++e) {
            int32_t a = succ2[u[e]], b = succ2[v[e]];
            if (a == b) continue;
            u[w2] = a;
            v[w2] = b;
            nw[w2] = nw[e];
            id[w2] = id[e];
            w2++;
        }
        ne = w2;
        nv = nroots;
    }
    /* sort + unique of the chosen ids (:375-377) */
    int32_t *mark = (int32_t *)xcalloc((size_t)m, sizeof(int32_t));
    for (int64_t k = 0; k < nm; ++k) mark[mst[k]] = 1;
    int64_t k = 0;
    for (int64_t e = 0; e < m; ++e)
        if (mark[e]) ids_out[k++] = (int32_t)e;
    *k_out = k;
    free(mark);
    free(u);
    free(v);
    free(id);
    free(nw);
    free(mst);
    free(bv);
    free(bid);
    free(bw);
    free(succ);
    free(succ2);
    free(newid);
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* conflict-free forest contraction                                         */
/* (src/edge_contractions_woc.cu:10-79, 141-193, 257-423 and                 */
/*  src/edge_contractions_woc_thrust.cu:95-599)                              */
/* ------------------------------------------------------------------------ */
typedef struct {
    int32_t nn;            /* num_nodes = A.max_dim() */
    int64_t m2;            /* directed forest entries */
    int32_t *r, *c;        /* sorted (r,c) */
    float *w;
    int32_t *off;          /* nn+1 */
    int64_t R;
    int32_t *rr, *rc;      /* repulsive edges */
    int32_t *lab;          /* cc labels */
} forest_t;

static void forest_offsets(forest_t *F)
{
    orc_compute_offsets(F->r, F->m2, F->nn - 1, F->off);
}

/* remove the undirected edges {a,b} listed (either direction) */
static void forest_remove_pairs(forest_t *F, const uint64_t *pairs, int64_t np)
{
    if (np == 0) return;
    uint64_t *keys = NEW(uint64_t, 2 * np);
    for (int64_t k = 0; k < np; ++k) {
        int32_t a = (int32_t)(pairs[k] >> 32), b = (int32_t)(pairs[k] & 0xFFFFFFFFu);
        keys[2 * k] = pack2(a, b);
        keys[2 * k + 1] = pack2(b, a);
    }
    int64_t *ord = stable_order_u64(keys, 2 * np);
    int64_t w2 = 0, q = 0;
    for (int64_t e = 0; e < F->m2; ++e) {
        uint64_t key = pack2(F->r[e], F->c[e]);
        while (q < 2 * np && keys[ord[q]] < key) q++;
        if (q < 2 * np && keys[ord[q]] == key) continue;
        F->r[w2] = F->r[e];
        F->c[w2] = F->c[e];
        F->w[w2] = F->w[e];
        w2++;
    }
    F->m2 = w2;
    free(ord);
    free(keys);
    forest_offsets(F);
}

/* remove_mst_by_mask (src/edge_contractions_woc.cu:287-339) */
static int forest_remove_mask(forest_t *F, const uint8_t *invalid)
{
    int64_t np = 0;
    for (int64_t e = 0; e < F->m2; ++e) np += invalid[e] != 0;
    if (np == 0) return 0;
    uint64_t *pairs = NEW(uint64_t, np);
    np = 0;
    for (int64_t e = 0; e < F->m2; ++e)
        if (invalid[e]) pairs[np++] = pack2(F->r[e], F->c[e]);
    forest_remove_pairs(F, pairs, np);
    free(pairs);
    return 1;
}

/* filter_by_cc (src/edge_contractions_woc.cu:257-276) */
static int64_t forest_filter_by_cc(forest_t *F)
{
    orc_cc(F->nn, F->off, F->c, F->lab);
    int64_t w2 = 0;
    for (int64_t k = 0; k < F->R; ++k) {
        if (F->lab[F->rr[k]] != F->lab[F->rc[k]]) continue;
        F->rr[w2] = F->rr[k];
        F->rc[w2] = F->rc[k];
        w2++;
    }
    F->R = w2;
    return w2;
}

/* first common neighbour; returns the positions in both rows (compute_lowest_common_neighbour,
 * include/rama_utils.h:62-84) */
static int32_t first_common(const int32_t *off, const int32_t *adj, int32_t a, int32_t b, int32_t *pa, int32_t *pb)
{
    int32_t x = off[a], y = off[b];
    while (x < off[a + 1] && y < off[b + 1]) {
        int32_t na = adj[x], nb = adj[y];
        if (na == nb) {
            *pa = x;
            *pb = y;
            return na;
        }
        if (na < nb)
            x++;
        else
            y++;
    }
    return -1;
}

/* check_triangles_cuda (src/edge_contractions_woc.cu:10-37) */
static int forest_check_triangles(forest_t *F)
{
    if (F->R == 0) return 0;
    uint8_t *inv = (uint8_t *)xcalloc((size_t)F->m2, 1);
    for (int64_t k = 0; k < F->R; ++k) {
        int32_t p1, p2;
        int32_t mid = first_common(F->off, F->c, F->rr[k], F->rc[k], &p1, &p2);
        if (mid < 0) continue;
        if (F->w[p1] < F->w[p2])
            inv[p1] = 1;
        else
            inv[p2] = 1;
    }
    int any = forest_remove_mask(F, inv);
    free(inv);
    return any;
}

/* check_quadrangles_cuda (src/edge_contractions_woc.cu:39-79) */
static int forest_check_quadrangles(forest_t *F)
{
    if (F->R == 0) return 0;
    uint8_t *inv = (uint8_t *)xcalloc((size_t)F->m2, 1);
    for (int64_t k = 0; k < F->R; ++k) {
        int32_t v1 = F->rr[k], v2 = F->rc[k];
        for (int32_t e1 = F->off[v1]; e1 < F->off[v1 + 1]; ++e1) {
            int32_t n1 = F->c[e1];
            int32_t p1, p2;
            int32_t mid = first_common(F->off, F->c, n1, v2, &p1, &p2);
            if (mid < 0) continue;
            float a = F->w[e1], b = F->w[p1], c = F->w[p2];
            if (a < b && a < c)
                inv[e1] = 1;
            else if (b < c)
                inv[p1] = 1;
            else
                inv[p2] = 1;
        }
    }
    int any = forest_remove_mask(F, inv);
    free(inv);
    return any;
}

/* check_pentagons_cuda (src/edge_contractions_woc.cu:81-139, called from the
 * commented-out line :414): for a repulsive edge (v1, v2), forest neighbours
 * n1 of v1 and n2 of v2 (n1 != n2) and the first common neighbour mid of n1
 * and n2, cut the weakest of the four forest edges of v1-n1-mid-n2-v2 in the
 * reference's comparison order. */
static int forest_check_pentagons(forest_t *F)
{
    if (F->R == 0) return 0;
    uint8_t *inv = (uint8_t *)xcalloc((size_t)F->m2, 1);
    for (int64_t k = 0; k < F->R; ++k) {
        int32_t v1 = F->rr[k], v2 = F->rc[k];
        for (int32_t e2 = F->off[v2]; e2 < F->off[v2 + 1]; ++e2) {
            for (int32_t e1 = F->off[v1]; e1 < F->off[v1 + 1]; ++e1) {
                int32_t n1 = F->c[e1], n2 = F->c[e2];
                if (n1 == n2) continue;
                int32_t p1, p2;
                if (first_common(F->off, F->c, n1, n2, &p1, &p2) < 0) continue;
                float a = F->w[e1], b = F->w[e2], c1 = F->w[p1], c2 = F->w[p2];
                if (a < b) {
                    if (a < c1 && a < c2)
                        inv[e1] = 1;
                    else if (c1 < c2)
                        inv[p1] = 1;
                    else
                        inv[p2] = 1;
                } else {
                    if (b < c1 && b < c2)
                        inv[e2] = 1;
                    else if (c1 < c2)
                        inv[p1] = 1;
                    else
                        inv[p2] = 1;
                }
            }
        }
    }
    int any = forest_remove_mask(F, inv);
    free(inv);
    return any;
}

/* filter_by_thresholding (src/edge_contractions_woc_thrust.cu:522-542) */
static int forest_threshold(forest_t *F)
{
    csum_acc acc;
    cacc_init(&acc);
    for (int64_t e = 0; e < F->m2; ++e) cacc_push(&acc, F->w[e] >= 0.0f ? (double)F->w[e] : 0.0);
    int64_t cnt = 0;
    for (int64_t e = 0; e < F->m2; ++e) cnt += F->w[e] >= 0.0f;
    double S = cacc_finish(&acc);
    float thr = (0.9f * (float)S) / (float)cnt;
    int64_t w2 = 0;
    for (int64_t e = 0; e < F->m2; ++e) {
        if (F->w[e] < thr) continue;
        F->r[w2] = F->r[e];
        F->c[w2] = F->c[e];
        F->w[w2] = F->w[e];
        w2++;
    }
    if (w2 == F->m2) return 0;
    F->m2 = w2;
    forest_offsets(F);
    return 1;
}

/* Rooted view of the forest: parent pointers from a BFS started at each
 * component's minimum vertex.  Used to read off the unique forest path of a
 * repulsive edge, which is what the reference's frontier expansion
 * (expand_cuda, filter_cycles, src/edge_contractions_woc_thrust.cu:149-410)
 * walks from both ends. */
typedef struct {
    int32_t *par, *dep;
    float *pw;
} rooted_t;

static void forest_root(const forest_t *F, rooted_t *T)
{
    int32_t n = F->nn;
    for (int32_t v = 0; v < n; ++v) {
        T->par[v] = -2;
        T->dep[v] = 0;
        T->pw[v] = 0.0f;
    }
    int32_t *queue = NEW(int32_t, n);
    for (int32_t s = 0; s < n; ++s) {
        if (T->par[s] != -2) continue;
        T->par[s] = -1;
        int32_t qh = 0, qt = 0;
        queue[qt++] = s;
        while (qh < qt) {
            int32_t x = queue[qh++];
            for (int32_t k = F->off[x]; k < F->off[x + 1]; ++k) {
                int32_t y = F->c[k];
                if (T->par[y] != -2) continue;
                T->par[y] = x;
                T->dep[y] = T->dep[x] + 1;
                T->pw[y] = F->w[k];
                queue[qt++] = y;
            }
        }
    }
    free(queue);
}

static int32_t path_length(const rooted_t *T, int32_t a, int32_t b)
{
    int32_t L = 0;
    while (T->dep[a] > T->dep[b]) {
        a = T->par[a];
        L++;
    }
    while (T->dep[b] > T->dep[a]) {
        b = T->par[b];
        L++;
    }
    while (a != b) {
        a = T->par[a];
        b = T->par[b];
        L += 2;
    }
    return L;
}

/* path v1 -> v2 as a list of (child,parent) edges in walking order */
static int32_t path_edges(const rooted_t *T, int32_t a, int32_t b, int32_t *eu, int32_t *ev, float *ew)
{
    int32_t la = 0, lb = 0;
    int32_t xa = a, xb = b;
    while (T->dep[xa] > T->dep[xb]) {
        xa = T->par[xa];
        la++;
    }
    while (T->dep[xb] > T->dep[xa]) {
        xb = T->par[xb];
        lb++;
    }
    while (xa != xb) {
        xa = T->par[xa];
        xb = T->par[xb];
        la++;
        lb++;
    }
    int32_t L = la + lb;
    xa = a;
    for (int32_t k = 0; k < la; ++k) {
        eu[k] = xa;
        ev[k] = T->par[xa];
        ew[k] = T->pw[xa];
        xa = T->par[xa];
    }
    xb = b;
    for (int32_t k = 0; k < lb; ++k) {
        eu[L - 1 - k] = xb;
        ev[L - 1 - k] = T->par[xb];
        ew[L - 1 - k] = T->pw[xb];
        xb = T->par[xb];
    }
    return L;
}

/* one expansion stage at depths (dr,dc): every repulsive edge whose forest
 * path has dr+dc edges has its frontiers meet; the bottleneck is the first
 * minimum met from v1 over the first dr edges and from v2 over the last dc
 * edges; the row side wins only when strictly smaller (reduce_intersecting_paths,
 * src/edge_contractions_woc_thrust.cu:201-216). */
static int forest_resolve(forest_t *F, const rooted_t *T, const int32_t *plen, int32_t dr, int32_t dc)
{
    int32_t s = dr + dc;
    int64_t np = 0;
    uint64_t *pairs = NULL;
    int32_t cap = 0;
    int32_t *eu = NULL, *ev = NULL;
    float *ew = NULL;
    for (int64_t k = 0; k < F->R; ++k) {
        if (plen[k] != s) continue;
        if (!pairs) pairs = NEW(uint64_t, F->R);
        if (s > cap) {
            free(eu);
            free(ev);
            free(ew);
            cap = s;
            eu = NEW(int32_t, cap);
            ev = NEW(int32_t, cap);
            ew = NEW(float, cap);
        }
        int32_t L = path_edges(T, F->rr[k], F->rc[k], eu, ev, ew);
        (void)L;
        float brow = FLT_MAX, bcol = FLT_MAX;
        int32_t irow = -1, icol = -1;
        for (int32_t q = 0; q < dr; ++q)
            if (ew[q] < brow) {
                brow = ew[q];
                irow = q;
            }
        for (int32_t q = 0; q < dc; ++q)
            if (ew[s - 1 - q] < bcol) {
                bcol = ew[s - 1 - q];
                icol = s - 1 - q;
            }
        int32_t pick = (brow < bcol) ? irow : icol;
        if (pick < 0) pick = irow >= 0 ? irow : 0;
        pairs[np++] = pack2(eu[pick], ev[pick]);
    }
    free(eu);
    free(ev);
    free(ew);
    if (np == 0) {
        free(pairs);
        return 0;
    }
    forest_remove_pairs(F, pairs, np);
    free(pairs);
    return 1;
}

int orc_woc(const orc_graph *A, int32_t *map_out, int64_t *map_size, int32_t *nr_out)
{
    return orc_woc_ex(A, map_out, map_size, nr_out, 0);
}

int orc_woc_ex(const orc_graph *A, int32_t *map_out, int64_t *map_size, int32_t *nr_out, int pentagons)
{
    forest_t F;
    memset(&F, 0, sizeof(F));
    F.nn = graph_max_dim(A);
    *map_size = 0;
    *nr_out = 0;
    /* ctor (src/edge_contractions_woc.cu:341-383): partition at cost > 0 */
    int64_t npos = 0;
    for (int64_t e = 0; e < A->n; ++e) npos += A->cost[e] > 0.0f;
    if (npos == 0) return ORC_OK;
    int32_t *pi = NEW(int32_t, npos), *pj = NEW(int32_t, npos);
    float *pw = NEW(float, npos);
    F.rr = NEW(int32_t, A->n - npos + 1);
    F.rc = NEW(int32_t, A->n - npos + 1);
    int64_t a = 0, b = 0;
    for (int64_t e = 0; e < A->n; ++e) {
        if (A->cost[e] > 0.0f) {
            pi[a] = A->row[e];
            pj[a] = A->col[e];
            pw[a] = A->cost[e];
            a++;
        } else {
            F.rr[b] = A->row[e];
            F.rc[b] = A->col[e];
            b++;
        }
    }
    F.R = b;
    int32_t *ids = NEW(int32_t, npos);
    int64_t k;
    orc_msf(npos, pi, pj, pw, ids, &k);
    /* to_undirected + coo_sorting of the forest */
    uint64_t *keys = NEW(uint64_t, 2 * k);
    for (int64_t q = 0; q < k; ++q) {
        int32_t e = ids[q];
        keys[2 * q] = pack2(pi[e], pj[e]);
        keys[2 * q + 1] = pack2(pj[e], pi[e]);
    }
    int64_t *ord = stable_order_u64(keys, 2 * k);
    F.m2 = 2 * k;
    F.r = NEW(int32_t, F.m2);
    F.c = NEW(int32_t, F.m2);
    F.w = NEW(float, F.m2);
    for (int64_t q = 0; q < 2 * k; ++q) {
        int64_t p = ord[q];
        F.r[q] = (int32_t)(keys[p] >> 32);
        F.c[q] = (int32_t)(keys[p] & 0xFFFFFFFFu);
        F.w[q] = pw[ids[p / 2]];
    }
    free(ord);
    free(keys);
    free(ids);
    free(pi);
    free(pj);
    free(pw);
    F.off = NEW(int32_t, F.nn + 1);
    F.lab = NEW(int32_t, F.nn);
    forest_offsets(&F);
    int32_t nr = 0;
    if (F.m2 > 0) {
        /* find_contraction_mapping (src/edge_contractions_woc.cu:387-423) */
        forest_filter_by_cc(&F);
        if (forest_check_triangles(&F)) forest_filter_by_cc(&F);
        forest_check_quadrangles(&F);
        if (pentagons) forest_check_pentagons(&F);
        if (F.m2 > 0) {
            /* edge_contractions_woc_thrust::find_contraction_mapping (:544-599) */
            int64_t R = forest_filter_by_cc(&F);
            rooted_t T;
            T.par = NEW(int32_t, F.nn);
            T.dep = NEW(int32_t, F.nn);
            T.pw = NEW(float, F.nn);
            int32_t *plen = NEW(int32_t, F.R + 1);
            int stale = 1;
            int32_t dr = 0, dc = 0;
            int32_t itr = 0;
#define WOC_RESET()                                            \
    do {                                                       \
        R = forest_filter_by_cc(&F);                           \
        dr = dc = 0;                                           \
        stale = 1;                                             \
    } while (0)
#define WOC_PATHS()                                            \
    do {                                                       \
        if (stale) {                                           \
            forest_root(&F, &T);                               \
            for (int64_t q = 0; q < F.R; ++q)                  \
                plen[q] = path_length(&T, F.rr[q], F.rc[q]);   \
            stale = 0;                                         \
        }                                                      \
    } while (0)
            while (R > 0 && F.m2 > 0) {
                if (itr % 5 == 0)
                    if (forest_threshold(&F)) WOC_RESET();
                if (R == 0 || F.m2 == 0) break;
                dr++;
                WOC_PATHS();
                if (forest_resolve(&F, &T, plen, dr, dc)) WOC_RESET();
                if (R == 0 || F.m2 == 0) break;
                dc++;
                WOC_PATHS();
                if (forest_resolve(&F, &T, plen, dr, dc)) WOC_RESET();
                itr++;
            }
#undef WOC_RESET
#undef WOC_PATHS
            free(plen);
            free(T.par);
            free(T.dep);
            free(T.pw);
            orc_compress_label_sequence(F.lab, F.nn, F.nn - 1, map_out);
            *map_size = F.nn;
            nr = (int32_t)F.m2;
        }
    }
    *nr_out = nr;
    free(F.r);
    free(F.c);
    free(F.w);
    free(F.off);
    free(F.lab);
    free(F.rr);
    free(F.rc);
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* conflicted cycles (src/conflicted_cycles_cuda.cu:13-343)                  */
/* ------------------------------------------------------------------------ */
/* number of cycle searches whose budget overflowed since the last reset
 * (reported per solve in orc_stats.truncations; single-threaded use) */
static int32_t g_truncations = 0;
typedef struct {
    int32_t *buf; /* 3*budget */
    int64_t budget, count;
    int full;
} tri_emit_t;

/* write_triangle (:13-29): sorted (min, median, max) */
static inline void tri_emit(tri_emit_t *t, int32_t a, int32_t b, int32_t c)
{
    if (t->full) return;
    if (t->count >= t->budget) {
        t->count++;
        t->full = 1;
        return;
    }
    int32_t lo = imin(a, imin(b, c)), hi = imax(a, imax(b, c));
    int32_t md = imax(imin(a, b), imin(imax(a, b), c));
    t->buf[3 * t->count] = lo;
    t->buf[3 * t->count + 1] = md;
    t->buf[3 * t->count + 2] = hi;
    t->count++;
}

static int tri_degenerate(const int32_t *t) { return t[0] == t[1] || t[0] == t[2] || t[1] == t[2]; }

/* normalize (remove degenerate, sort, unique) -- rearrange_triangles
 * (include/rama_utils.h:352-363) and normalize_triangles (:325-350) */
static int64_t tri_normalize(int32_t *buf, int64_t n)
{
    int64_t w = 0;
    for (int64_t k = 0; k < n; ++k) {
        if (tri_degenerate(buf + 3 * k)) continue;
        int32_t a = buf[3 * k], b = buf[3 * k + 1], c = buf[3 * k + 2];
        int32_t lo = imin(a, imin(b, c)), hi = imax(a, imax(b, c));
        int32_t md = imax(imin(a, b), imin(imax(a, b), c));
        buf[3 * w] = lo;
        buf[3 * w + 1] = md;
        buf[3 * w + 2] = hi;
        w++;
    }
    if (w == 0) return 0;
    /* stable sort by t3, then by (t1,t2) */
    uint64_t *k1 = NEW(uint64_t, w);
    for (int64_t k = 0; k < w; ++k) k1[k] = (uint32_t)buf[3 * k + 2];
    int64_t *o1 = stable_order_u64(k1, w);
    for (int64_t k = 0; k < w; ++k) k1[k] = pack2(buf[3 * o1[k]], buf[3 * o1[k] + 1]);
    int64_t *o2 = stable_order_u64(k1, w);
    int32_t *tmp = NEW(int32_t, 3 * w);
    int64_t u = 0;
    for (int64_t k = 0; k < w; ++k) {
        const int32_t *t = buf + 3 * o1[o2[k]];
        if (u > 0 && tmp[3 * (u - 1)] == t[0] && tmp[3 * (u - 1) + 1] == t[1] && tmp[3 * (u - 1) + 2] == t[2]) continue;
        tmp[3 * u] = t[0];
        tmp[3 * u + 1] = t[1];
        tmp[3 * u + 2] = t[2];
        u++;
    }
    memcpy(buf, tmp, sizeof(int32_t) * (size_t)(3 * u));
    free(tmp);
    free(o1);
    free(o2);
    free(k1);
    return u;
}

/* all common neighbours of a and b in ascending order */
#define FOR_COMMON(off, adj, A_, B_, MID, BODY)                                    \
    do {                                                                           \
        int32_t x_ = (off)[A_], y_ = (off)[B_];                                    \
        int32_t xe_ = (off)[(A_) + 1], ye_ = (off)[(B_) + 1];                      \
        while (x_ < xe_ && y_ < ye_) {                                             \
            int32_t na_ = (adj)[x_], nb_ = (adj)[y_];                              \
            if (na_ == nb_) {                                                      \
                int32_t MID = na_;                                                 \
                x_++;                                                              \
                y_++;                                                              \
                BODY;                                                              \
            } else if (na_ < nb_)                                                  \
                x_++;                                                              \
            else                                                                   \
                y_++;                                                              \
        }                                                                          \
    } while (0)

/* Expansions of one stage of the cycle search and the triangles each emits
 * (3-cycles :31-61, 4-cycles :63-101, 5-cycles :103-148).  emit_first()
 * emits the first `keep` emissions of expansion x, in the reference's order. */
typedef struct {
    int kind; /* 3, 4 or 5 */
    const csr_t *P;
    const int32_t *rr, *rc;
    const int64_t *xo; /* kinds 4, 5: first expansion of each rep edge (R + 1) */
    int64_t R;
} stage_t;

static void stage_locate(const stage_t *S, int64_t x, int64_t *r, int64_t *loc)
{
    if (S->kind == 3) {
        *r = x;
        *loc = 0;
        return;
    }
    int64_t lo = 0, hi = S->R; /* largest r with xo[r] <= x */
    while (lo < hi) {
        int64_t mid = (lo + hi + 1) >> 1;
        if (S->xo[mid] <= x)
            lo = mid;
        else
            hi = mid - 1;
    }
    *r = lo;
    *loc = x - S->xo[lo];
}

/* emissions of expansion x (keep < 0: count only, emit nothing) */
static int64_t stage_expand(const stage_t *S, int64_t x, int64_t keep, tri_emit_t *T)
{
    int64_t r, loc, n = 0;
    stage_locate(S, x, &r, &loc);
    const csr_t *P = S->P;
    int32_t v1 = S->rr[r], v2 = S->rc[r];
#define EMIT(a, b, c)                                   \
    do {                                                \
        if (keep >= 0 && n < keep) tri_emit(T, a, b, c); \
        n++;                                            \
    } while (0)
    if (S->kind == 3) {
        FOR_COMMON(P->off, P->adj, v1, v2, mid, EMIT(v1, v2, mid));
    } else if (S->kind == 4) {
        int32_t n1 = P->adj[P->off[v1] + (int32_t)loc];
        FOR_COMMON(P->off, P->adj, n1, v2, mid, {
            EMIT(v1, v2, n1);
            EMIT(v2, n1, mid);
        });
    } else {
        int64_t d1 = P->off[v1 + 1] - P->off[v1];
        int32_t n1 = P->adj[P->off[v1] + (int32_t)(loc % d1)];
        int32_t n2 = P->adj[P->off[v2] + (int32_t)(loc / d1)];
        if (n1 != n2) {
            FOR_COMMON(P->off, P->adj, n1, n2, mid, {
                EMIT(v1, v2, n1);
                EMIT(v2, n1, mid);
                EMIT(v2, mid, n2);
            });
        }
    }
#undef EMIT
    return n;
}

#define STAGE_CHUNK ((int64_t)1 << 24)

/* One stage over X expansions in chunks; a chunk that does not fit the room
 * left keeps its emissions round-robin (C4) and fills the budget. */
static void stage_run(const stage_t *S, int64_t X, tri_emit_t *T)
{
    int64_t *m = NEW(int64_t, X < STAGE_CHUNK ? X + 1 : STAGE_CHUNK);
    for (int64_t x0 = 0; x0 < X && T->count <= T->budget; x0 += STAGE_CHUNK) {
        int64_t xn = X - x0 < STAGE_CHUNK ? X - x0 : STAGE_CHUNK;
        int64_t M = 0, mx = 0;
        for (int64_t q = 0; q < xn; ++q) {
            m[q] = stage_expand(S, x0 + q, -1, T);
            M += m[q];
            if (m[q] > mx) mx = m[q];
        }
        int64_t rem = T->budget - T->count;
        if (M <= rem) {
            for (int64_t q = 0; q < xn; ++q)
                if (m[q]) stage_expand(S, x0 + q, m[q], T);
            continue;
        }
        /* largest K with sum_q min(m_q, K) <= rem */
        int64_t lo = 0, hi = mx;
        while (lo < hi) {
            int64_t K = (lo + hi + 1) >> 1, s = 0;
            for (int64_t q = 0; q < xn; ++q) s += m[q] < K ? m[q] : K;
            if (s <= rem)
                lo = K;
            else
                hi = K - 1;
        }
        const int64_t K = lo;
        int64_t sK = 0;
        for (int64_t q = 0; q < xn; ++q) sK += m[q] < K ? m[q] : K;
        const int64_t extra = rem - sK;
        int64_t big = 0;
        for (int64_t q = 0; q < xn; ++q) {
            int64_t keep = m[q] < K ? m[q] : K;
            if (m[q] > K) {
                if (big < extra) keep++;
                big++;
            }
            if (keep) stage_expand(S, x0 + q, keep, T);
        }
        T->count = T->budget + 1; /* the reference's counter has overflowed */
        T->full = 1;
    }
    free(m);
}

int orc_conflicted_cycles(const orc_graph *A, int32_t max_len, float tri_factor, float tol_ratio, int32_t *tri_out,
                          int64_t tri_cap, int64_t *num_out, int64_t *raw_count)
{
    *num_out = 0;
    *raw_count = 0;
    if (max_len > 5) return ORC_ERR_INVALID_ARG;
    if (max_len < 3 || A->n == 0) return ORC_OK;
    float mn = A->cost[0];
    for (int64_t e = 1; e < A->n; ++e)
        if (A->cost[e] < mn) mn = A->cost[e];
    float thresh = mn * tol_ratio;                  /* determine_threshold (:170-174) */
    float pos_tol = -1.0f * thresh;                 /* create_matrices (:176-220) */
    int64_t np = 0, R = 0;
    for (int64_t e = 0; e < A->n; ++e) {
        np += A->cost[e] > pos_tol;
        R += A->cost[e] < thresh;
    }
    if (np == 0 || R == 0) return ORC_OK;
    int32_t N = graph_max_dim(A);
    int32_t *pr = NEW(int32_t, np), *pc = NEW(int32_t, np), *rr = NEW(int32_t, R), *rc = NEW(int32_t, R);
    float *pw = NEW(float, np);
    int64_t a = 0, b = 0;
    for (int64_t e = 0; e < A->n; ++e) {
        if (A->cost[e] > pos_tol) {
            pr[a] = A->row[e];
            pc[a] = A->col[e];
            pw[a] = A->cost[e];
            a++;
        }
        if (A->cost[e] < thresh) {
            rr[b] = A->row[e];
            rc[b] = A->col[e];
            b++;
        }
    }
    csr_t P;
    build_symmetric_csr(N, np, pr, pc, pw, &P);
    int64_t budget = (int64_t)(int32_t)(tri_factor * (float)R); /* (:247) */
    if (budget < 0) budget = 0;
    tri_emit_t T;
    T.buf = NEW(int32_t, 3 * (budget + 1));
    T.budget = budget;
    T.count = 0;
    T.full = 0;
    int64_t *xo = NEW(int64_t, R + 1);
    stage_t S = {3, &P, rr, rc, xo, R};
    /* find_triangles_parallel (:31-61): one expansion per rep edge */
    stage_run(&S, R, &T);
    if (max_len >= 4 && T.count < budget) {
        T.count = tri_normalize(T.buf, T.count);
        /* find_quadrangles_parallel (:63-101): a rep edge and a neighbour of its row */
        xo[0] = 0;
        for (int64_t r = 0; r < R; ++r) xo[r + 1] = xo[r] + (P.off[rr[r] + 1] - P.off[rr[r]]);
        S.kind = 4;
        stage_run(&S, xo[R], &T);
    }
    if (max_len >= 5 && T.count < budget) {
        T.count = tri_normalize(T.buf, T.count);
        /* find_pentagons_parallel (:103-148): a rep edge and a neighbour of each end */
        xo[0] = 0;
        for (int64_t r = 0; r < R; ++r)
            xo[r + 1] = xo[r] + (int64_t)(P.off[rr[r] + 1] - P.off[rr[r]]) * (int64_t)(P.off[rc[r] + 1] - P.off[rc[r]]);
        S.kind = 5;
        stage_run(&S, xo[R], &T);
    }
    free(xo);
    int64_t keep = T.count < budget ? T.count : budget;
    if (T.count > budget) g_truncations++;
    if (keep > tri_cap) keep = tri_cap;
    memcpy(tri_out, T.buf, sizeof(int32_t) * (size_t)(3 * keep));
    *num_out = keep;
    *raw_count = T.count;
    free(T.buf);
    csr_free(&P);
    free(pr);
    free(pc);
    free(rr);
    free(rc);
    free(pw);
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* triangle message passing (src/multicut_message_passing.cu:15-360)         */
/* ------------------------------------------------------------------------ */
struct orc_mp {
    int64_t T, E;
    int32_t *t1, *t2, *t3;
    int32_t *row, *col;
    float *cost;
    int32_t *cnt;
    float *c12, *c13, *c23;
    int32_t *e12, *e13, *e23;
    int32_t *inc_off; /* E+1 */
    int32_t *inc;     /* 3T: 3*tri + slot, in (tri, slot) order per edge */
    float *diff;      /* 3T */
};

static int64_t edge_find(const int32_t *off, const int32_t *col, int32_t a, int32_t b)
{
    int32_t lo = off[a], hi = off[a + 1];
    while (lo < hi) {
        int32_t m = lo + (hi - lo) / 2;
        if (col[m] < b)
            lo = m + 1;
        else
            hi = m;
    }
    return (lo < off[a + 1] && col[lo] == b) ? lo : -1;
}

orc_mp *orc_mp_create(const orc_graph *A, const int32_t *t1, const int32_t *t2, const int32_t *t3, int64_t T0)
{
    orc_mp *mp = (orc_mp *)xcalloc(1, sizeof(orc_mp));
    int32_t *buf = NEW(int32_t, 3 * T0 + 3);
    for (int64_t k = 0; k < T0; ++k) {
        buf[3 * k] = t1[k];
        buf[3 * k + 1] = t2[k];
        buf[3 * k + 2] = t3[k];
    }
    int64_t T = tri_normalize(buf, T0); /* normalize_triangles (:79) */
    mp->T = T;
    /* triangle edges not in A, sorted unique; union with A (:81-158) */
    int32_t nmax = graph_max_dim(A);
    for (int64_t k = 0; k < 3 * T; ++k) nmax = imax(nmax, buf[k] + 1);
    int32_t *aoff = NEW(int32_t, nmax + 2);
    orc_compute_offsets(A->row, A->n, nmax, aoff);
    uint64_t *nk = NEW(uint64_t, 3 * T + 1);
    int64_t nn = 0;
    for (int64_t k = 0; k < T; ++k) {
        int32_t a = buf[3 * k], b = buf[3 * k + 1], c = buf[3 * k + 2];
        int32_t pr[3][2] = {{a, b}, {a, c}, {b, c}};
        for (int s = 0; s < 3; ++s)
            if (edge_find(aoff, A->col, pr[s][0], pr[s][1]) < 0) nk[nn++] = pack2(pr[s][0], pr[s][1]);
    }
    int64_t *no = stable_order_u64(nk, nn);
    int64_t nu = 0;
    uint64_t *nku = NEW(uint64_t, nn + 1);
    for (int64_t k = 0; k < nn; ++k) {
        uint64_t key = nk[no[k]];
        if (nu > 0 && nku[nu - 1] == key) continue;
        nku[nu++] = key;
    }
    free(no);
    free(nk);
    int64_t E = A->n + nu;
    mp->E = E;
    mp->row = NEW(int32_t, E);
    mp->col = NEW(int32_t, E);
    mp->cost = NEW(float, E);
    int64_t x = 0, y = 0, w = 0;
    while (x < A->n || y < nu) {
        uint64_t ka = x < A->n ? pack2(A->row[x], A->col[x]) : UINT64_MAX;
        uint64_t kb = y < nu ? nku[y] : UINT64_MAX;
        if (ka <= kb) {
            mp->row[w] = A->row[x];
            mp->col[w] = A->col[x];
            mp->cost[w] = A->cost[x];
            x++;
        } else {
            mp->row[w] = (int32_t)(kb >> 32);
            mp->col[w] = (int32_t)(kb & 0xFFFFFFFFu);
            mp->cost[w] = 0.0f;
            y++;
        }
        w++;
    }
    free(nku);
    /* correspondences + counters (compute_triangle_edge_correspondence, :15-62) */
    int32_t *moff = NEW(int32_t, nmax + 2);
    orc_compute_offsets(mp->row, E, nmax, moff);
    mp->t1 = NEW(int32_t, T);
    mp->t2 = NEW(int32_t, T);
    mp->t3 = NEW(int32_t, T);
    mp->e12 = NEW(int32_t, T);
    mp->e13 = NEW(int32_t, T);
    mp->e23 = NEW(int32_t, T);
    mp->c12 = (float *)xcalloc((size_t)T, sizeof(float));
    mp->c13 = (float *)xcalloc((size_t)T, sizeof(float));
    mp->c23 = (float *)xcalloc((size_t)T, sizeof(float));
    mp->cnt = (int32_t *)xcalloc((size_t)E, sizeof(int32_t));
    for (int64_t k = 0; k < T; ++k) {
        int32_t a = buf[3 * k], b = buf[3 * k + 1], c = buf[3 * k + 2];
        mp->t1[k] = a;
        mp->t2[k] = b;
        mp->t3[k] = c;
        mp->e12[k] = (int32_t)edge_find(moff, mp->col, a, b);
        mp->e13[k] = (int32_t)edge_find(moff, mp->col, a, c);
        mp->e23[k] = (int32_t)edge_find(moff, mp->col, b, c);
        mp->cnt[mp->e12[k]]++;
        mp->cnt[mp->e13[k]]++;
        mp->cnt[mp->e23[k]]++;
    }
    mp->inc_off = NEW(int32_t, E + 1);
    mp->inc_off[0] = 0;
    for (int64_t e = 0; e < E; ++e) mp->inc_off[e + 1] = mp->inc_off[e] + mp->cnt[e];
    mp->inc = NEW(int32_t, 3 * T + 1);
    mp->diff = NEW(float, 3 * T + 1);
    int32_t *fill = NEW(int32_t, E + 1);
    memcpy(fill, mp->inc_off, sizeof(int32_t) * (size_t)E);
    for (int64_t k = 0; k < T; ++k) {
        mp->inc[fill[mp->e12[k]]++] = (int32_t)(3 * k);
        mp->inc[fill[mp->e13[k]]++] = (int32_t)(3 * k + 1);
        mp->inc[fill[mp->e23[k]]++] = (int32_t)(3 * k + 2);
    }
    free(fill);
    free(moff);
    free(aoff);
    free(buf);
    return mp;
}

void orc_mp_free(orc_mp *mp)
{
    if (!mp) return;
    free(mp->t1);
    free(mp->t2);
    free(mp->t3);
    free(mp->row);
    free(mp->col);
    free(mp->cost);
    free(mp->cnt);
    free(mp->c12);
    free(mp->c13);
    free(mp->c23);
    free(mp->e12);
    free(mp->e13);
    free(mp->e23);
    free(mp->inc_off);
    free(mp->inc);
    free(mp->diff);
    free(mp);
}

/* triangle_lb_func (:186-199) */
static inline float tri_lb(float c12, float c13, float c23)
{
    float lb = 0.0f;
    lb = fminf(lb, c12 + c13);
    lb = fminf(lb, c12 + c23);
    lb = fminf(lb, c13 + c23);
    lb = fminf(lb, c12 + c13 + c23);
    return lb;
}

/* lower_bound = edge_lower_bound + triangle_lower_bound (:201-216), CSUM (C2) */
double orc_mp_lower_bound(orc_mp *mp)
{
    csum_acc a;
    cacc_init(&a);
    for (int64_t e = 0; e < mp->E; ++e) cacc_push(&a, mp->cost[e] < 0.0f ? (double)mp->cost[e] : 0.0);
    double le = cacc_finish(&a);
    cacc_init(&a);
    for (int64_t t = 0; t < mp->T; ++t) cacc_push(&a, (double)tri_lb(mp->c12[t], mp->c13[t], mp->c23[t]));
    double lt = cacc_finish(&a);
    return le + lt;
}

/* send_messages_to_triplets (:218-269) */
void orc_mp_send_messages_to_triplets(orc_mp *mp)
{
    for (int64_t t = 0; t < mp->T; ++t) {
        mp->c12[t] += mp->cost[mp->e12[t]] / (float)mp->cnt[mp->e12[t]];
        mp->c13[t] += mp->cost[mp->e13[t]] / (float)mp->cnt[mp->e13[t]];
        mp->c23[t] += mp->cost[mp->e23[t]] / (float)mp->cnt[mp->e23[t]];
    }
    for (int64_t e = 0; e < mp->E; ++e)
        if (mp->cnt[e] > 0) mp->cost[e] = 0.0f;
}

/* decrease_triangle_costs_func::min_marginal (:275-280) */
static inline float min_marginal(float x, float y, float z)
{
    float mm1 = fminf(x + y + z, fminf(x + y, x + z));
    float yz = y + z;
    float mm0 = (0.0 < (double)yz) ? 0.0f : yz;
    return mm1 - mm0;
}

/* the six min-marginal moves of decrease_triangle_costs_func (:282-332);
 * the 1/3 and 1/2 steps evaluate in double like the reference's
 * `t -= 1.0/3.0*mm` on float operands. */
static inline void tri_update(float *p12, float *p13, float *p23, float *d12, float *d13, float *d23)
{
    float t12 = *p12, t13 = *p13, t23 = *p23;
    float e12 = 0.0f, e13 = 0.0f, e23 = 0.0f;
    {
        float mm = min_marginal(t12, t13, t23);
        t12 = (float)((double)t12 - (1.0 / 3.0) * (double)mm);
        e12 = (float)((double)e12 + (1.0 / 3.0) * (double)mm);
    }
    {
        float mm = min_marginal(t13, t12, t23);
        t13 = (float)((double)t13 - (1.0 / 2.0) * (double)mm);
        e13 = (float)((double)e13 + (1.0 / 2.0) * (double)mm);
    }
    {
        float mm = min_marginal(t23, t12, t13);
        t23 -= mm;
        e23 += mm;
    }
    {
        float mm = min_marginal(t12, t13, t23);
        t12 = (float)((double)t12 - (1.0 / 2.0) * (double)mm);
        e12 = (float)((double)e12 + (1.0 / 2.0) * (double)mm);
    }
    {
        float mm = min_marginal(t13, t12, t23);
        t13 -= mm;
        e13 += mm;
    }
    {
        float mm = min_marginal(t12, t13, t23);
        t12 -= mm;
        e12 += mm;
    }
    *p12 = t12;
    *p13 = t13;
    *p23 = t23;
    *d12 = e12;
    *d13 = e13;
    *d23 = e23;
}

/* send_messages_to_edges (:335-348); arriving messages summed by RSUM (C3) */
void orc_mp_send_messages_to_edges(orc_mp *mp)
{
    for (int64_t t = 0; t < mp->T; ++t)
        tri_update(&mp->c12[t], &mp->c13[t], &mp->c23[t], &mp->diff[3 * t], &mp->diff[3 * t + 1], &mp->diff[3 * t + 2]);
    for (int64_t e = 0; e < mp->E; ++e) {
        if (mp->cnt[e] == 0) continue;
        rsum_acc a;
        racc_init(&a);
        for (int32_t k = mp->inc_off[e]; k < mp->inc_off[e + 1]; ++k) racc_push(&a, mp->diff[mp->inc[k]]);
        mp->cost[e] = mp->cost[e] + racc_finish(&a);
    }
}

void orc_mp_iteration(orc_mp *mp)
{
    orc_mp_send_messages_to_triplets(mp);
    orc_mp_send_messages_to_edges(mp);
}

void orc_mp_info(const orc_mp *mp, int64_t *num_edges, int64_t *num_triangles)
{
    if (num_edges) *num_edges = mp->E;
    if (num_triangles) *num_triangles = mp->T;
}

void orc_mp_copy_edges(const orc_mp *mp, int32_t *row, int32_t *col, float *cost, int32_t *counter)
{
    size_t E = (size_t)mp->E;
    if (row) memcpy(row, mp->row, 4 * E);
    if (col) memcpy(col, mp->col, 4 * E);
    if (cost) memcpy(cost, mp->cost, 4 * E);
    if (counter) memcpy(counter, mp->cnt, 4 * E);
}

void orc_mp_copy_triangles(const orc_mp *mp, int32_t *t1, int32_t *t2, int32_t *t3, float *c12, float *c13, float *c23,
                           int32_t *e12, int32_t *e13, int32_t *e23)
{
    size_t T = (size_t)mp->T;
    if (t1) memcpy(t1, mp->t1, 4 * T);
    if (t2) memcpy(t2, mp->t2, 4 * T);
    if (t3) memcpy(t3, mp->t3, 4 * T);
    if (c12) memcpy(c12, mp->c12, 4 * T);
    if (c13) memcpy(c13, mp->c13, 4 * T);
    if (c23) memcpy(c23, mp->c23, 4 * T);
    if (e12) memcpy(e12, mp->e12, 4 * T);
    if (e13) memcpy(e13, mp->e13, 4 * T);
    if (e23) memcpy(e23, mp->e23, 4 * T);
}

/* ------------------------------------------------------------------------ */
/* dual solver (src/dual_solver.cu:7-63)                                     */
/* ------------------------------------------------------------------------ */
/* get_lb (include/rama_utils.h:179-190), CSUM */
static double graph_lb(const orc_graph *A)
{
    csum_acc a;
    cacc_init(&a);
    for (int64_t e = 0; e < A->n; ++e) cacc_push(&a, A->cost[e] < 0.0f ? (double)A->cost[e] : 0.0);
    return cacc_finish(&a);
}

static double dual_update_cycle_length(orc_graph **pA, int32_t c, int32_t num_iter, float tri_factor, float tol,
                                       int64_t *num_tri)
{
    orc_graph *A = *pA;
    /* the budget is at most tri_factor * E; allocate for it */
    int64_t cap = (int64_t)(tri_factor * (double)A->n) + 8;
    int32_t *tri = NEW(int32_t, 3 * cap);
    int64_t num = 0, raw = 0;
    orc_conflicted_cycles(A, c, tri_factor, tol, tri, cap, &num, &raw);
    *num_tri = raw;
    if (raw == 0) {
        free(tri);
        return graph_lb(A);
    }
    int32_t *t1 = NEW(int32_t, num + 1), *t2 = NEW(int32_t, num + 1), *t3 = NEW(int32_t, num + 1);
    for (int64_t k = 0; k < num; ++k) {
        t1[k] = tri[3 * k];
        t2[k] = tri[3 * k + 1];
        t3[k] = tri[3 * k + 2];
    }
    free(tri);
    orc_mp *mp = orc_mp_create(A, t1, t2, t3, num);
    free(t1);
    free(t2);
    free(t3);
    double prev = 0.0;
    for (int32_t it = 0; it < num_iter; ++it) {
        double lb = orc_mp_lower_bound(mp);
        if (it > 0 && (lb - prev) < 1e-3) break;
        orc_mp_iteration(mp);
        prev = lb;
    }
    double fin = orc_mp_lower_bound(mp);
    orc_graph *B = orc_graph_from_sorted(mp->E, mp->row, mp->col, mp->cost);
    orc_mp_free(mp);
    orc_graph_free(A);
    *pA = B;
    return fin;
}

double orc_dual_solver(orc_graph **pA, int32_t max_len, int32_t num_iter, float tri_factor, int32_t num_outer,
                       float tol, int64_t *num_triangles_last)
{
    if (num_triangles_last) *num_triangles_last = 0;
    if (max_len < 3 || num_iter == 0 || num_outer == 0) return graph_lb(*pA);
    double prev = 0.0, fin = 0.0;
    int64_t nt = 0;
    for (int32_t o = 0; o < num_outer; ++o) {
        for (int32_t c = 3; c <= max_len; ++c) fin = dual_update_cycle_length(pA, c, num_iter, tri_factor, tol, &nt);
        if (nt == 0 || (o > 0 && (fin - prev) < 1e-3)) break;
        prev = fin;
    }
    if (num_triangles_last) *num_triangles_last = nt;
    return fin;
}

/* ------------------------------------------------------------------------ */
/* FP64 oracle of the dual, for the error report of the FP32 messages        */
/* ------------------------------------------------------------------------ */
/* The dual solver (src/dual_solver.cu:7-63) with every cost, message and
 * bound in double.  The triangle search runs on the costs rounded to float:
 * it only selects triangles (thresholds, counts), and the FP32 solve makes the
 * same selection.  Message passing (src/multicut_message_passing.cu:218-348)
 * and the bound (:178-216) are evaluated in FP64 throughout. */
static inline double tri_lb64(double c12, double c13, double c23)
{
    double lb = 0.0;
    lb = fmin(lb, c12 + c13);
    lb = fmin(lb, c12 + c23);
    lb = fmin(lb, c13 + c23);
    lb = fmin(lb, c12 + c13 + c23);
    return lb;
}

static inline double min_marginal64(double x, double y, double z)
{
    double mm1 = fmin(x + y + z, fmin(x + y, x + z));
    double yz = y + z;
    double mm0 = yz > 0.0 ? 0.0 : yz;
    return mm1 - mm0;
}

typedef struct {
    double *cost, *c12, *c13, *c23, *diff;
} mp64_t;

static double mp64_lower_bound(const orc_mp *mp, const mp64_t *d)
{
    csum_acc a;
    cacc_init(&a);
    for (int64_t e = 0; e < mp->E; ++e) cacc_push(&a, d->cost[e] < 0.0 ? d->cost[e] : 0.0);
    double le = cacc_finish(&a);
    cacc_init(&a);
    for (int64_t t = 0; t < mp->T; ++t) cacc_push(&a, tri_lb64(d->c12[t], d->c13[t], d->c23[t]));
    return le + cacc_finish(&a);
}

static void mp64_iteration(const orc_mp *mp, mp64_t *d)
{
    for (int64_t t = 0; t < mp->T; ++t) {
        d->c12[t] += d->cost[mp->e12[t]] / (double)mp->cnt[mp->e12[t]];
        d->c13[t] += d->cost[mp->e13[t]] / (double)mp->cnt[mp->e13[t]];
        d->c23[t] += d->cost[mp->e23[t]] / (double)mp->cnt[mp->e23[t]];
    }
    for (int64_t e = 0; e < mp->E; ++e)
        if (mp->cnt[e] > 0) d->cost[e] = 0.0;
    const double third = 1.0 / 3.0, half = 1.0 / 2.0;
    for (int64_t t = 0; t < mp->T; ++t) {
        double t12 = d->c12[t], t13 = d->c13[t], t23 = d->c23[t], e12 = 0.0, e13 = 0.0, e23 = 0.0, mm;
        mm = min_marginal64(t12, t13, t23);
        t12 -= third * mm;
        e12 += third * mm;
        mm = min_marginal64(t13, t12, t23);
        t13 -= half * mm;
        e13 += half * mm;
        mm = min_marginal64(t23, t12, t13);
        t23 -= mm;
        e23 += mm;
        mm = min_marginal64(t12, t13, t23);
        t12 -= half * mm;
        e12 += half * mm;
        mm = min_marginal64(t13, t12, t23);
        t13 -= mm;
        e13 += mm;
        mm = min_marginal64(t12, t13, t23);
        t12 -= mm;
        e12 += mm;
        d->c12[t] = t12;
        d->c13[t] = t13;
        d->c23[t] = t23;
        d->diff[3 * t] = e12;
        d->diff[3 * t + 1] = e13;
        d->diff[3 * t + 2] = e23;
    }
    for (int64_t e = 0; e < mp->E; ++e)
        for (int32_t k = mp->inc_off[e]; k < mp->inc_off[e + 1]; ++k) d->cost[e] += d->diff[mp->inc[k]];
}

/* one cycle length: the graph *pA carries float costs, *pcd the same costs
 * in double; both are replaced by the reparametrised graph */
static double dual_update_cycle_length_f64(orc_graph **pA, double **pcd, int32_t c, int32_t num_iter,
                                           float tri_factor, float tol, int64_t *num_tri)
{
    orc_graph *A = *pA;
    const double *cd = *pcd;
    csum_acc acc;
    int64_t cap = (int64_t)(tri_factor * (double)A->n) + 8;
    int32_t *tri = NEW(int32_t, 3 * cap);
    int64_t num = 0, raw = 0;
    orc_conflicted_cycles(A, c, tri_factor, tol, tri, cap, &num, &raw);
    *num_tri = raw;
    if (raw == 0) {
        free(tri);
        cacc_init(&acc);
        for (int64_t e = 0; e < A->n; ++e) cacc_push(&acc, cd[e] < 0.0 ? cd[e] : 0.0);
        return cacc_finish(&acc);
    }
    int32_t *t1 = NEW(int32_t, num + 1), *t2 = NEW(int32_t, num + 1), *t3 = NEW(int32_t, num + 1);
    for (int64_t k = 0; k < num; ++k) {
        t1[k] = tri[3 * k];
        t2[k] = tri[3 * k + 1];
        t3[k] = tri[3 * k + 2];
    }
    free(tri);
    orc_mp *mp = orc_mp_create(A, t1, t2, t3, num);
    free(t1);
    free(t2);
    free(t3);
    /* double costs of the merged edge list: A's own edges keep theirs, the
     * added triangle chords start at 0 */
    mp64_t d;
    d.cost = NEW(double, mp->E + 1);
    d.c12 = (double *)xcalloc((size_t)mp->T + 1, sizeof(double));
    d.c13 = (double *)xcalloc((size_t)mp->T + 1, sizeof(double));
    d.c23 = (double *)xcalloc((size_t)mp->T + 1, sizeof(double));
    d.diff = NEW(double, 3 * mp->T + 1);
    int32_t nmax = graph_max_dim(A);
    for (int64_t e = 0; e < mp->E; ++e) nmax = imax(nmax, mp->col[e] + 1);
    int32_t *aoff = NEW(int32_t, nmax + 2);
    orc_compute_offsets(A->row, A->n, nmax, aoff);
    for (int64_t e = 0; e < mp->E; ++e) {
        int64_t x = mp->row[e] < nmax ? edge_find(aoff, A->col, mp->row[e], mp->col[e]) : -1;
        d.cost[e] = x >= 0 ? cd[x] : 0.0;
    }
    free(aoff);
    double prev = 0.0;
    for (int32_t it = 0; it < num_iter; ++it) {
        double lb = mp64_lower_bound(mp, &d);
        if (it > 0 && (lb - prev) < 1e-3) break;
        mp64_iteration(mp, &d);
        prev = lb;
    }
    double fin = mp64_lower_bound(mp, &d);
    float *cf = NEW(float, mp->E + 1);
    for (int64_t e = 0; e < mp->E; ++e) cf[e] = (float)d.cost[e];
    orc_graph *B = orc_graph_from_sorted(mp->E, mp->row, mp->col, cf);
    orc_mp_free(mp);
    free(cf);
    free(d.c12);
    free(d.c13);
    free(d.c23);
    free(d.diff);
    orc_graph_free(A);
    free(*pcd);
    *pA = B;
    *pcd = d.cost;
    return fin;
}

int orc_dual_lb_f64(int64_t n, const int32_t *i, const int32_t *j, const float *c, int32_t max_len, int32_t num_iter,
                    float tri_factor, int32_t num_outer, float tol, double *lb)
{
    orc_graph *A = orc_graph_from_edges(n, i, j, c);
    double *cd = NEW(double, A->n + 1);
    for (int64_t e = 0; e < A->n; ++e) cd[e] = (double)A->cost[e];
    double fin = 0.0, prev = 0.0;
    if (max_len < 3 || num_iter == 0 || num_outer == 0) {
        csum_acc acc;
        cacc_init(&acc);
        for (int64_t e = 0; e < A->n; ++e) cacc_push(&acc, cd[e] < 0.0 ? cd[e] : 0.0);
        fin = cacc_finish(&acc);
    } else {
        int64_t nt = 0;
        for (int32_t o = 0; o < num_outer; ++o) {
            for (int32_t cl = 3; cl <= max_len; ++cl)
                fin = dual_update_cycle_length_f64(&A, &cd, cl, num_iter, tri_factor, tol, &nt);
            if (nt == 0 || (o > 0 && (fin - prev) < 1e-3)) break;
            prev = fin;
        }
    }
    free(cd);
    orc_graph_free(A);
    *lb = fin;
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* options presets (include/multicut_solver_options.h:4-53)                  */
/* ------------------------------------------------------------------------ */
void orc_opts_init(orc_opts *o, const char *mode)
{
    o->max_cycle_length_lb = 5;
    o->num_dual_itr_lb = 10;
    o->max_cycle_length_primal = 3;
    o->num_dual_itr_primal = 5;
    o->num_outer_itr_dual = 1;
    o->mean_multiplier_mm = 0.05f;
    o->matching_thresh_crossover_ratio = 0.05f;
    o->tri_memory_factor = 2.0f;
    o->only_compute_lb = 0;
    o->max_time_sec = -1;
    o->dump_timeline = 0;
    o->verbose = 0;
    o->sanitize_graph = 0;
    o->woc_pentagons = 0;
    if (!mode) return;
    if (strcmp(mode, "P") == 0) {
        o->max_cycle_length_lb = 0;
        o->num_dual_itr_lb = 0;
        o->max_cycle_length_primal = 0;
        o->num_dual_itr_primal = 0;
    } else if (strcmp(mode, "PD+") == 0) {
        o->max_cycle_length_lb = 5;
        o->num_dual_itr_lb = 10;
        o->max_cycle_length_primal = 5;
        o->num_dual_itr_primal = 10;
    } else if (strcmp(mode, "D") == 0) {
        o->max_cycle_length_lb = 5;
        o->num_dual_itr_lb = 10;
        o->num_outer_itr_dual = 5;
        o->only_compute_lb = 1;
    }
}

/* ------------------------------------------------------------------------ */
/* sanitize (include/rama_utils.h:429-466)                                   */
/* ------------------------------------------------------------------------ */
int orc_sanitize(int64_t n, int32_t *i, int32_t *j, float *c, int64_t *n_out, int32_t *ids_mapping, int64_t ids_cap,
                 int64_t *ids_size)
{
    uint64_t *keys = NEW(uint64_t, n);
    for (int64_t e = 0; e < n; ++e) keys[e] = pack2(imin(i[e], j[e]), imax(i[e], j[e]));
    int64_t *perm = stable_order_u64(keys, n);
    int32_t *ni = NEW(int32_t, n), *nj = NEW(int32_t, n);
    float *nc = NEW(float, n);
    int64_t u = 0;
    for (int64_t k = 0; k < n; ++k) {
        int64_t p = perm[k];
        if (k > 0 && keys[p] == keys[perm[k - 1]]) continue; /* unique_by_key keeps the first */
        ni[u] = (int32_t)(keys[p] >> 32);
        nj[u] = (int32_t)(keys[p] & 0xFFFFFFFFu);
        nc[u] = c[p];
        u++;
    }
    int32_t mx = -1;
    for (int64_t e = 0; e < u; ++e) mx = imax(mx, nj[e]);
    int64_t size = (int64_t)mx + 1;
    if (size > ids_cap) {
        free(keys);
        free(perm);
        free(ni);
        free(nj);
        free(nc);
        return ORC_ERR_INVALID_ARG;
    }
    memset(ids_mapping, 0, sizeof(int32_t) * (size_t)size);
    for (int64_t e = 0; e < u; ++e) ids_mapping[ni[e]] = ids_mapping[nj[e]] = 1;
    int32_t run = 0;
    for (int64_t v = 0; v < size; ++v) {
        int32_t m = ids_mapping[v];
        ids_mapping[v] = run;
        run += m;
    }
    for (int64_t e = 0; e < u; ++e) {
        i[e] = ids_mapping[ni[e]];
        j[e] = ids_mapping[nj[e]];
        c[e] = nc[e];
    }
    *n_out = u;
    *ids_size = size;
    free(keys);
    free(perm);
    free(ni);
    free(nj);
    free(nc);
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* full solve (src/rama_cuda.cu:64-212)                                      */
/* ------------------------------------------------------------------------ */
static double now_sec(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

int orc_solve(int64_t n, const int32_t *i, const int32_t *j, const float *c, const orc_opts *o, int32_t *labels_out,
              int64_t labels_cap, int64_t *num_labels, double *lb_out, orc_stats *stats)
{
    orc_stats st;
    memset(&st, 0, sizeof(st));
    *num_labels = 0;
    *lb_out = 0.0;
    for (int64_t e = 0; e < n; ++e)
        if (i[e] < 0 || j[e] < 0 || i[e] == j[e]) {
            st.status = ORC_ERR_INVALID_ARG;
            if (stats) *stats = st;
            return ORC_ERR_INVALID_ARG;
        }
    if (n == 0) {
        if (stats) *stats = st;
        return ORC_OK;
    }
    int32_t *ii = NEW(int32_t, n), *jj = NEW(int32_t, n);
    float *cc = NEW(float, n);
    memcpy(ii, i, 4 * (size_t)n);
    memcpy(jj, j, 4 * (size_t)n);
    memcpy(cc, c, 4 * (size_t)n);
    int32_t *ids_mapping = NULL;
    int64_t ids_size = 0;
    if (o->sanitize_graph) {
        int32_t mx = 0;
        for (int64_t e = 0; e < n; ++e) mx = imax(mx, imax(i[e], j[e]));
        ids_mapping = NEW(int32_t, (int64_t)mx + 1);
        orc_sanitize(n, ii, jj, cc, &n, ids_mapping, (int64_t)mx + 1, &ids_size);
    }
    double t0 = now_sec();
    g_truncations = 0;
    orc_graph *A = orc_graph_from_edges(n, ii, jj, cc);
    free(ii);
    free(jj);
    free(cc);
    int64_t ntri = 0;
    double lb = orc_dual_solver(&A, o->max_cycle_length_lb, o->num_dual_itr_lb, o->tri_memory_factor,
                                o->num_outer_itr_dual, 1e-4f, &ntri);
    st.triangles_initial = ntri;
    *lb_out = lb;
    int32_t N0 = graph_max_dim(A);
    int32_t *node_mapping = NEW(int32_t, N0);
    for (int32_t v = 0; v < N0; ++v) node_mapping[v] = v;
    int rc = ORC_OK;
    if (!o->only_compute_lb) {
        int try_mm = !(o->matching_thresh_crossover_ratio > 1.0f);
        int32_t *map = NULL;
        for (int64_t iter = 0; A->n > 0; ++iter) {
            if (iter > 0)
                orc_dual_solver(&A, o->max_cycle_length_primal, o->num_dual_itr_primal, 1.0f, 1, 1e-4f, NULL);
            int64_t msize = 0;
            int32_t nr = 0;
            free(map);
            map = NEW(int32_t, graph_max_dim(A) + 1);
            if (try_mm) {
                orc_matching(A, o->mean_multiplier_mm, map, &msize, &nr);
                st.matching_rounds++;
                if ((float)nr < (float)A->rows * o->matching_thresh_crossover_ratio) try_mm = 0;
            } else {
                orc_woc_ex(A, map, &msize, &nr, o->woc_pentagons);
                st.mst_rounds++;
            }
            if (nr == 0) break;
            orc_graph *B = orc_contract(A, map, msize);
            if (orc_has_bad_contractions(B)) {
                orc_graph_free(B);
                rc = ORC_ERR_BAD_CONTRACTION;
                break;
            }
            orc_graph_free(A);
            A = B;
            orc_remove_diagonal(A);
            /* map_node_labels (src/rama_cuda.cu:32-52) */
            for (int32_t v = 0; v < N0; ++v)
                if (node_mapping[v] < msize) node_mapping[v] = map[node_mapping[v]];
            st.rounds++;
            if (o->max_time_sec >= 0 && (int64_t)(now_sec() - t0) > o->max_time_sec) break;
        }
        free(map);
        if (o->sanitize_graph) {
            /* desanitize_node_labels (include/rama_utils.h:468-493) */
            if (ids_size > labels_cap) rc = ORC_ERR_INVALID_ARG;
            else {
                for (int64_t v = 0; v < ids_size; ++v) {
                    int32_t cur = ids_mapping[v];
                    labels_out[v] = (v == ids_size - 1 || cur != ids_mapping[v + 1]) ? node_mapping[cur] : -1;
                }
                *num_labels = ids_size;
            }
        } else if (N0 > labels_cap)
            rc = ORC_ERR_INVALID_ARG;
        else {
            memcpy(labels_out, node_mapping, 4 * (size_t)N0);
            *num_labels = N0;
        }
    }
    free(ids_mapping);
    free(node_mapping);
    orc_graph_free(A);
    st.status = rc;
    st.truncations = g_truncations;
    if (stats) *stats = st;
    return rc;
}

/* objective (get_obj, include/rama_utils.h:192-205), CSUM */
double orc_objective(int64_t n, const int32_t *i, const int32_t *j, const float *c, const int32_t *labels)
{
    csum_acc a;
    cacc_init(&a);
    for (int64_t e = 0; e < n; ++e) cacc_push(&a, labels[i[e]] != labels[j[e]] ? (double)c[e] : 0.0);
    return cacc_finish(&a);
}
