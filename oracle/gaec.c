/*
 * gaec.c -- sequential greedy additive edge contraction (GAEC) with union-find.
 *
 * TEST/BASELINE INFRASTRUCTURE ONLY.  The reference has no CPU solver; this is
 * the project-written single-thread CPU baseline that bench.py reports beside
 * the GPU numbers.  Algorithm: repeatedly contract the attractive edge of
 * largest cost; the edges of the merged cluster to a common neighbour are
 * summed.  Edge costs live in one open-addressing hash table keyed by the
 * (smaller, larger) cluster pair; each cluster keeps a list of neighbours
 * that may hold stale entries (checked against the table).  The smaller
 * cluster is merged into the larger, so the work is O(E log V) table
 * operations.  A lazy max-heap holds (cost, endpoints); an entry is stale if
 * an endpoint was merged away or the pair's cost changed.
 */
#include "rama_oracle.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int32_t *a;
    int32_t n, cap;
} ivec_t;

typedef struct {
    float c;
    int32_t u, v;
} hent_t;

typedef struct {
    hent_t *h;
    int64_t n, cap;
} heap_t;

typedef struct {
    uint64_t *key; /* 0 = empty, 1 = deleted, else pair + 2 */
    float *val;
    uint64_t mask;
} table_t;

static void *gx(size_t n)
{
    void *p = malloc(n ? n : 1);
    if (!p) {
        fprintf(stderr, "gaec: out of memory\n");
        abort();
    }
    return p;
}

static void ivec_push(ivec_t *v, int32_t x)
{
    if (v->n == v->cap) {
        int32_t nc = v->cap ? 2 * v->cap : 4;
        int32_t *na = (int32_t *)gx(sizeof(int32_t) * (size_t)nc);
        if (v->n) memcpy(na, v->a, sizeof(int32_t) * (size_t)v->n);
        free(v->a);
        v->a = na;
        v->cap = nc;
    }
    v->a[v->n++] = x;
}

static void heap_push(heap_t *H, float c, int32_t u, int32_t v)
{
    if (H->n == H->cap) {
        int64_t nc = H->cap ? 2 * H->cap : 1024;
        hent_t *nh = (hent_t *)gx(sizeof(hent_t) * (size_t)nc);
        if (H->n) memcpy(nh, H->h, sizeof(hent_t) * (size_t)H->n);
        free(H->h);
        H->h = nh;
        H->cap = nc;
    }
    hent_t e = {c, u, v};
    int64_t k = H->n++;
    while (k > 0) {
        int64_t p = (k - 1) / 2;
        if (H->h[p].c >= e.c) break;
        H->h[k] = H->h[p];
        k = p;
    }
    H->h[k] = e;
}

static hent_t heap_pop(heap_t *H)
{
    hent_t top = H->h[0];
    hent_t last = H->h[--H->n];
    int64_t k = 0;
    for (;;) {
        int64_t l = 2 * k + 1, r = l + 1, m = k;
        float mc = last.c;
        if (l < H->n && H->h[l].c > mc) {
            m = l;
            mc = H->h[l].c;
        }
        if (r < H->n && H->h[r].c > mc) m = r;
        if (m == k) break;
        H->h[k] = H->h[m];
        k = m;
    }
    if (H->n) H->h[k] = last;
    return top;
}

static inline uint64_t pair_key(int32_t a, int32_t b)
{
    int32_t lo = a < b ? a : b, hi = a < b ? b : a;
    return (((uint64_t)(uint32_t)lo << 32) | (uint32_t)hi) + 2;
}

static inline uint64_t mix(uint64_t x)
{
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdULL;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ULL;
    x ^= x >> 33;
    return x;
}

/* returns the slot holding key, or -1 */
static int64_t tab_find(const table_t *T, uint64_t key)
{
    uint64_t s = mix(key) & T->mask;
    for (;;) {
        uint64_t k = T->key[s];
        if (k == key) return (int64_t)s;
        if (k == 0) return -1;
        s = (s + 1) & T->mask;
    }
}

/* adds c to key (inserting it); returns 1 if the key was new */
static int tab_add(table_t *T, uint64_t key, float c, float *out)
{
    uint64_t s = mix(key) & T->mask;
    int64_t tomb = -1;
    for (;;) {
        uint64_t k = T->key[s];
        if (k == key) {
            T->val[s] += c;
            *out = T->val[s];
            return 0;
        }
        if (k == 1 && tomb < 0) tomb = (int64_t)s;
        if (k == 0) {
            uint64_t d = tomb >= 0 ? (uint64_t)tomb : s;
            T->key[d] = key;
            T->val[d] = c;
            *out = c;
            return 1;
        }
        s = (s + 1) & T->mask;
    }
}

int orc_gaec(int64_t m, const int32_t *i, const int32_t *j, const float *c, int32_t N, int32_t *labels_out)
{
    uint64_t cap = 16;
    while (cap < (uint64_t)(4 * m + 16)) cap <<= 1;
    table_t T;
    T.key = (uint64_t *)calloc(cap, sizeof(uint64_t));
    T.val = (float *)gx(sizeof(float) * cap);
    T.mask = cap - 1;
    ivec_t *adj = (ivec_t *)calloc((size_t)N + 1, sizeof(ivec_t));
    int32_t *parent = (int32_t *)gx(sizeof(int32_t) * ((size_t)N + 1));
    uint8_t *dead = (uint8_t *)calloc((size_t)N + 1, 1);
    if (!T.key || !adj || !dead) return ORC_ERR_OOM;
    for (int32_t v = 0; v < N; ++v) parent[v] = v;
    for (int64_t e = 0; e < m; ++e) {
        if (i[e] == j[e]) continue;
        float nv;
        if (tab_add(&T, pair_key(i[e], j[e]), c[e], &nv)) {
            ivec_push(&adj[i[e]], j[e]);
            ivec_push(&adj[j[e]], i[e]);
        }
    }
    heap_t H = {NULL, 0, 0};
    for (uint64_t s = 0; s < cap; ++s)
        if (T.key[s] > 1 && T.val[s] > 0.0f) {
            uint64_t k = T.key[s] - 2;
            heap_push(&H, T.val[s], (int32_t)(k >> 32), (int32_t)(k & 0xffffffffu));
        }
    while (H.n > 0) {
        hent_t h = heap_pop(&H);
        if (h.c <= 0.0f) break;
        if (dead[h.u] || dead[h.v]) continue;
        int64_t s = tab_find(&T, pair_key(h.u, h.v));
        if (s < 0 || T.val[s] != h.c) continue;
        int32_t a = h.u, b = h.v;
        if (adj[a].n < adj[b].n) {
            int32_t t = a;
            a = b;
            b = t;
        }
        /* merge b into a */
        T.key[s] = 1;
        for (int32_t q = 0; q < adj[b].n; ++q) {
            int32_t w = adj[b].a[q];
            if (w == a || dead[w]) continue;
            int64_t sb = tab_find(&T, pair_key(b, w));
            if (sb < 0) continue; /* stale duplicate */
            float cw = T.val[sb];
            T.key[sb] = 1;
            float nv;
            if (tab_add(&T, pair_key(a, w), cw, &nv)) {
                ivec_push(&adj[a], w);
                ivec_push(&adj[w], a);
            }
            if (nv > 0.0f) heap_push(&H, nv, a, w);
        }
        free(adj[b].a);
        adj[b].a = NULL;
        adj[b].n = adj[b].cap = 0;
        dead[b] = 1;
        parent[b] = a;
    }
    for (int32_t v = 0; v < N; ++v) {
        int32_t r = v;
        while (parent[r] != r) r = parent[r];
        labels_out[v] = r;
    }
    for (int32_t v = 0; v < N; ++v) free(adj[v].a);
    free(adj);
    free(parent);
    free(dead);
    free(T.key);
    free(T.val);
    free(H.h);
    return ORC_OK;
}
