/*
 * gaec.c -- sequential greedy additive edge contraction (GAEC) with union-find.
 *
 * TEST/BASELINE INFRASTRUCTURE ONLY.  The reference has no CPU solver; this is
 * the project-written single-thread CPU baseline that bench.py reports beside
 * the GPU numbers.  Algorithm: repeatedly contract the attractive edge of
 * largest cost; parallel edges of the merged cluster are summed.  A lazy max
 * heap holds (cost, endpoints, endpoint versions); an entry is stale once
 * either endpoint has been merged since it was pushed.
 */
#include "rama_oracle.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int32_t nb;
    float c;
} adj_t;

typedef struct {
    adj_t *a;
    int32_t n, cap;
} adjv_t;

typedef struct {
    float c;
    int32_t u, v, vu, vv;
} hent_t;

typedef struct {
    hent_t *h;
    int64_t n, cap;
} heap_t;

static void *gx(size_t n)
{
    void *p = malloc(n ? n : 1);
    if (!p) {
        fprintf(stderr, "gaec: out of memory\n");
        abort();
    }
    return p;
}

static void adj_push(adjv_t *v, int32_t nb, float c)
{
    if (v->n == v->cap) {
        int32_t nc = v->cap ? 2 * v->cap : 4;
        adj_t *na = (adj_t *)gx(sizeof(adj_t) * (size_t)nc);
        if (v->n) memcpy(na, v->a, sizeof(adj_t) * (size_t)v->n);
        free(v->a);
        v->a = na;
        v->cap = nc;
    }
    v->a[v->n].nb = nb;
    v->a[v->n].c = c;
    v->n++;
}

static void heap_push(heap_t *H, hent_t e)
{
    if (H->n == H->cap) {
        int64_t nc = H->cap ? 2 * H->cap : 1024;
        hent_t *nh = (hent_t *)gx(sizeof(hent_t) * (size_t)nc);
        if (H->n) memcpy(nh, H->h, sizeof(hent_t) * (size_t)H->n);
        free(H->h);
        H->h = nh;
        H->cap = nc;
    }
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

/* remove neighbour `nb` from v, returning its cost (0 if absent) */
static float adj_take(adjv_t *v, int32_t nb, int *found)
{
    for (int32_t k = 0; k < v->n; ++k)
        if (v->a[k].nb == nb) {
            float c = v->a[k].c;
            v->a[k] = v->a[--v->n];
            *found = 1;
            return c;
        }
    *found = 0;
    return 0.0f;
}

int orc_gaec(int64_t m, const int32_t *i, const int32_t *j, const float *c, int32_t N, int32_t *labels_out)
{
    adjv_t *adj = (adjv_t *)calloc((size_t)N + 1, sizeof(adjv_t));
    int32_t *ver = (int32_t *)calloc((size_t)N + 1, sizeof(int32_t));
    int32_t *parent = (int32_t *)gx(sizeof(int32_t) * ((size_t)N + 1));
    int32_t *pos = (int32_t *)gx(sizeof(int32_t) * ((size_t)N + 1));
    if (!adj || !ver) return ORC_ERR_OOM;
    for (int32_t v = 0; v < N; ++v) {
        parent[v] = v;
        pos[v] = -1;
    }
    /* build adjacency, summing duplicate edges */
    for (int64_t e = 0; e < m; ++e) {
        int32_t a = i[e], b = j[e];
        if (a == b) continue;
        int found = 0;
        for (int32_t k = 0; k < adj[a].n; ++k)
            if (adj[a].a[k].nb == b) {
                adj[a].a[k].c += c[e];
                found = 1;
                break;
            }
        if (found) {
            for (int32_t k = 0; k < adj[b].n; ++k)
                if (adj[b].a[k].nb == a) {
                    adj[b].a[k].c += c[e];
                    break;
                }
        } else {
            adj_push(&adj[a], b, c[e]);
            adj_push(&adj[b], a, c[e]);
        }
    }
    heap_t H = {NULL, 0, 0};
    for (int32_t a = 0; a < N; ++a)
        for (int32_t k = 0; k < adj[a].n; ++k) {
            int32_t b = adj[a].a[k].nb;
            if (a < b && adj[a].a[k].c > 0.0f) {
                hent_t h = {adj[a].a[k].c, a, b, 0, 0};
                heap_push(&H, h);
            }
        }
    while (H.n > 0) {
        hent_t h = heap_pop(&H);
        if (ver[h.u] != h.vu || ver[h.v] != h.vv || ver[h.u] < 0 || ver[h.v] < 0) continue;
        if (h.c <= 0.0f) break;
        int32_t a = h.u, b = h.v;
        if (adj[a].n < adj[b].n) {
            int32_t t = a;
            a = b;
            b = t;
        }
        /* merge b into a */
        int f;
        adj_take(&adj[a], b, &f);
        for (int32_t k = 0; k < adj[a].n; ++k) pos[adj[a].a[k].nb] = k;
        for (int32_t k = 0; k < adj[b].n; ++k) {
            int32_t w = adj[b].a[k].nb;
            float cw = adj[b].a[k].c;
            if (w == a) continue;
            int fw;
            adj_take(&adj[w], b, &fw);
            if (pos[w] >= 0) {
                adj[a].a[pos[w]].c += cw;
                for (int32_t q = 0; q < adj[w].n; ++q)
                    if (adj[w].a[q].nb == a) {
                        adj[w].a[q].c += cw;
                        break;
                    }
            } else {
                pos[w] = adj[a].n;
                adj_push(&adj[a], w, cw);
                adj_push(&adj[w], a, cw);
            }
        }
        for (int32_t k = 0; k < adj[a].n; ++k) pos[adj[a].a[k].nb] = -1;
        free(adj[b].a);
        adj[b].a = NULL;
        adj[b].n = adj[b].cap = 0;
        ver[b] = -1;
        ver[a]++;
        parent[b] = a;
        for (int32_t k = 0; k < adj[a].n; ++k) {
            int32_t w = adj[a].a[k].nb;
            if (adj[a].a[k].c > 0.0f) {
                hent_t e2;
                e2.c = adj[a].a[k].c;
                e2.u = a;
                e2.v = w;
                e2.vu = ver[a];
                e2.vv = ver[w];
                heap_push(&H, e2);
            }
        }
    }
    for (int32_t v = 0; v < N; ++v) {
        int32_t r = v;
        while (parent[r] != r) r = parent[r];
        labels_out[v] = r;
    }
    for (int32_t v = 0; v < N; ++v) free(adj[v].a);
    free(adj);
    free(ver);
    free(parent);
    free(pos);
    free(H.h);
    return ORC_OK;
}
