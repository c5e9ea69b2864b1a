/*
 * CPU oracle for the batched HNSW search -- TEST INFRASTRUCTURE ONLY.
 *
 * This file restates, in plain C, the reference's compiled search path so that the CUDA engine
 * can be checked against it bit for bit. Only the test suite, the smoke check and the CPU-baseline
 * leg of the benchmark load it; the product path never does.
 *
 * Followed functions (anamankev/hnsw-engine):
 *   dist_row          <- src/hnsw_engine/numba_engine.py:57-70   (_distance: float64 accumulation,
 *                        strictly sequential i = 0..d-1, separate multiply and add -- build with
 *                        -ffp-contract=off so no fused multiply-add changes the rounding)
 *   layer_links       <- numba_engine.py:73-86   (_links)
 *   search_layer      <- numba_engine.py:98-148  (_search_layer, Algorithm 2)
 *   search_layer0_f   <- numba_engine.py:151-198 (_search_layer0_filtered)
 *   oracle_search_batch <- numba_engine.py:422-503 (_search_batch, Algorithm 5), generalised to a
 *                        per-query ef array; each query gets max(ef[row], k) on layer 0 (:473, :487)
 *   oracle_rerank_batch <- numba_engine.py:506-530 (_rerank_batch)
 *
 * Heaps order (distance, id) pairs exactly as Python compares tuples (heapq in the reference):
 * candidates pop the minimum (d, id); results evict the maximum (d, id). No pair is ever pushed
 * twice (the visited set forbids it), so any correct priority queue reproduces heapq's order.
 * Counters are kept per query: [0] distance computations, [1] hops (node expansions), with the
 * reference's definitions (:130, :139, :451).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    double d;
    int64_t id;
} item_t;

static inline int item_lt(item_t a, item_t b) { return a.d < b.d || (a.d == b.d && a.id < b.id); }

/* ------------------------------------------------------------------ growable binary heaps */
typedef struct {
    item_t *v;
    int64_t n, cap;
    int max_heap; /* 0: root is the minimum (d, id); 1: root is the maximum */
} heap_t;

static inline int heap_before(const heap_t *h, item_t a, item_t b) {
    return h->max_heap ? item_lt(b, a) : item_lt(a, b);
}

static int heap_reserve(heap_t *h, int64_t want) {
    if (want <= h->cap) return 0;
    int64_t cap = h->cap ? h->cap : 64;
    while (cap < want) cap *= 2;
    item_t *nv = (item_t *)realloc(h->v, (size_t)cap * sizeof(item_t));
    if (!nv) return -1;
    h->v = nv;
    h->cap = cap;
    return 0;
}

static int heap_push(heap_t *h, item_t x) {
    if (heap_reserve(h, h->n + 1)) return -1;
    int64_t i = h->n++;
    while (i > 0) {
        int64_t p = (i - 1) / 2;
        if (!heap_before(h, x, h->v[p])) break;
        h->v[i] = h->v[p];
        i = p;
    }
    h->v[i] = x;
    return 0;
}

static item_t heap_pop(heap_t *h) {
    item_t top = h->v[0];
    item_t last = h->v[--h->n];
    int64_t i = 0, n = h->n;
    for (;;) {
        int64_t c = 2 * i + 1;
        if (c >= n) break;
        if (c + 1 < n && heap_before(h, h->v[c + 1], h->v[c])) c++;
        if (!heap_before(h, h->v[c], last)) break;
        h->v[i] = h->v[c];
        i = c;
    }
    if (n > 0) h->v[i] = last;
    return top;
}

static int cmp_item(const void *a, const void *b) {
    item_t x = *(const item_t *)a, y = *(const item_t *)b;
    if (item_lt(x, y)) return -1;
    if (item_lt(y, x)) return 1;
    return 0;
}

/* ------------------------------------------------------------------ graph and distances */
typedef struct {
    const void *vectors;
    int vec_u8; /* rows are uint8 codes instead of float32 */
    int64_t n;
    int32_t dim;
    int32_t metric; /* 0 l2, 1 ip, 2 cosine */
    const int32_t *links0;
    int32_t links0_stride;
    const int32_t *count0;
    const int32_t *links_up;
    int32_t links_up_stride;
    const int32_t *count_up;
    const int64_t *upper_offset;
} graph_t;

typedef struct {
    uint32_t *visited;
    uint32_t epoch;
    heap_t cand, res;
    int64_t dist, hops;
} worker_t;

/* Distance from float64 query q to stored row j (numba_engine.py:57-70). */
static double dist_row(const graph_t *g, const double *q, int64_t j) {
    double acc = 0.0;
    const int32_t dim = g->dim;
    if (g->vec_u8) {
        const uint8_t *x = (const uint8_t *)g->vectors + (size_t)j * (size_t)dim;
        if (g->metric == 0) {
            for (int32_t i = 0; i < dim; i++) {
                double t = (double)x[i] - q[i];
                acc += t * t;
            }
            return acc;
        }
        for (int32_t i = 0; i < dim; i++) acc += (double)x[i] * q[i];
    } else {
        const float *x = (const float *)g->vectors + (size_t)j * (size_t)dim;
        if (g->metric == 0) {
            for (int32_t i = 0; i < dim; i++) {
                double t = (double)x[i] - q[i];
                acc += t * t;
            }
            return acc;
        }
        for (int32_t i = 0; i < dim; i++) acc += (double)x[i] * q[i];
    }
    return g->metric == 1 ? -acc : 1.0 - acc;
}

static inline const int32_t *layer_links(const graph_t *g, int64_t node, int32_t layer,
                                         int32_t *count) {
    if (layer == 0) {
        *count = g->count0[node];
        return g->links0 + (size_t)node * (size_t)g->links0_stride;
    }
    int64_t row = g->upper_offset[node] + layer - 1;
    *count = g->count_up[row];
    return g->links_up + (size_t)row * (size_t)g->links_up_stride;
}

static uint32_t next_epoch(worker_t *w, int64_t n) { /* numba_engine.py:89-95 */
    w->epoch += 1;
    if (w->epoch >= 4294967295u) {
        memset(w->visited, 0, (size_t)n * sizeof(uint32_t));
        w->epoch = 1;
    }
    return w->epoch;
}

/* Sorted ascending copy of the results heap into out; returns the count. */
static int64_t drain_sorted(heap_t *res, item_t *out) {
    int64_t m = res->n;
    memcpy(out, res->v, (size_t)m * sizeof(item_t));
    qsort(out, (size_t)m, sizeof(item_t), cmp_item);
    return m;
}

/* Algorithm 2 (numba_engine.py:98-148). entry/out may alias; out needs room for ef items. */
static int search_layer(const graph_t *g, worker_t *w, const double *q, const item_t *entry,
                        int64_t n_entry, int64_t ef, int32_t layer, item_t *out, int64_t *n_out) {
    uint32_t epoch = next_epoch(w, g->n);
    w->cand.n = 0;
    w->res.n = 0;
    for (int64_t i = 0; i < n_entry; i++) {
        if (heap_push(&w->cand, entry[i]) || heap_push(&w->res, entry[i])) return -1;
    }
    while (w->res.n > ef) heap_pop(&w->res);
    for (int64_t i = 0; i < n_entry; i++) w->visited[entry[i].id] = epoch;

    while (w->cand.n > 0) {
        item_t c = heap_pop(&w->cand);
        if (c.d > w->res.v[0].d) break;
        w->hops += 1;
        int32_t cnt;
        const int32_t *nb = layer_links(g, c.id, layer, &cnt);
        double worst = w->res.v[0].d;
        for (int32_t idx = 0; idx < cnt; idx++) {
            int64_t e = nb[idx];
            if (w->visited[e] == epoch) continue;
            w->visited[e] = epoch;
            double d = dist_row(g, q, e);
            w->dist += 1;
            if (w->res.n < ef || d < worst) {
                item_t x = {d, e};
                if (heap_push(&w->cand, x) || heap_push(&w->res, x)) return -1;
                if (w->res.n > ef) heap_pop(&w->res);
                worst = w->res.v[0].d;
            }
        }
    }
    *n_out = drain_sorted(&w->res, out);
    return 0;
}

/* Filtered layer 0 (numba_engine.py:151-198): results hold allowed nodes only. */
static int search_layer0_f(const graph_t *g, worker_t *w, const double *q, const item_t *entry,
                           int64_t n_entry, int64_t ef, const uint8_t *allowed, item_t *out,
                           int64_t *n_out) {
    uint32_t epoch = next_epoch(w, g->n);
    w->cand.n = 0;
    w->res.n = 0;
    for (int64_t i = 0; i < n_entry; i++) {
        if (heap_push(&w->cand, entry[i])) return -1;
        if (allowed[entry[i].id] && heap_push(&w->res, entry[i])) return -1;
    }
    while (w->res.n > ef) heap_pop(&w->res);
    for (int64_t i = 0; i < n_entry; i++) w->visited[entry[i].id] = epoch;

    while (w->cand.n > 0) {
        item_t c = heap_pop(&w->cand);
        if (w->res.n == ef && c.d > w->res.v[0].d) break;
        w->hops += 1;
        double worst = w->res.n > 0 ? w->res.v[0].d : INFINITY;
        int32_t cnt = g->count0[c.id];
        const int32_t *nb = g->links0 + (size_t)c.id * (size_t)g->links0_stride;
        for (int32_t idx = 0; idx < cnt; idx++) {
            int64_t e = nb[idx];
            if (w->visited[e] == epoch) continue;
            w->visited[e] = epoch;
            double d = dist_row(g, q, e);
            w->dist += 1;
            if (w->res.n < ef || d < worst) {
                item_t x = {d, e};
                if (heap_push(&w->cand, x)) return -1;
                if (allowed[e]) {
                    if (heap_push(&w->res, x)) return -1;
                    if (w->res.n > ef) heap_pop(&w->res);
                    worst = w->res.v[0].d;
                }
            }
        }
    }
    *n_out = drain_sorted(&w->res, out);
    return 0;
}

/*
 * Algorithm 5 for every query (numba_engine.py:422-503).
 *   queries: (nq, dim) float32 (q_f64 = 0) or float64 (q_f64 = 1; the code-space queries of
 *            QuantizedIndex, numba_engine.py:674-701)
 *   ef:      (nq,) raw efSearch per query; layer 0 uses max(ef[row], k)
 *   allowed: NULL (unfiltered) or (n,) bytes, nonzero = allowed
 *   out_counters: (nq, 2) distance computations and hops of each query
 * Returns 0, or -1 if memory ran out.
 */
int oracle_search_batch(const void *queries, int32_t q_f64, int64_t nq, int32_t dim, int32_t k,
                        const int32_t *ef, int32_t metric, const void *vectors, int32_t vec_u8,
                        int64_t n, const int32_t *links0, int32_t links0_stride,
                        const int32_t *count0, const int32_t *links_up, int32_t links_up_stride,
                        const int32_t *count_up, const int64_t *upper_offset, int64_t entry_point,
                        int32_t max_level, const uint8_t *allowed, int64_t *out_ids,
                        double *out_dists, int64_t *out_counters, int32_t n_threads) {
    graph_t g = {vectors, vec_u8, n, dim, metric, links0, links0_stride, count0,
                 links_up, links_up_stride, count_up, upper_offset};
    int failed = 0;
    if (n_threads < 1) n_threads = 1;
#pragma omp parallel num_threads(n_threads) reduction(| : failed)
    {
        worker_t w;
        memset(&w, 0, sizeof(w));
        w.visited = (uint32_t *)calloc((size_t)(n > 0 ? n : 1), sizeof(uint32_t));
        w.res.max_heap = 1;
        int64_t ef_cap = 1;
        for (int64_t r = 0; r < nq; r++) {
            int64_t e = ef[r] > k ? ef[r] : k;
            if (e > ef_cap) ef_cap = e;
        }
        item_t *found = (item_t *)malloc((size_t)ef_cap * sizeof(item_t));
        double *q = (double *)malloc((size_t)(dim > 0 ? dim : 1) * sizeof(double));
        if (!w.visited || !found || !q) failed = 1;
#pragma omp for schedule(dynamic, 16)
        for (int64_t row = 0; row < nq; row++) {
            if (failed) continue;
            if (q_f64) {
                memcpy(q, (const double *)queries + (size_t)row * dim, (size_t)dim * sizeof(double));
            } else {
                const float *qf = (const float *)queries + (size_t)row * dim;
                for (int32_t i = 0; i < dim; i++) q[i] = (double)qf[i];
            }
            w.dist = 0;
            w.hops = 0;
            item_t entry = {dist_row(&g, q, entry_point), entry_point};
            w.dist += 1;
            int64_t n_found = 1;
            found[0] = entry;
            for (int32_t layer = max_level; layer > 0; layer--) {
                if (search_layer(&g, &w, q, found, n_found, 1, layer, found, &n_found)) failed = 1;
            }
            int64_t ef_row = ef[row] > k ? ef[row] : k;
            int rc = allowed ? search_layer0_f(&g, &w, q, found, n_found, ef_row, allowed, found,
                                               &n_found)
                             : search_layer(&g, &w, q, found, n_found, ef_row, 0, found, &n_found);
            if (rc) failed = 1;
            for (int32_t i = 0; i < k; i++) {
                out_ids[row * k + i] = i < n_found ? found[i].id : -1;
                out_dists[row * k + i] = i < n_found ? found[i].d : INFINITY;
            }
            out_counters[2 * row] = w.dist;
            out_counters[2 * row + 1] = w.hops;
        }
        free(w.visited);
        free(w.cand.v);
        free(w.res.v);
        free(found);
        free(q);
    }
    return failed ? -1 : 0;
}

/*
 * Exact re-ranking (numba_engine.py:506-530): float64 distances from each float32 query to its
 * candidate ids (entries < 0 skipped), sorted by (distance, id), first k kept, padded -1 / inf.
 */
int oracle_rerank_batch(const float *queries, int64_t nq, int32_t dim, const float *vectors,
                        int64_t n, int32_t metric, const int64_t *candidates, int32_t n_cand,
                        int32_t k, int64_t *out_ids, double *out_dists, int32_t n_threads) {
    graph_t g;
    memset(&g, 0, sizeof(g));
    g.vectors = vectors;
    g.n = n;
    g.dim = dim;
    g.metric = metric;
    int failed = 0;
    if (n_threads < 1) n_threads = 1;
#pragma omp parallel num_threads(n_threads) reduction(| : failed)
    {
        item_t *scored = (item_t *)malloc((size_t)(n_cand > 0 ? n_cand : 1) * sizeof(item_t));
        double *q = (double *)malloc((size_t)(dim > 0 ? dim : 1) * sizeof(double));
        if (!scored || !q) failed = 1;
#pragma omp for schedule(static)
        for (int64_t row = 0; row < nq; row++) {
            if (failed) continue;
            for (int32_t i = 0; i < dim; i++) q[i] = (double)queries[row * dim + i];
            int64_t m = 0;
            for (int32_t j = 0; j < n_cand; j++) {
                int64_t e = candidates[row * n_cand + j];
                if (e >= 0) {
                    scored[m].d = dist_row(&g, q, e);
                    scored[m].id = e;
                    m++;
                }
            }
            qsort(scored, (size_t)m, sizeof(item_t), cmp_item);
            for (int32_t i = 0; i < k; i++) {
                out_ids[row * k + i] = i < m ? scored[i].id : -1;
                out_dists[row * k + i] = i < m ? scored[i].d : INFINITY;
            }
        }
        free(scored);
        free(q);
    }
    return failed ? -1 : 0;
}

/* Number of threads an unbounded OpenMP region would use (for reporting). */
int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
