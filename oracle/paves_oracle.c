/*
 * paves_oracle.c — CPU oracle for the PAVES GPU search path.
 *
 * TEST INFRASTRUCTURE ONLY. This file restates, in plain C, the reference
 * algorithms the GPU path must agree with. Only tests/, the package's
 * smoke() check and bench.py's cpu_baseline leg may load it, and only as
 * the checker; the product never calls it.
 *
 * Restated from the reference (paths within SakuraMarble/PAVES):
 *   pvo_pred_eval      extension/paves/src/engine/engine.cpp:397-431
 *                      (FvPred::eval_node) in the serialized node form of
 *                      gpu_engine.cu:238-279 (fv_eval_dev)
 *   pvo_exact_topk     engine.cpp:1082-1132 (BruteCursor::compute): exact
 *                      filtered scan, results ordered by (distance, id);
 *                      distances are accumulated in FP64 (exact for the
 *                      integer-valued data of the benchmark configurations)
 *                      and also reported as a sequential FP32 sum
 *   pvo_graph_entry    engine.cpp:1539-1559 (fv_index_graph_entry)
 *   pvo_hnsw_search    engine.cpp:1661-1713 (HnswCursor::run_phase) for one
 *                      phase at fixed ef, started from a level-0 entry
 *
 * Parity pinning: tests/golden/ holds outputs of the reference engine built
 * from its own sources (oracle/Makefile -> oracle/_ref/), and
 * tests/test_oracle_golden.py checks this file against them.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int32_t kind, col, op, nchildren, child0, nvalues, val0, pad;
    double value;
} PvoNode; /* byte-compatible with FvGpuPredNode */

enum { CMP_LT, CMP_LE, CMP_EQ, CMP_GE, CMP_GT, CMP_NE };
enum { NODE_CMP, NODE_IN, NODE_AND, NODE_OR, NODE_NOT };

int pvo_pred_eval(const PvoNode *nodes, const int32_t *children, const double *invals,
                  const double *cols, uint64_t count, int32_t ni, uint64_t row) {
    const PvoNode *n = &nodes[ni];
    switch (n->kind) {
        case NODE_CMP: {
            double v = cols[(uint64_t)n->col * count + row];
            switch (n->op) {
                case CMP_LT: return v < n->value;
                case CMP_LE: return v <= n->value;
                case CMP_EQ: return v == n->value;
                case CMP_GE: return v >= n->value;
                case CMP_GT: return v > n->value;
                case CMP_NE: return v == v && v != n->value;
            }
            return 0;
        }
        case NODE_IN: {
            double v = cols[(uint64_t)n->col * count + row];
            for (int i = 0; i < n->nvalues; i++)
                if (v == invals[n->val0 + i]) return 1;
            return 0;
        }
        case NODE_AND:
            for (int i = 0; i < n->nchildren; i++)
                if (!pvo_pred_eval(nodes, children, invals, cols, count,
                                   children[n->child0 + i], row))
                    return 0;
            return 1;
        case NODE_OR:
            for (int i = 0; i < n->nchildren; i++)
                if (pvo_pred_eval(nodes, children, invals, cols, count,
                                  children[n->child0 + i], row))
                    return 1;
            return 0;
        case NODE_NOT:
            return !pvo_pred_eval(nodes, children, invals, cols, count,
                                  children[n->child0], row);
    }
    return 0;
}

/* Bitmap of one predicate over all rows (u32 words, bit r%32 of word r/32). */
void pvo_pred_bitmap(const PvoNode *nodes, const int32_t *children, const double *invals,
                     const double *cols, uint64_t count, int32_t root, uint32_t *words,
                     uint64_t *npass) {
    uint64_t nw = (count + 31) / 32, np = 0;
    memset(words, 0, nw * 4);
    for (uint64_t r = 0; r < count; r++) {
        if (root < 0 || pvo_pred_eval(nodes, children, invals, cols, count, root, r)) {
            words[r >> 5] |= 1u << (r & 31);
            np++;
        }
    }
    *npass = np;
}

/* (distance, id) max-heap of capacity k, top = worst */
typedef struct { double d; uint32_t id; float d32; } Ent;
static int worse(const Ent *a, const Ent *b) {
    return a->d > b->d || (a->d == b->d && a->id > b->id);
}
static void sift_down(Ent *h, int n, int i) {
    for (;;) {
        int l = 2 * i + 1, r = l + 1, m = i;
        if (l < n && worse(&h[l], &h[m])) m = l;
        if (r < n && worse(&h[r], &h[m])) m = r;
        if (m == i) return;
        Ent t = h[i]; h[i] = h[m]; h[m] = t;
        i = m;
    }
}
static void sift_up(Ent *h, int i) {
    while (i) {
        int p = (i - 1) / 2;
        if (!worse(&h[i], &h[p])) return;
        Ent t = h[i]; h[i] = h[p]; h[p] = t;
        i = p;
    }
}
static int cmp_ent(const void *a, const void *b) {
    const Ent *x = a, *y = b;
    if (x->d < y->d) return -1;
    if (x->d > y->d) return 1;
    return x->id < y->id ? -1 : x->id > y->id;
}

/*
 * Exact filtered top-k for nq queries. roots[q] is the query's predicate
 * root (-1 = none). Outputs per query: ids/d64/d32 [q*k ..] ascending by
 * (d64, id), cnt[q] = min(k, passing), passing[q] = rows satisfying the
 * predicate.
 */
typedef struct {
    const float *vecs; uint64_t count; int dim; const float *queries; int nq;
    const int32_t *roots; const PvoNode *nodes; const int32_t *children;
    const double *invals; const double *cols; int k; uint32_t *ids; double *d64;
    float *d32; uint32_t *cnt; uint64_t *passing; int next; pthread_mutex_t mu;
} TopkJob;

static void topk_one(TopkJob *J, int q) {
    const int k = J->k, dim = J->dim;
    Ent *h = (Ent *)malloc(sizeof(Ent) * (size_t)(k > 0 ? k : 1));
    int n = 0;
    uint64_t np = 0;
    const float *qv = J->queries + (uint64_t)q * dim;
    for (uint64_t r = 0; r < J->count; r++) {
        if (J->roots[q] >= 0 &&
            !pvo_pred_eval(J->nodes, J->children, J->invals, J->cols, J->count, J->roots[q], r))
            continue;
        np++;
        const float *x = J->vecs + r * (uint64_t)dim;
        double s = 0.0;
        float s32 = 0.f;
        for (int j = 0; j < dim; j++) {
            double t = (double)x[j] - (double)qv[j];
            s += t * t;
            float t32 = x[j] - qv[j];
            s32 += t32 * t32;
        }
        Ent e = {s, (uint32_t)r, s32};
        if (n < k) {
            h[n] = e;
            sift_up(h, n);
            n++;
        } else if (k > 0 && worse(&h[0], &e)) {
            h[0] = e;
            sift_down(h, n, 0);
        }
    }
    qsort(h, n, sizeof(Ent), cmp_ent);
    for (int i = 0; i < n; i++) {
        J->ids[(uint64_t)q * k + i] = h[i].id;
        J->d64[(uint64_t)q * k + i] = h[i].d;
        J->d32[(uint64_t)q * k + i] = h[i].d32;
    }
    J->cnt[q] = (uint32_t)n;
    J->passing[q] = np;
    free(h);
}

static void *topk_worker(void *arg) {
    TopkJob *J = (TopkJob *)arg;
    for (;;) {
        pthread_mutex_lock(&J->mu);
        int q = J->next++;
        pthread_mutex_unlock(&J->mu);
        if (q >= J->nq) return NULL;
        topk_one(J, q);
    }
}

/*
 * Exact filtered top-k for nq queries on `threads` threads. roots[q] is the
 * query's predicate root (-1 = none). Outputs per query: ids/d64/d32
 * [q*k ..] ascending by (d64, id), cnt[q] = min(k, passing), passing[q] =
 * rows satisfying the predicate.
 */
void pvo_exact_topk(const float *vecs, uint64_t count, int dim, const float *queries, int nq,
                    const int32_t *roots, const PvoNode *nodes, const int32_t *children,
                    const double *invals, const double *cols, int k, uint32_t *ids,
                    double *d64, float *d32, uint32_t *cnt, uint64_t *passing, int threads) {
    TopkJob J = {vecs, count, dim, queries, nq, roots, nodes, children, invals, cols,
                 k, ids, d64, d32, cnt, passing, 0, PTHREAD_MUTEX_INITIALIZER};
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t th[256];
    for (int t = 1; t < threads; t++) pthread_create(&th[t], NULL, topk_worker, &J);
    topk_worker(&J);
    for (int t = 1; t < threads; t++) pthread_join(th[t], NULL);
}

static float l2f(const float *a, const float *b, int dim) {
    float s = 0.f;
    for (int j = 0; j < dim; j++) {
        float t = a[j] - b[j];
        s += t * t;
    }
    return s;
}

/* Greedy descent through the upper layers (engine.cpp:1539-1559). upper
 * lists are slabs of (M+1) u32 per level: [cnt, neighbours...]. */
uint32_t pvo_graph_entry(const float *vecs, int dim, const uint64_t *upper_offs,
                         const uint32_t *upper, uint32_t M, int max_level, uint64_t entry,
                         const float *q) {
    uint64_t ep = entry;
    for (int lc = max_level; lc >= 1; lc--) {
        float d = l2f(q, vecs + ep * dim, dim);
        int changed = 1;
        while (changed) {
            changed = 0;
            const uint32_t *lst = upper + upper_offs[ep] + (uint64_t)(lc - 1) * (M + 1);
            uint32_t c = lst[0];
            for (uint32_t i = 0; i < c; i++) {
                float nd = l2f(q, vecs + (uint64_t)lst[1 + i] * dim, dim);
                if (nd < d) {
                    d = nd;
                    ep = lst[1 + i];
                    changed = 1;
                }
            }
        }
    }
    return (uint32_t)ep;
}

/* binary heaps over (float d, u32 id) pairs, lexicographic like std::pair */
typedef struct { float d; uint32_t id; } Pr;
static int pr_lt(Pr a, Pr b) { return a.d < b.d || (a.d == b.d && a.id < b.id); }
typedef struct { Pr *a; int n, cap; int max; } Heap; /* max=1: max-heap */
static int hbefore(const Heap *h, Pr x, Pr y) { return h->max ? pr_lt(y, x) : pr_lt(x, y); }
static void hpush(Heap *h, Pr x) {
    if (h->n == h->cap) {
        h->cap = h->cap ? 2 * h->cap : 64;
        h->a = (Pr *)realloc(h->a, sizeof(Pr) * h->cap);
    }
    int i = h->n++;
    h->a[i] = x;
    while (i) {
        int p = (i - 1) / 2;
        if (!hbefore(h, h->a[i], h->a[p])) break;
        Pr t = h->a[i]; h->a[i] = h->a[p]; h->a[p] = t;
        i = p;
    }
}
static void hpop(Heap *h) {
    h->a[0] = h->a[--h->n];
    int i = 0;
    for (;;) {
        int l = 2 * i + 1, r = l + 1, m = i;
        if (l < h->n && hbefore(h, h->a[l], h->a[m])) m = l;
        if (r < h->n && hbefore(h, h->a[r], h->a[m])) m = r;
        if (m == i) break;
        Pr t = h->a[i]; h->a[i] = h->a[m]; h->a[m] = t;
        i = m;
    }
}
static int cmp_pr(const void *a, const void *b) {
    Pr x = *(const Pr *)a, y = *(const Pr *)b;
    return pr_lt(x, y) ? -1 : pr_lt(y, x) ? 1 : 0;
}

/*
 * One filtered level-0 beam-search phase at width ef from `entry`
 * (engine.cpp:1631-1713): traversal unrestricted, only passing nodes enter
 * the result heap. l0 rows: [cnt, neighbours...] of stride l0_stride.
 * Writes up to ef results ascending by (dist, id); returns the count.
 * *exhausted = frontier emptied or max_visited reached.
 */
int pvo_hnsw_search(const float *vecs, uint64_t count, int dim, const uint32_t *l0,
                    uint32_t l0_stride, uint32_t entry, const float *q, int root,
                    const PvoNode *nodes, const int32_t *children, const double *invals,
                    const double *cols, int ef, uint64_t max_visited, uint32_t *out_ids,
                    float *out_d, int *exhausted) {
    uint8_t *seen = (uint8_t *)calloc(count, 1);
    Heap cand = {0}, res = {0};
    cand.max = 0;
    res.max = 1;
    uint64_t visited = 1;
    int exh = 0;
    float epd = l2f(q, vecs + (uint64_t)entry * dim, dim);
    seen[entry] = 1;
    Pr e0 = {epd, entry};
    hpush(&cand, e0);
    if (root < 0 || pvo_pred_eval(nodes, children, invals, cols, count, root, entry))
        hpush(&res, e0);
    while (cand.n) {
        Pr c = cand.a[0];
        if (res.n >= ef && c.d > res.a[0].d) break;
        if (visited >= max_visited) {
            exh = 1;
            break;
        }
        hpop(&cand);
        const uint32_t *lst = l0 + (uint64_t)c.id * l0_stride;
        uint32_t cnt = lst[0];
        for (uint32_t i = 0; i < cnt; i++) {
            uint32_t n2 = lst[1 + i];
            if (seen[n2]) continue;
            seen[n2] = 1;
            visited++;
            float d = l2f(q, vecs + (uint64_t)n2 * dim, dim);
            if (res.n < ef || d < res.a[0].d) {
                Pr p = {d, n2};
                hpush(&cand, p);
                if (root < 0 || pvo_pred_eval(nodes, children, invals, cols, count, root, n2)) {
                    hpush(&res, p);
                    if (res.n > ef) hpop(&res);
                }
            }
        }
    }
    if (cand.n == 0) exh = 1;
    qsort(res.a, res.n, sizeof(Pr), cmp_pr);
    int n = res.n;
    for (int i = 0; i < n; i++) {
        out_ids[i] = res.a[i].id;
        out_d[i] = res.a[i].d;
    }
    free(cand.a);
    free(res.a);
    free(seen);
    *exhausted = exh;
    return n;
}
