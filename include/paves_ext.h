/*
 * paves_ext.h — additions to the drop-in ABI (libpaves_gpu.so).
 *
 * None of these replace a reference entry point; they sit beside the
 * gpu_engine.h surface declared in paves_gpu.h:
 *   - host-side predicate validation (no device needed),
 *   - prepared batches whose inputs stay resident in device memory, for
 *     callers that issue the same batch repeatedly or that measure the
 *     device-side cost alone,
 *   - per-stage device timings of the last call.
 * Same conventions as paves_gpu.h: plain C, host pointers and sizes, 0 or
 * -1 + errbuf.
 */
#ifndef PAVES_B200_EXT_H
#define PAVES_B200_EXT_H

#include "paves_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Scan modes of a prepared batch. */
#define PV_MODE_EXACT 0 /* exact FP32 scan */
#define PV_MODE_LOW 1   /* reduced-precision (index precision) scan + FP32 re-rank */

/* Validates and compiles the predicates of a batch on the host exactly as
 * fv_gpu_brute_batch does, without touching a device. *nprog receives the
 * number of distinct predicates. Returns 0 or -1 + errbuf. */
int pv_pred_check(int nq, const FvGpuQueryDesc *qd, const FvGpuPredNode *nodes, int nnodes,
                  const int32_t *children, int nchildren, const double *invals, int ninvals,
                  int ncols, int *nprog, char *errbuf, size_t errlen);

typedef struct PvBatch PvBatch;

/* Compiles the batch's predicates and copies queries + predicate programs
 * to the device once. topb as in fv_gpu_brute_batch (nq may exceed
 * FV_GPU_MAX_BATCH, up to 65536). */
PvBatch *pv_batch_create(FvGpuIndex *g, int nq, const float *queries,
                         const FvGpuQueryDesc *qd, const FvGpuPredNode *nodes, int nnodes,
                         const int32_t *children, int nchildren, const double *invals,
                         int ninvals, uint32_t topb, int mode, char *errbuf, size_t errlen);

/* Runs the device-side work of the batch (bitmaps, scan, re-rank, merge)
 * iters times back to back on the index's stream and waits. stage_ms, if
 * not NULL, receives the summed device time of each stage over the iters
 * (4 floats: bitmap, scan, rerank, merge); *total_ms the whole. */
int pv_batch_run(PvBatch *b, int iters, float *stage_ms, float *total_ms, char *errbuf,
                 size_t errlen);

/* Copies the last run's results to the caller (layout of fv_gpu_brute_batch). */
int pv_batch_fetch(PvBatch *b, FvHit *out, uint32_t *out_cnt, uint8_t *truncated,
                   char *errbuf, size_t errlen);

void pv_batch_free(PvBatch *b);

/* Exact top-topb WITHOUT a predicate that allocates no device memory.
 * No counterpart in the reference: it exists for callers that must not
 * allocate on the device while serving, because cudaMalloc synchronizes
 * the whole device (a latency-bound serving loop cannot pay that per call)
 * or because a framework that owns the device's memory forbids raw
 * allocations. Scratch comes from one 2 MiB array linked into the library
 * (held on every device that loads it until the process exits).
 * d_queries (nq x dim f32), d_out (nq x topb FvHit) and d_cnt (nq u32) are
 * DEVICE pointers on g's device, allocated by the caller however it may;
 * results have the layout and order of fv_gpu_brute_batch (exact FP32).
 * The call reads d_queries on the index's own stream, which does not wait
 * for the caller's streams: the queries must be complete on the device
 * before the call (e.g. synchronize the stream that wrote them first).
 * Limits: nq <= PV_NOALLOC_MAX_BATCH, topb <= PV_NOALLOC_MAX_TOPB, else -1
 * with a message. The first call on a device looks up the array's device
 * address, so make it before any stream capture. All calls share the array:
 * calls that overlap on the GPU race and must be serialized by the caller.
 * Synchronous: returns after the results are in d_out / d_cnt. */
#define PV_NOALLOC_MAX_BATCH 32
#define PV_NOALLOC_MAX_TOPB 32
int pv_brute_batch_noalloc(FvGpuIndex *g, int nq, const float *d_queries, uint32_t topb,
                           FvHit *d_out, uint32_t *d_cnt, char *errbuf, size_t errlen);

/* ---- HNSW construction (host, multi-threaded) ----
 * Builds the graph sections of a PAVES index file for count x dim rows
 * (kept borrowed during the call): M = upper-level degree, 2M at level 0,
 * ef_construction beam width, threads <= 0 = all cores. Same construction
 * as the engine's builder (engine_api.h:45 fv_builder_finish), so files
 * written from it open in the engine. NULL + errbuf on bad parameters. */
typedef struct PvHnsw PvHnsw;
PvHnsw *pv_hnsw_build(const float *vectors, uint64_t count, int dim, int M,
                      int ef_construction, int threads, char *errbuf, size_t errlen);
void pv_hnsw_free(PvHnsw *h);
/* M, top level, entry node and the number of u32 upper-level slots. */
int pv_hnsw_info(const PvHnsw *h, uint32_t *M, int *max_level, uint64_t *entry,
                 uint64_t *upper_len);
/* Copies the sections: l0 [count][2M+1], levels [count], upper_offs
 * [count+1], upper [upper_len] (any pointer may be NULL). */
int pv_hnsw_export(const PvHnsw *h, uint32_t *l0, uint8_t *levels, uint64_t *upper_offs,
                   uint32_t *upper);
/* The same sections built on the GPU (no counterpart in the reference,
 * whose builder is CPU-only, engine_api.h:45 fv_builder_finish): every
 * level from exact nearest neighbours instead of insertion-time beam
 * searches. Per level, each node's `candidates` nearest nodes of that level
 * (this library's exact scans, the nodes as queries; BF16 tensor cores when
 * certified exact, precision FV_GPU_PREC_BF16, else FP32), the
 * neighbour-selection rule (keep a candidate closer to the node than to
 * every kept neighbour) to 2M at level 0 / M above, reverse edges, and the
 * rule again over forward + reverse candidates. Node levels are drawn as
 * the host builder draws them; the entry node is the lowest-numbered node
 * of the top level. The graph differs from the host builder's; it is
 * searched by the same code. candidates in [2M, 1023]; NULL + errbuf on
 * bad parameters or a device error. */
PvHnsw *pv_hnsw_build_gpu(const float *vectors, uint64_t count, int dim, int M, int candidates,
                          int device, int precision, char *errbuf, size_t errlen);
/* Level-0 entry point per query by greedy descent through the upper levels
 * (engine_api.h:199 fv_index_graph_entry), parallel over queries. */
int pv_hnsw_entries(const float *vectors, int dim, const uint64_t *upper_offs,
                    const uint32_t *upper, uint32_t M, int max_level, uint64_t entry,
                    const float *queries, int nq, uint32_t *out, int threads);

/* ---- GPU worker micro-batch loop (request slots + one worker thread) ----
 * Replaces the PostgreSQL background worker and shared-memory arbiter of
 * the reference (arbiter.h:106-162 FvArbSlot/FvArbiter, arbiter.h:253
 * paves_arbiter_submit, worker.c:149-598) for a process that serves from
 * several threads. Backends call pv_arbiter_submit from any thread; one
 * worker thread gathers SUBMITTED slots for up to wait_us (leaving after
 * idle_us without arrivals), groups them by (relid, strategy), runs one
 * batch per group through the executor (fv_gpu_brute_batch /
 * fv_gpu_graph_batch unless replaced) and answers each slot. */
#define PV_ARB_MAX_DIM 2000
#define PV_ARB_MAX_NODES 48
#define PV_ARB_MAX_CHILDREN 96
#define PV_ARB_MAX_INVALS 128
#define PV_ARB_MAX_SPANS 128
#define PV_ARB_MAX_RESULTS 1024
#define PV_STRAT_GPU_BRUTE 3 /* paves.h:48 FV_STRAT_GPU_BRUTE */
#define PV_STRAT_GPU_HNSW 4  /* paves.h:49 FV_STRAT_GPU_HNSW */

typedef struct PvArbiter PvArbiter;

/* One batch as the worker hands it to an executor: the arguments of
 * fv_gpu_brute_batch (strategy PV_STRAT_GPU_BRUTE) or fv_gpu_graph_batch
 * (PV_STRAT_GPU_HNSW, qd[i].entry set, want = ef). flags = truncated /
 * exhausted per query. Returns >= 0 or -1. */
typedef struct PvArbBatch {
    FvGpuIndex *g;
    int strategy, nq, dim;
    const float *queries;
    const FvGpuQueryDesc *qd;
    const uint8_t *dedup;
    const FvGpuPredNode *nodes;
    int nnodes;
    const int32_t *children;
    int nchildren;
    const double *invals;
    int ninvals;
    const FvGpuSpan *spans;
    int nspans;
    const uint64_t *spanoff;
    int nspanoff;
    uint32_t want;
    uint64_t max_visited;
    FvHit *out;
    uint32_t *out_cnt;
    uint8_t *flags;
} PvArbBatch;
typedef int (*pv_arb_exec_fn)(void *ctx, const PvArbBatch *b);

/* nslots request slots (512 in the reference), batches of at most
 * batch_max requests; starts the worker thread. NULL on bad arguments. */
PvArbiter *pv_arbiter_create(int nslots, int batch_max, int wait_us, int idle_us);
/* Registers an index under relid: ino identifies the file (requests with
 * another ino are answered ERROR), tids[count] maps rows to heap tids (NULL
 * = row numbers), vectors/upper_offs/upper/M/max_level/entry give the upper
 * levels for the graph entry descent (upper NULL = start at entry). All
 * borrowed until pv_arbiter_destroy. 0 or -1. */
int pv_arbiter_attach(PvArbiter *a, uint32_t relid, uint64_t ino, FvGpuIndex *g,
                      const uint64_t *tids, uint64_t count, int dim, const float *vectors,
                      const uint64_t *upper_offs, const uint32_t *upper, uint32_t M,
                      int max_level, uint64_t entry);
/* Replaces the executor (NULL restores the GPU batch calls). */
void pv_arbiter_set_executor(PvArbiter *a, pv_arb_exec_fn fn, void *ctx);
/* One request; blocks until answered. Returns 1 with out[*ncnt] (node =
 * tid) and *more filled, 0 when no slot/worker is available, a capacity is
 * exceeded or the worker did not answer within timeout_ms (<= 0: 10 s) and
 * the slot was reclaimed (the caller keeps the query), -1 when the worker
 * answered ERROR (same meaning as arbiter.h:253 paves_arbiter_submit). */
int pv_arbiter_submit(PvArbiter *a, uint32_t relid, uint64_t ino, int strategy, int dim,
                      const float *query, const FvGpuPredNode *nodes, int nnodes,
                      const int32_t *children, int nchildren, const double *invals,
                      int ninvals, const FvGpuSpan *spans, int nspans, int need_eval,
                      int dedup, uint32_t want, uint64_t max_visited, int sel_permille,
                      FvHit *out, uint32_t *ncnt, uint8_t *more, int timeout_ms);
/* Batches run, requests served, requests waiting, worker alive (0/1). */
int pv_arbiter_stats(PvArbiter *a, uint64_t *batches, uint64_t *requests, uint32_t *inflight,
                     int *worker_ready);
/* Service-time EWMAs of (relid, strategy) in us (arbiter.h:80-97):
 * q_us[5] per selectivity bucket, whole batch, batch size x16. -1 if none. */
int pv_arbiter_feedback(PvArbiter *a, uint32_t relid, int strategy, uint32_t *q_us,
                        uint32_t *batch_us, uint32_t *batch_n16);
/* Failure injection on the host: the worker exits after its current batch
 * without answering it (a crashed worker); waiting backends reclaim. */
void pv_arbiter_kill_worker(PvArbiter *a);
void pv_arbiter_destroy(PvArbiter *a);

/* ---- learned router (no counterpart in the reference) ----
 * A 12 -> 64 -> 64 -> 5 MLP (ReLU; bf16 weights, fp32 accumulation) that
 * predicts per query one action: 0 = exact/low-precision scan, 1..4 =
 * graph search at ef 32, 64, 128, 256. It stands beside the reference's
 * plain rule (planner.c:185-346 cost model, exec.c:415-424 beam width),
 * which stays the fallback. Features per query (12 floats):
 *   [0] log10(selectivity) from the query's predicate bitmap popcount
 *   [1] |q|   [2..9] distances to the 8 nearest centroids, ascending
 *   [10] log2(k)   [11] predicate root kind (0 none, 1 CMP, 2 IN, 3 AND,
 *   4 OR, 5 NOT).
 * Parameters (PV_MLP_NPARAMS fp32, the optimizer's master copy): W1
 * [12][64], b1 [64], W2 [64][64], b2 [64], W3 [64][5], b3 [5], row-major
 * with the input index first. */
#define PV_MLP_IN 12
#define PV_MLP_HIDDEN 64
#define PV_MLP_OUT 5
#define PV_MLP_NPARAMS (12 * 64 + 64 + 64 * 64 + 64 + 64 * 5 + 5)
typedef struct PvRouter PvRouter;
/* centroids [ncent][dim] (8 <= ncent <= 65536) are copied to the device. */
PvRouter *pv_router_create(int device, const float *centroids, int ncent, int dim,
                           char *errbuf, size_t errlen);
void pv_router_free(PvRouter *r);
/* Sets the master weights and the feature standardization (x - mean) / std;
 * resets the optimizer state. */
int pv_router_set_params(PvRouter *r, const float *params, const float *feat_mean,
                         const float *feat_std, char *errbuf, size_t errlen);
int pv_router_get_params(PvRouter *r, float *params, float *feat_mean, float *feat_std);
/* Features of a batch on g's device (predicate arrays as fv_gpu_brute_batch,
 * k[nq] per query) -> feats [nq][12]. */
int pv_router_features(PvRouter *r, FvGpuIndex *g, int nq, const float *queries,
                       const FvGpuQueryDesc *qd, const FvGpuPredNode *nodes, int nnodes,
                       const int32_t *children, int nchildren, const double *invals,
                       int ninvals, const uint32_t *k, float *feats, char *errbuf,
                       size_t errlen);
/* Logits [n][5] of feats [n][12] (raw features; standardized inside). */
int pv_router_forward(PvRouter *r, int n, const float *feats, float *logits, char *errbuf,
                      size_t errlen);
/* Gradient of the sample-weighted mean cross-entropy over the n samples
 * with respect to the parameters (through the bf16 forward), and the loss.
 * sample_w may be NULL (all 1). */
int pv_router_grad(PvRouter *r, int n, const float *feats, const int32_t *labels,
                   const float *sample_w, float *grad, float *loss, char *errbuf,
                   size_t errlen);
/* Adam (beta 0.9/0.999, eps 1e-8) on shuffled minibatches of `batch`
 * samples, floor(n / batch) steps per epoch, each step one CUDA graph
 * launch; epoch_loss[epochs] receives the mean batch loss per epoch. */
int pv_router_train(PvRouter *r, int n, const float *feats, const int32_t *labels,
                    const float *sample_w, int epochs, int batch, float lr, uint64_t seed,
                    float *epoch_loss, char *errbuf, size_t errlen);

/* Learned-routed filtered top-k batch (no reference counterpart): builds
 * the batch's predicate bitmaps, computes the router's features and MLP
 * action per query on the device, and answers each query by the route
 * chosen for it (see split): the graph search at its beam width, or the
 * scan of the index's precision. The scan starts speculatively beside the
 * routing (a scan costs about the same for one query as for a query tile);
 * the graph search runs on a second stream, and a batch whose every query
 * went to the graph discards the scan. plan
 * (optional, replaces the router, r may then be NULL): per query 0 = scan
 * or the beam width to use. k[nq] <= topb; out has stride topb and holds
 * min(k, found) hits per query. split 0: a batch that is scanned (any
 * query routed to the scan) answers every query from the scan, which is
 * exact on certified data and already paid for; split 1: each query takes
 * its own route, graph-routed ones from the graph search run beside the
 * scan. qd[i].entry must hold the level-0 entry
 * point when the index has a graph. decided[nq] (optional) receives each
 * query's beam width (0 = scan), *executed 0 when every query was answered
 * by the scan, 1 when every query took the graph, 2 for a split batch;
 * stage_ms[3] the
 * device time of the bitmaps, of the routing (features, MLP, decision read
 * back; it runs beside the speculative scan) and of the search after the
 * bitmaps: the batch took stage_ms[0] + stage_ms[2]. */
int pv_routed_batch(FvGpuIndex *g, PvRouter *r, int nq, const float *queries,
                    const FvGpuQueryDesc *qd, const FvGpuPredNode *nodes, int nnodes,
                    const int32_t *children, int nchildren, const double *invals, int ninvals,
                    const uint32_t *k, uint32_t topb, const uint16_t *plan, float margin,
                    int split,
                    FvHit *out, uint32_t *out_cnt, uint16_t *decided, int *executed,
                    float *stage_ms, char *errbuf, size_t errlen);

/* ---- stream of uneven micro-batches (no counterpart in the reference) ----
 * For a serving loop whose batches vary in size, k and filters. At creation
 * the stream autotunes, per batch-size bucket (1, 2, 4, ... max_batch) and
 * result-width bucket (16 and max_k, or max_k alone when <= 16), the scan
 * shape (exact FP32 scan, or the index's reduced-precision tensor-core scan
 * with its epilogue groups, pipeline stages and CTA count) by timing the
 * candidates on the sample queries (tune_queries [ntune][dim]); choices are
 * read from / saved to tune_path (NULL: neither). It then captures one
 * CUDA graph per bucket: H2D of the staged batch, predicate bitmaps, scan,
 * merge, re-rank, D2H. pv_stream_run pads a batch to its bucket, replays
 * the graph and returns per query min(k[q], found) hits in out[nq][max_k]
 * ascending by (dist, id); queries whose reduced-precision superset cannot
 * be certified are re-run exactly on g, and batches whose predicates exceed
 * the bucket's capacity (8 instructions and 8 IN values per query on
 * average) run through g's ordinary path. *device_ms: the graph's device
 * time. g must outlive the stream; calls on one stream are serialized. */
#define PV_STREAM_MAX_K 256
typedef struct PvStream PvStream;
PvStream *pv_stream_create(FvGpuIndex *g, int max_batch, uint32_t max_k,
                           const float *tune_queries, int ntune, const char *tune_path,
                           char *errbuf, size_t errlen);
int pv_stream_run(PvStream *s, int nq, const float *queries, const FvGpuQueryDesc *qd,
                  const FvGpuPredNode *nodes, int nnodes, const int32_t *children,
                  int nchildren, const double *invals, int ninvals, const uint32_t *k,
                  FvHit *out, uint32_t *out_cnt, float *device_ms, char *errbuf,
                  size_t errlen);
/* Bucket i's size, width and tuned plan (mode PV_MODE_EXACT / PV_MODE_LOW,
 * epilogue groups, stages, CTAs along the rows; 0 = built-in) and measured
 * ms; returns the number of buckets (i < 0: just the number). */
int pv_stream_info(PvStream *s, int i, int *B, uint32_t *topb, int *mode, int *epi, int *ns,
                   int *grow, float *tuned_ms);
/* Queries of the last run re-run exactly; 1 if it bypassed the graphs. */
int pv_stream_last(PvStream *s, int *uncertain, int *fallback);
void pv_stream_free(PvStream *s);

/* ---- persistent micro-batch kernel (no counterpart in the reference) ----
 * The reference worker answers each micro-batch with separate synchronous
 * launches (worker.c:268-276, loop worker.c:453-598). A PvServe keeps ONE
 * cooperative kernel (one CTA per SM) resident on g's device, started from
 * a captured CUDA graph when the runtime allows the capture (else launched
 * directly), and feeds it a queue of staged micro-batches: uneven sizes
 * (1..max_batch), a k per query (<= max_k) and a filter per query. Each
 * batch runs inside the kernel as grid-synchronous phases (query prep,
 * predicate bitmaps unless every filter is broad, seeding pass and merge,
 * the tensor-core main pass, merge and exact re-rank) and its results are
 * written into host-mapped memory. Every wait of the kernel is bounded by
 * the GPU clock: the wait for the next batch by idle_ms (the kernel then
 * leaves; the next pv_serve_run starts it again), each grid barrier by a
 * limit after which the kernel leaves with a failure status (pv_serve_run
 * returns -1 with "wait expired"), the scan's own waits as in the one-shot
 * kernel. g must be a BF16 or FP8 upload and outlive the server; while the
 * kernel is resident it holds every SM of the device, so other work on the
 * device waits for it to leave (pv_serve_stop, or idle_ms without a batch).
 * Batches beyond the capacities, and queries whose reduced-precision
 * superset cannot be certified, run on g's ordinary path with the kernel
 * stopped. out[nq][max_k] holds min(k, found) hits per query ascending by
 * (dist, id); *device_ms the batch's time inside the kernel (GPU clock from
 * taking the batch to its completion word). NULL / -1 + errbuf on error. */
#define PV_SERVE_MAX_K 256
typedef struct PvServe PvServe;
PvServe *pv_serve_create(FvGpuIndex *g, int max_batch, uint32_t max_k, uint32_t idle_ms,
                         char *errbuf, size_t errlen);
int pv_serve_run(PvServe *s, int nq, const float *queries, const FvGpuQueryDesc *qd,
                 const FvGpuPredNode *nodes, int nnodes, const int32_t *children, int nchildren,
                 const double *invals, int ninvals, const uint32_t *k, FvHit *out,
                 uint32_t *out_cnt, float *device_ms, char *errbuf, size_t errlen);
/* running (the kernel is resident), last_exit of the last kernel (0 stopped
 * or never started, 1 left after idle_ms without a batch, -1 a wait
 * expired), batches completed, graph_launch (1: started from the captured
 * graph), and for the last batch: fallback (ran on g's ordinary path),
 * uncertain (queries re-run exactly). */
int pv_serve_status(PvServe *s, int *running, int *last_exit, uint64_t *batches,
                    int *graph_launch, int *fallback, int *uncertain);
/* Stops the kernel (it leaves before its next batch) and waits for it. */
int pv_serve_stop(PvServe *s, char *errbuf, size_t errlen);
/* Limits for the next start: idle_ms, the grid-barrier limit barrier_ms,
 * and skip_cta >= 0, which makes that CTA skip its arrival at the first
 * barrier of the next batch (a failure made on the host side of the
 * barrier protocol: the other CTAs' bounded waits expire; -1 none).
 * Stops a resident kernel. -1 on bad values. */
int pv_serve_limits(PvServe *s, uint32_t idle_ms, uint32_t barrier_ms, int skip_cta);
void pv_serve_free(PvServe *s);

/* Device time (ms) of the kernels of the last synchronous batch call on g. */
float pv_last_kernel_ms(const FvGpuIndex *g);

/* Candidates per query the last reduced-precision scan on g re-ranked in
 * exact FP32 (4 x topb, or topb when its BF16 distances were certified
 * exact: integer rows and queries with all sums below 2^24); 0 if none. */
int pv_last_superset(const FvGpuIndex *g);

/* Queries of the last reduced-precision batch call on g whose candidate
 * superset the merge could not certify complete (a per-CTA candidate list
 * of 64 filled up below the superset's last key). fv_gpu_brute_batch and
 * pv_routed_batch re-run those queries with the exact scan; pv_batch_fetch
 * only reports them. */
int pv_last_uncertain(const FvGpuIndex *g);

/* Selective filters: a batch whose queries share one filter that the
 * index's sorted attribute values bound to at most max(4096, count / 16)
 * matching rows scans only those rows (the bitmap compacted to a row list,
 * then the exact FP32 scan over the list) — the reference's posting-list
 * driver route (engine.cpp:464-599, gpu_engine.cu:2249-2260). Results are
 * those of the full scan. pv_last_sparse: 1 if the last brute batch on g
 * took this route. pv_filter_bound: the bound for one filter (node 0 is
 * the root; nnodes 0 = no filter -> count). */
int pv_last_sparse(const FvGpuIndex *g);
/* Stored device layout. No reference counterpart: the reference converts
 * its rows at every upload (gpu_engine.cu:1692-1773). The low-precision
 * rows ([count][kpad], kpad = dim rounded up to 64 for BF16 / 128 for FP8),
 * their norms and FP8 scales (f32 [count]) are read back with
 * pv_index_export (PV_PART_*; pv_index_part_bytes gives each part's size,
 * -1 if the index has no such part) and stored beside the index file; a
 * later pv_index_upload_prepared copies them back instead of converting,
 * and takes the stored row_amax (the BF16 exactness certificate's input)
 * instead of scanning every row on the host. Arguments otherwise as
 * fv_gpu_index_upload; NULL on error with the message in errbuf. */
enum { PV_PART_LOWP_ROWS = 1, PV_PART_NORMS = 2, PV_PART_SCALES = 3 };
int64_t pv_index_part_bytes(const FvGpuIndex *g, int part);
int pv_index_export(FvGpuIndex *g, int part, void *dst, uint64_t bytes, float *row_amax,
                    char *errbuf, size_t errlen);
FvGpuIndex *pv_index_upload_prepared(const float *vectors, const double *cols,
                                     const uint32_t *post_rows, const uint32_t *l0,
                                     uint32_t l0_stride, uint64_t count, int dim, int ncols,
                                     int device, int precision, const void *vlow,
                                     const float *norms, const float *scales, float row_amax,
                                     char *errbuf, size_t errlen);

/* Shape of the tensor-core scan for later batches on g (0 = automatic):
 * epilogue warp groups (1, 2, 3), pipeline stages (2..8), CTAs along rows per
 * query tile, query replicas down the tile (1, 2, 4; capped so that each
 * replica's share of a 128-row tile is at least 32 rows), seeding pass
 * (1 = always when the index has 8+ tiles per CTA, 2 = never; the main
 * pass then bounds itself from its own lists). -1: bad value. */
int pv_tc_shape(FvGpuIndex *g, int epi, int ns, int grow, int rep, int seed);
/* on = 1: later reduced-precision batches on g re-rank 4 x topb candidates
 * even when the BF16 distances are certified exact (the superset that
 * inexact distances need); 0 restores the certified width. -1: bad value. */
int pv_tc_wide_superset(FvGpuIndex *g, int on);
/* Limit (ns, at most 10 s; 0 = the default 2 s) after which a wait of the
 * tensor-core scan gives up: the kernel records which role gave up, waits
 * (up to 2 s, whatever this limit) for the copies and MMAs it issued,
 * frees its tensor memory and returns, and the batch call returns -1 with
 * "wait expired" in errbuf; the index stays usable. -1: bad value. */
int pv_tc_timeout(FvGpuIndex *g, uint64_t ns);
/* Exact-mode batches (FP32 uploads through fv_gpu_brute_batch, or
 * PV_MODE_EXACT) of 16+ queries over rows of at most 128 dims scan on the
 * tensor cores: the f32 rows read as TF32, the top 4 x topb (at least 16;
 * topb itself on integer rows, where the distances are exact) re-ranked in
 * FP32, and each query's answer certified by an error bound of the scan
 * distances; a query the bound cannot separate is re-run on the CUDA-core
 * scan. on = 0 keeps every exact batch on the CUDA cores. -1: bad value.
 * pv_last_exact_tc: 1 if the last brute batch on g took the tensor cores. */
int pv_exact_tc(FvGpuIndex *g, int on);
int pv_last_exact_tc(const FvGpuIndex *g);
int pv_filter_bound(const FvGpuIndex *g, const FvGpuPredNode *nodes, int nnodes,
                    const int32_t *children, int nchildren, const double *invals, int ninvals,
                    uint64_t *bound, char *errbuf, size_t errlen);

/* Kernels launched by the last batch call on g (summed over the iterations
 * of pv_batch_run). */
int pv_last_launches(const FvGpuIndex *g);

/* Counters of the last fv_gpu_graph_batch call: per query [steps, visited,
 * predicate probes, results]; copies min(nq, last nq) rows, returns rows. */
int pv_graph_stats(const FvGpuIndex *g, uint32_t *out, int nq);

#ifdef __cplusplus
}
#endif
#endif /* PAVES_B200_EXT_H */
