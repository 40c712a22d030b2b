/*
 * paves_gpu.h — the drop-in C ABI of libpaves_gpu.so.
 *
 * These are the entry points the PAVES engine (engine.cpp) binds when it is
 * built with -DFV_GPU. Each one replaces the function of the same name in
 * the reference CUDA backend; the citation beside each declaration names the
 * reference interface (extension/paves/src/engine/gpu_engine.h) it stands in
 * for. Struct layouts are byte-compatible with the reference's
 * engine_api.h / gpu_engine.h so an unmodified engine.cpp links against this
 * library and passes the same arrays.
 *
 * Everything here is plain C: host pointers and sizes only. Calls are
 * synchronous (they return after results are in the caller's buffers) and
 * serialized per index handle. A CUDA context is created lazily on the first
 * upload, so it always happens after fork().
 *
 * If the including translation unit has already seen the reference's
 * engine_api.h (PAVES_ENGINE_API_H defined), the shared structs are taken
 * from there; otherwise they are declared below with identical layout.
 */
#ifndef PAVES_B200_GPU_H
#define PAVES_B200_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifndef PAVES_ENGINE_API_H
/* Predicate node kinds and comparison operators (engine_api.h:69-70). */
enum { FV_CMP_LT, FV_CMP_LE, FV_CMP_EQ, FV_CMP_GE, FV_CMP_GT, FV_CMP_NE };
enum { FV_NODE_CMP, FV_NODE_IN, FV_NODE_AND, FV_NODE_OR, FV_NODE_NOT };

/* Flattened predicate node (engine_api.h:102-112), 40 bytes. Children and IN
 * values are ranges [child0, child0+nchildren) / [val0, val0+nvalues) into
 * the side arrays; a column value that is NaN compares false everywhere. */
typedef struct FvGpuPredNode {
    int32_t kind;
    int32_t col;
    int32_t op;
    int32_t nchildren;
    int32_t child0;
    int32_t nvalues;
    int32_t val0;
    int32_t pad;
    double value;
} FvGpuPredNode;

/* Posting-list span [lo, hi) of column col (engine_api.h:114-117), 12 B. */
typedef struct FvGpuSpan {
    int32_t col;
    uint32_t lo, hi;
} FvGpuSpan;

/* One result row: node id and SQUARED L2 distance (engine_api.h:145-148). */
typedef struct FvHit {
    uint64_t node;
    float dist;
} FvHit;
#endif /* PAVES_ENGINE_API_H */

#ifndef PAVES_GPU_ENGINE_H
typedef struct FvGpuIndex FvGpuIndex;

/* Device precision of the resident vectors (gpu_engine.h:33-34 for FP32 and
 * SQ8; BF16 and FP8 are additions with new numbers, nothing is renumbered).
 *   FP32: exact scan; ids ordered by (distance, id).
 *   SQ8:  the reference's approximate mode; served here by the BF16 scan with
 *         an exact FP32 re-rank (results approximate by contract).
 *   BF16: bf16 tensor-core distances + exact FP32 re-rank of a superset.
 *   FP8:  fp8-e4m3 per-vector-scaled distances + exact FP32 re-rank. */
#define FV_GPU_PREC_FP32 0
#define FV_GPU_PREC_SQ8 1

/* Caps (gpu_engine.h:36-44); requests beyond them return -1. */
#define FV_GPU_MAX_TOPB 4096
#define FV_GPU_MAX_SPANS 4096
#define FV_GPU_MAX_EF 512
#define FV_GPU_MAX_BATCH 1024

/* Per-query descriptor (gpu_engine.h:52-60), 32 bytes. proot is the query's
 * root node in the concatenated predicate arrays (-1 = no predicate); spans
 * of the query are spans[span0 .. span0+nspans) with prefix offsets at
 * spanoff[soff0 ..]; entry is the graph-search level-0 entry point; total is
 * the brute enumeration size. */
typedef struct FvGpuQueryDesc {
    int32_t proot;
    int32_t need_eval;
    int32_t span0;
    int32_t nspans;
    int32_t soff0;
    uint32_t entry;
    uint64_t total;
} FvGpuQueryDesc;
#endif /* PAVES_GPU_ENGINE_H */

#define FV_GPU_PREC_BF16 2
#define FV_GPU_PREC_FP8 3

/* Replaces fv_gpu_available (gpu_engine.h:63): 1 if a usable CUDA device
 * exists in this process. */
int fv_gpu_available(void);

/* Replaces fv_gpu_index_upload (gpu_engine.h:69-73). Copies the rows
 * (count x dim f32), the scalar columns (ncols x count f64, column-major),
 * the posting rows (ncols x count u32) and, when l0 != NULL, the level-0
 * adjacency (count x l0_stride u32, [cnt, neighbours...]) into the
 * device-resident layout. device -1 picks the device with the most free
 * memory. precision is FV_GPU_PREC_*. NULL + errbuf on failure. */
FvGpuIndex *fv_gpu_index_upload(const float *vectors, const double *cols,
                                const uint32_t *post_rows,
                                const uint32_t *l0, uint32_t l0_stride,
                                uint64_t count, int dim, int ncols, int device,
                                int precision, char *errbuf, size_t errlen);

/* Replaces fv_gpu_index_free (gpu_engine.h:74). NULL is a no-op. */
void fv_gpu_index_free(FvGpuIndex *g);

/* Replaces fv_gpu_index_device (gpu_engine.h:75). */
int fv_gpu_index_device(const FvGpuIndex *g);

/* Replaces fv_gpu_index_precision (gpu_engine.h:76). */
int fv_gpu_index_precision(const FvGpuIndex *g);

/* Replaces fv_gpu_brute_batch (gpu_engine.h:86-94). Filtered top-topb for
 * nq queries: out[q*topb ..] ascending by (dist, node), out_cnt[q] entries,
 * truncated[q] nonzero when more passing rows exist than were returned.
 * With FV_GPU_PREC_FP32 the result is exact. Returns 0, or -1 + errbuf. */
int fv_gpu_brute_batch(FvGpuIndex *g, int nq, const float *queries,
                       const FvGpuQueryDesc *qd, const uint8_t *dedup,
                       const FvGpuPredNode *nodes, int nnodes,
                       const int32_t *children, int nchildren,
                       const double *invals, int ninvals,
                       const FvGpuSpan *spans, int nspans_total,
                       const uint64_t *spanoff, int nspanoff, uint32_t topb,
                       FvHit *out, uint32_t *out_cnt, uint8_t *truncated,
                       char *errbuf, size_t errlen);

/* Replaces fv_gpu_graph_batch (gpu_engine.h:104-109). Filtered level-0 beam
 * search from qd[q].entry; traversal is unrestricted, only predicate-passing
 * nodes are results (ef <= FV_GPU_MAX_EF). out[q*ef ..] ascending by
 * (dist, node); exhausted[q] nonzero when a larger ef cannot add results.
 * Returns 0, or -1 + errbuf. */
int fv_gpu_graph_batch(FvGpuIndex *g, int nq, const float *queries,
                       const FvGpuQueryDesc *qd, const FvGpuPredNode *nodes,
                       int nnodes, const int32_t *children, int nchildren,
                       const double *invals, int ninvals, uint32_t ef,
                       uint64_t max_visited, FvHit *out, uint32_t *out_cnt,
                       uint8_t *exhausted, char *errbuf, size_t errlen);

/* Replaces fv_gpu_tile_variant_qt (engine_api.h:194): the query-tile width
 * the batched scan uses for this dimension (0 = unsupported dimension). */
int fv_gpu_tile_variant_qt(int dim);

/* Replaces fv_gpu_mem_probe (engine_api.h:195): free/total bytes of the
 * best device; returns the device id or -1. */
int fv_gpu_mem_probe(uint64_t *free_bytes, uint64_t *total_bytes);

#ifdef __cplusplus
}
#endif
#endif /* PAVES_B200_GPU_H */
