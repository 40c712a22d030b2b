// pv_internal.h — declarations shared between the library's sources.
#pragma once

#include "index.h"

float pv_integral_amax(const float *v, uint64_t n);
bool pv_bf16_exact(int dim, float row_amax, float q_amax);

namespace pv {

FvGpuIndex *index_view(const FvGpuIndex *g);  // index.cu
// raises (never lowers) fn's dynamic shared-memory limit on this device
cudaError_t raise_smem_limit(const void *fn, size_t bytes);  // index.cu

// ---- predicates (pred.cpp, bitmap.cu)
int compile_predicates(int nq, const int32_t *proot, size_t proot_stride,
                       const FvGpuPredNode *nodes, int nnodes, const int32_t *children,
                       int nchildren, const double *invals, int ninvals, int ncols,
                       PredBatch &pb, char *errbuf, size_t errlen);
cudaError_t launch_bitmaps(const double *cols, uint64_t nrows, const PredInsn *insns,
                           const PredProg *progs, const double *consts, int P,
                           uint32_t *bitmaps, uint64_t bm_words, unsigned long long *popcnt,
                           int sm_count, cudaStream_t st, int ninsns, int nconsts,
                           int ncols = 1 << 30, bool one_range = false);
// Same, with the batch's {P, ninsns, nconsts} read on the device from
// dcounts (each at most its cap): one launch shape for a CUDA graph.
cudaError_t launch_bitmaps_capped(const double *cols, uint64_t nrows, const PredInsn *insns,
                                  const PredProg *progs, const double *consts,
                                  const int *dcounts, int P_cap, int insn_cap, int const_cap,
                                  uint32_t *bitmaps, uint64_t bm_words,
                                  unsigned long long *popcnt, int sm_count, cudaStream_t st,
                                  int ncols = 1 << 30);

// ---- per-query top-KO of dense key runs (scan_tc.cu): keys of query q are
// dense[q][0 .. dcnt[q]) (<= dcap), at most the bound tau[q] (tau null: no
// bound); KO <= 1024. Writes out [nq][KO] ascending, out_cnt, trunc (from
// popcnt[qprog[q]] or nrows), tau_out[q] = min(tau_out[q], KO-th key) and
// unc[q] (a full list's last key, fullmin[q], at or below the answer's end).
cudaError_t launch_dense_merge(const uint64_t *dense, uint64_t dcap, uint32_t *dcnt,
                               bool reset_cnt, const unsigned long long *fullmin,
                               const unsigned long long *tau, int KO, const int32_t *qprog,
                               const unsigned long long *popcnt, uint64_t nrows, int nq,
                               FvHit *out, uint32_t *out_cnt, uint8_t *trunc,
                               unsigned long long *tau_out, uint8_t *unc, cudaStream_t st);

// ---- exact FP32 scan (scan_f32.cu)
struct ScanF32Args {
    const float *__restrict__ vecs;
    uint64_t nrows;
    int dpad;
    const float *__restrict__ queries;  // [nq][dpad]
    int nq;
    const uint32_t *__restrict__ bitmaps;  // [P][bm_words]
    uint64_t bm_words;
    const int32_t *__restrict__ qprog;  // [nq]
    int K, S, CB;
    uint64_t rows_per_cta;  // multiple of 32
    int grow;               // CTAs along the rows
    int qtiles;
    unsigned long long *tau;  // [nq]
    uint64_t *part;           // [nq][grow][K]
    uint32_t *part_cnt;       // [nq][grow]
};

struct ScanPlan {
    int QT, DCH, S, CB, grow, qtiles;
    uint64_t rows_per_cta;
    size_t smem;
    int M;  // merge buffer (keys)
    size_t merge_smem;
};

int scan_f32_max_qt(int dim);
// min_rows: rows per CTA at least
bool plan_scan_f32(uint64_t nrows, int dpad, int nq, int K, int sm_count, ScanPlan &pl,
                   uint64_t min_rows = 2048);
cudaError_t launch_scan_f32(const ScanF32Args &a, const ScanPlan &pl, cudaStream_t st);
// register-blocked exact scan for query tiles of 32 / 64 (scan_f32t.cu):
// false when the batch is too small, K > 64 or dpad > 256
bool plan_scan_f32t(uint64_t nrows, int dpad, int nq, int K, int sm_count, ScanPlan &pl);
cudaError_t launch_scan_f32t(const ScanF32Args &a, const ScanPlan &pl, cudaStream_t st);
cudaError_t launch_merge(const uint64_t *part, const uint32_t *part_cnt, int grow, int K,
                         const ScanPlan &pl, const unsigned long long *tau,
                         const int32_t *qprog, const unsigned long long *popcnt,
                         uint64_t nrows, int nq, FvHit *out, uint32_t *out_cnt,
                         uint8_t *trunc, cudaStream_t st,
                         unsigned long long *tau_out = nullptr, int kout = 0,
                         uint8_t *unc = nullptr, int kuse = 0);

// ---- batch staging (brute.cu)
struct DevBatch {
    Buf *stage_h = nullptr;
    Buf *stage_d = nullptr;
    int nq = 0, P = 0, ninsns = 0, nconsts = 0;
    size_t off_q = 0, off_qprog = 0, off_progs = 0, off_insns = 0, off_consts = 0, off_extra = 0;
    size_t bytes = 0;
    float q_amax = -1.f;  // max |q| if all queries are integers <= 256, else -1
    // {P, ninsns, nconsts} also staged at off_counts: P / ninsns / nconsts
    // above are then capacities and the bitmap kernel reads the counts
    bool counts_on_device = false;
    size_t off_counts = 0;
    // sparse route: every query uses program 0, whose matches are at most
    // sparse_bound rows (0 = dense)
    uint64_t sparse_bound = 0;
    // one program in range form whose terms are all well formed (constants
    // in the pool, columns in the table): the lean bitmap kernel
    bool one_range = false;
};

int brute_prepare(FvGpuIndex *g, int nq, const float *queries, const PredBatch &pb,
                  DevBatch &db, size_t extra_bytes, char *errbuf, size_t errlen);
int brute_upload(FvGpuIndex *g, DevBatch &db, char *errbuf, size_t errlen);
// ev (optional): 5 events recorded before bitmaps, before scan, after scan,
// after re-rank and after merge. bm_done (with bitmaps_ready: the caller's
// bitmap kernel is the last launch on the stream): recorded once the
// bitmaps are complete (behind query prep, which runs beside them, on the
// tensor-core routes). bitmaps_ready: the batch's bitmaps and
// popcounts are already in g->scan (no bitmap launch).
int brute_launch(FvGpuIndex *g, DevBatch &db, uint32_t topb, int mode, FvHit *d_out,
                 uint32_t *d_cnt, uint8_t *d_trunc, char *errbuf, size_t errlen,
                 cudaEvent_t *ev = nullptr, bool bitmaps_ready = false,
                 cudaEvent_t bm_done = nullptr);
// Re-runs exactly the queries with unc[q] != 0 on g (host buffers; call with
// g->mu held) and writes their results over out / out_cnt / truncated.
int redo_flagged(FvGpuIndex *g, int nq, const float *queries, const PredBatch &pb,
                 uint32_t topb, const uint8_t *unc, FvHit *out, uint32_t *out_cnt,
                 uint8_t *truncated, char *errbuf, size_t errlen);
// ---- selective filters (sparse.cu)
// Filters bounded by at most this many rows take the sparse route: exact
// distances of the listed rows cost less than a full scan below ~1/16 of
// the index.
inline uint64_t sparse_limit(uint64_t nrows) { return nrows / 16 > 4096 ? nrows / 16 : 4096; }
void build_sorted_cols(FvGpuIndex *g, const double *cols, const uint32_t *post_rows);
uint64_t prog_upper_bound(const FvGpuIndex *g, const PredInsn *ins, int n, const double *consts);
double prog_pass_estimate(const FvGpuIndex *g, const PredInsn *ins, int n, const double *consts);
// lazy filters pay one filter test per row that beats the threshold; a
// selective filter leaves a loose threshold (few passing rows), so only
// programs estimated to pass at least this fraction are tested lazily
constexpr double PV_LAZY_MIN_PASS = 0.125;
// Sparse batches whose filter matches at least this many rows (bounded on
// the host) scan their compacted rows on the tensor cores when the batch's
// mode can (sparse_tc_launch); smaller ones compute every listed row's
// exact distance on the CUDA cores (sparse_launch). Measured at batch 64
// over 1M rows: at a bound of 10,000 rows both routes took 0.078 ms (1 %
// filter), at ~1,000 matching rows the CUDA-core route was faster (0.040
// vs 0.064 ms); a compacted pass pays its warm-up admissions on every
// tile, since it has too few tiles for a seeding pass.
constexpr uint64_t PV_SPARSE_TC_MIN_ROWS = 16384;
int sparse_tc_launch(FvGpuIndex *g, DevBatch &db, uint32_t topb, uint64_t bound, bool tf32,
                     FvHit *d_out, uint32_t *d_cnt, uint8_t *d_trunc, cudaEvent_t *ev,
                     char *errbuf, size_t errlen);
int sparse_launch(FvGpuIndex *g, DevBatch &db, uint32_t topb, uint64_t bound, FvHit *d_out,
                  uint32_t *d_cnt, uint8_t *d_trunc, char *errbuf, size_t errlen);
int tc_redo_uncertain(FvGpuIndex *g, int nq, const float *queries, const PredBatch &pb,
                      uint32_t topb, FvHit *out, uint32_t *out_cnt, uint8_t *truncated,
                      char *errbuf, size_t errlen);
int brute_run_host(FvGpuIndex *g, int nq, const float *queries, const PredBatch &pb,
                   uint32_t topb, int mode, FvHit *out, uint32_t *out_cnt,
                   uint8_t *truncated, char *errbuf, size_t errlen);

// ---- tensor-core scan (scan_tc.cu)
bool tc_shape_fits(const FvGpuIndex *g, uint32_t topb, int epi, int ns);
int tc_superset(const FvGpuIndex *g, uint32_t topb, float q_amax);
bool tc_supported(const FvGpuIndex *g);
int tf32_superset(const FvGpuIndex *g, uint32_t topb, float q_amax);
bool tf32_supported(const FvGpuIndex *g);
// Exact-mode batches of at least this many queries scan on the tensor cores
// (f32 rows read as TF32 + certified exact re-rank); smaller ones stream
// the f32 rows through the CUDA cores, bandwidth-bound either way.
constexpr int PV_EXACT_TC_MIN_NQ = 16;
// internal brute mode: exact on the CUDA cores only (the re-run of queries
// the tensor-core scan could not certify)
constexpr int PV_MODE_SIMT = 2;
// Lazy filters for the tensor-core scan: *flag (device memory, read when
// the kernel runs) != 0 means the batch has no bitmaps and every program is
// in range form; the scan then evaluates a query's program only for rows
// whose key beats its threshold (truncation flags are not computed).
struct TcLazy {
    const int *flag;
    const PredProg *progs;
    const PredInsn *insns;
    const double *consts;
    int nconsts;
};
// A compacted row set for the tensor-core scan (the sparse route): nrows
// rows (a multiple of 128) in the scan's operand layout (low-precision rows
// of kpad elements, or f32 rows of dpad), their norms (and fp8 scales), and
// the index row of each (keys carry the index row). The batch's bitmaps
// then mark which compacted rows are valid.
struct TcRowSet {
    const void *rows;
    const float *norms;
    const float *scales;
    uint64_t nrows;
    const uint32_t *rowids;
    const unsigned long long *nrows_dev;  // rows that exist (device), <= nrows
};
int launch_scan_tc(FvGpuIndex *g, int nq, float q_amax, const float *d_q,
                   const int32_t *d_qprog,
                   const uint32_t *bitmaps, uint64_t bm_words,
                   const unsigned long long *popcnt, uint32_t topb, FvHit *d_out,
                   uint32_t *d_cnt, uint8_t *d_trunc, cudaEvent_t *ev, char *errbuf,
                   size_t errlen, const TcLazy *lz = nullptr, bool tf32 = false,
                   const TcRowSet *rs = nullptr, bool behind_bitmaps = false,
                   cudaEvent_t prep_done = nullptr);
// behind_bitmaps: the last launch on the stream is this batch's bitmap
// kernel (query prep then runs beside it); prep_done: recorded behind
// query prep
// Reads and clears the watchdog word of the last tensor-core scan after the
// stream was synchronized; -1 + errbuf if a bounded wait expired.
int check_tc_watchdog(FvGpuIndex *g, char *errbuf, size_t errlen);
// Queues the watchdog word's copy into pinned h_word on g's stream (after
// the results' copy); the next check_tc_watchdog reads it there.
void tc_watchdog_enqueue(FvGpuIndex *g, int *h_word);

// ---- HNSW sections (hnsw_build.cpp) for the GPU builder (hnsw_gpu.cu)
}  // namespace pv
typedef struct PvHnsw PvHnsw;
namespace pv {
PvHnsw *hnsw_sections(const float *vectors, uint64_t count, int dim, int M);
const uint8_t *hnsw_levels(const PvHnsw *h);
uint32_t *hnsw_l0(PvHnsw *h);
uint32_t *hnsw_upper_list(PvHnsw *h, uint64_t node, int level);
void hnsw_set_entry(PvHnsw *h, uint64_t entry, int level, int efc);

// ---- graph search (graph.cu)
// ---- graph search (graph.cu)
struct GraphOut {
    size_t off_cnt, off_exh, off_st, bytes;  // hits at 0, then counts, exhausted, stats
};
GraphOut graph_out_layout(int nq, uint32_t ef);
// Launches the beam search of nq staged queries on g's stream (bitmaps of
// the batch already in g->scan.bitmaps); d_efq (optional) gives per-query
// ef <= ef; outputs land in od with layout lo.
int graph_launch(FvGpuIndex *g, int nq, const float *d_q, const uint32_t *d_entries,
                 const int32_t *d_qprog, const uint16_t *d_efq, uint32_t ef,
                 uint64_t max_visited, char *od, const GraphOut &lo, char *errbuf,
                 size_t errlen, cudaStream_t st = nullptr);
int graph_run_host(FvGpuIndex *g, int nq, const float *queries, const uint32_t *entries,
                   const PredBatch &pb, uint32_t ef, uint64_t max_visited, FvHit *out,
                   uint32_t *out_cnt, uint8_t *exhausted, char *errbuf, size_t errlen);

}  // namespace pv
